"""The CPU oracle against the reference itself (CPU only).

The golden fixtures were produced by the reference's own kernel sources
(tests/golden/make_golden.py through oracle/refk_harness.c).  The oracle
restates the reference's arithmetic in the same order and literal types, so
it must reproduce them bit for bit, in FP64 and in FP32.
"""
import numpy as np
import pytest

import pyoracle as po
from _golden import golden_names, load

NAMES = golden_names()


def test_goldens_present():
    assert len(NAMES) >= 15


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_golden(name):
    p, z = load(name)
    f = z["f0"].copy()
    f, mv = po.run_oracle(p, f, z["solids"], 0, int(z["steps"]), int(z["frame_rate"]))
    assert np.array_equal(f, z["f"]), "populations differ from the reference"
    assert np.array_equal(mv, z["mv"]), "macro variables differ from the reference"


def _random_case(rng, dims, nsubs, acc, comp, bc):
    if dims == 3:
        p = po.Params(dims=3, LX=7, LY=6, LZ=5, nsubs=nsubs, accurate=acc,
                      compressible=comp, tau=(0.8, 0.7),
                      gaccel=(1e-4, -2e-5, 3e-5, 0, 0, 0), sink=1e-3)
    else:
        p = po.Params(dims=2, LX=9, LY=8, LZ=1, nsubs=nsubs, accurate=acc,
                      compressible=comp, tau=(0.9, 0.75),
                      gaccel=(1e-4, 2e-5, 0, 0, 0, 0), sink=1e-3)
    if bc:
        p.pressure_s_in = (1, 0)
        p.pressure_n_out = (1, 0)
        p.rho_in, p.rho_out = 1.01, 1.0
        p.zeroconcgrad_n = p.zeroconcgrad_s = 1
        p.bc_ramp_start, p.bc_ramp_stop = 2, 7
    sol = rng.choice([0, 1, 255], size=p.NN, p=[0.7, 0.2, 0.1]).astype(np.uint8)
    f = rng.standard_normal((p.nsubs, p.Q, p.NN)) * 1e-3
    if not acc:   # plain populations carry the full density
        w = ([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4) if dims == 2 else \
            ([1 / 3] + [1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] * 2 + [1 / 36] * 8)
        f[0] += np.array(w)[:, None]
    if nsubs == 2:
        f[1] = np.abs(f[1])
    return p, sol, f


LIVE = [(3, 1, 1, 0, False), (3, 2, 1, 0, False), (3, 1, 0, 1, False),
        (2, 1, 1, 0, True), (2, 2, 1, 0, True), (2, 1, 0, 1, True)]


@pytest.mark.parametrize("case", LIVE)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_matches_reference_live(case, dtype):
    """Fresh random cases against the reference harness, where it was built."""
    dims, nsubs, acc, comp, bc = case
    p, sol, f = _random_case(np.random.default_rng(hash(case) & 0xffff), dims, nsubs,
                             acc, comp, bc)
    variant = po.variant_name(p, dtype)
    if not po.reference_available(variant):
        pytest.skip("oracle/_ref/%s not built (needs the reference tree)" % variant)
    f = f.astype(dtype)
    f2 = f.copy()
    f, mv = po.run_oracle(p, f, sol, 0, 10, frame_rate=3)
    f2, mv2 = po.run_reference(variant, p, f2, sol, 0, 10, frame_rate=3)
    assert np.isfinite(f).all()
    assert np.array_equal(f, f2)
    assert np.array_equal(mv, mv2)


def test_oracle_conserves_mass_periodic():
    rng = np.random.default_rng(5)
    p = po.Params(dims=3, LX=12, LY=10, LZ=8, tau=(0.7, 1.0), gaccel=(1e-5, 0, 0, 0, 0, 0))
    sol = (rng.random(p.NN) < 0.3).astype(np.uint8)
    f = rng.standard_normal((1, 19, p.NN)) * 1e-3
    m0 = f[0][:, sol != 1].sum()
    f, mv = po.run_oracle(p, f, sol, 0, 40, frame_rate=40)
    assert abs(f[0][:, sol != 1].sum() - m0) < 1e-12


def test_oracle_continues_from_an_odd_time():
    """A run stopped after an odd step continues from the swapped state:
    5 + 3 steps equal 8 steps bit for bit; a negative start is rejected."""
    p = po.Params(dims=3, LX=6, LY=5, LZ=4, gaccel=(1e-4, 0, 0, 0, 0, 0))
    rng = np.random.default_rng(2)
    f0 = rng.standard_normal((1, 19, p.NN)) * 1e-3
    sol = (rng.random(p.NN) < 0.2).astype(np.uint8)
    fa, mva = po.run_oracle(p, f0.copy(), sol, 0, 8, 1)
    fb, mvb = po.run_oracle(p, f0.copy(), sol, 0, 5, 1)
    fb, mvb = po.run_oracle(p, fb, sol, 5, 3, 1, mv=mvb)
    assert np.array_equal(fa, fb) and np.array_equal(mva, mvb)
    with pytest.raises(ValueError):
        po.run_oracle(p, f0.copy(), sol, -1, 2)


@pytest.mark.parametrize("variant,dims", [("d2q9p_f64", 2), ("d3q19p_f64", 3)])
def test_reference_host_loops_run_and_conserve_mass(variant, dims):
    """The reference's own host time loop (stream_collide_stream.c +
    collide.c), the CPU cost baseline of bench.py --cpu-table: on a closed
    periodic lattice with solids and a body force it keeps every value
    finite and the total mass.  It updates solid nodes as well (unlike the
    device kernels), so mass moves between fluid and solid nodes and only
    the sum over all nodes is kept."""
    if not po.reference_available(variant):
        pytest.skip("oracle/_ref not built")
    from lbx import geometry
    if dims == 2:
        p = po.Params(dims=2, LX=24, LY=20, LZ=1, accurate=0, compressible=1, tau=(0.9, 1.0),
                      gaccel=(1e-5, 0, 0, 0, 0, 0))
        sol = geometry.transpose_2d(geometry.disc_pack(20, 24, radius=3, porosity=0.6, seed=3),
                                    20, 24)
    else:
        p = po.Params(dims=3, LX=12, LY=10, LZ=8, accurate=0, compressible=1, tau=(0.9, 1.0),
                      gaccel=(1e-5, 0, 0, 0, 0, 0))
        sol = geometry.sphere_pack(12, 10, 8, radius=2, porosity=0.6, seed=3)
    n = p.NN
    f = po.init_feq(p, np.ones((1, n)), np.zeros((1, n)), np.zeros((1, n)), np.zeros((1, n)))
    m0 = f.sum()
    po.reference_cpu_loops(variant, p, f, sol, 0, 20)
    assert np.isfinite(f).all()
    assert abs(f.sum() - m0) <= 1e-12 * m0
