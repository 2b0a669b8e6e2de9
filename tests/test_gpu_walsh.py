"""Walsh partial bounce-back (WALSH_NS_ON with COMPUTE_ON_SOLIDS) on the GPU.

The dense step kernel's Walsh path is compared with the reference's own
kernel sources built with both flags (golden fixtures), with the CPU oracle
on larger lattices, and through properties that hold at any size: ns = 0
everywhere is the plain periodic update (bit-exact in FP64), and the blend
conserves mass.  Every node is updated in Walsh runs, so every node is
compared.  Tolerances (norm-wise relative): FP64 1e-12, FP32 1e-5.
"""
import dataclasses

import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from _golden import golden_names, load, rel_err

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float64): 1e-12, np.dtype(np.float32): 1e-5}
W19 = np.array([1 / 3] + [1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] * 2 + [1 / 36] * 8)


def to_lbx(p: po.Params, dtype) -> lbx.Params:
    kw = {k: getattr(p, k) for k in (
        "dims", "LX", "LY", "LZ", "nsubs", "accurate", "compressible", "tau", "rho_A",
        "gaccel", "sink", "sigma_t_on", "sigma_t_off", "kahan")}
    return lbx.Params(precision=np.dtype(dtype).itemsize, walsh=1, **kw)


def run_gpu(p, f0, sol, ns, steps, fr, dtype):
    with lbx.Domain(to_lbx(p, dtype), sol) as d:
        d.set_ns(ns)
        d.upload_f(f0)
        d.run(0, steps, fr)
        d.sync()
        return d.download_f(), d.download_mv(), d.info()


def run_oracle(p, f0, sol, ns, steps, fr):
    q = dataclasses.replace(p, walsh=1, ns=np.asarray(ns, dtype=np.float64))
    return po.run_oracle(q, f0.copy(), sol, 0, steps, fr)


def _pairs(f, mv):
    yield "f", f
    for s in range(mv.shape[0]):
        for c in range(mv.shape[1]):
            yield "mv[%d][%d]" % (s, c), mv[s, c]


def assert_close(f, mv, f_ref, mv_ref, dtype, truth=None):
    """Within the tolerance of the reference (or the oracle).  FP32 where
    that result is itself more than 1e-5 from the FP64 run `truth` (plain
    compressible populations cancel in the momentum sums): as close to the
    FP64 run as the FP32 reference is, up to 25% for FP32 rounding."""
    tol = TOL[np.dtype(dtype)]
    tp = dict(_pairs(*truth)) if truth is not None else None
    ours = dict(_pairs(f, mv))
    for k, a_ref in _pairs(f_ref, mv_ref):
        e = rel_err(ours[k], a_ref)
        if e <= tol:
            continue
        assert tp is not None, "%s: %g" % (k, e)
        e_ref, e_ours = rel_err(a_ref, tp[k]), rel_err(ours[k], tp[k])
        assert e_ref > tol and e_ours <= 1.25 * e_ref, \
            "%s: %g from the reference; vs FP64 ours %g, reference %g" % (k, e, e_ours, e_ref)


def draw_ns(rng, n, sol=None):
    """Fractions in [0, 1] with exact 0 and 1 among them; where a mask is
    given, its solid nodes get 0.8 (the reference's 2D rule: ns where the
    mask is solid, 0 elsewhere, with a mixed field on top)."""
    ns = rng.uniform(0.0, 1.0, n)
    pick = rng.choice([0, 1, 2], size=n, p=[0.5, 0.3, 0.2])
    ns = np.where(pick == 1, 0.0, np.where(pick == 2, 1.0, ns))
    if sol is not None:
        ns = np.where(sol == 1, 0.8, ns)
    return ns


@pytest.mark.parametrize("name", golden_names(walsh=True))
def test_gpu_walsh_matches_reference_golden(name):
    p, z = load(name)
    dtype = z["f0"].dtype
    steps, fr = int(z["steps"]), int(z["frame_rate"])
    f, mv, info = run_gpu(p, z["f0"], z["solids"], p.ns, steps, fr, dtype)
    assert info["layout"] == "dense"
    assert_close(f, mv, z["f"], z["mv"], dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("model", [(1, 0), (0, 1), (1, 1)])
def test_gpu_walsh_matches_oracle_d3q19(dtype, model):
    acc, comp = model
    p = po.Params(dims=3, LX=40, LY=36, LZ=32, accurate=acc, compressible=comp,
                  tau=(0.8, 1.0), gaccel=(1e-5, 2e-6, -1e-6, 0, 0, 0))
    sol = geometry.sphere_pack(40, 36, 32, radius=4, porosity=0.45, seed=11)
    rng = np.random.default_rng(31)
    ns = draw_ns(rng, p.NN, sol)
    f0 = rng.standard_normal((1, 19, p.NN)) * 1e-4
    if not acc:
        f0[0] += W19[:, None]
    f0 = f0.astype(dtype)
    f, mv, _ = run_gpu(p, f0, sol, ns, 30, 15, dtype)
    fo, mvo = run_oracle(p, f0, sol, ns, 30, 15)
    truth = run_oracle(p, f0.astype(np.float64), sol, ns, 30, 15) if dtype == np.float32 else None
    assert_close(f, mv, fo, mvo, dtype, truth)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gpu_walsh_matches_oracle_solute(dtype):
    p = po.Params(dims=3, LX=24, LY=20, LZ=18, nsubs=2, tau=(0.9, 0.7), sink=1e-3,
                  sigma_t_on=2, sigma_t_off=21, gaccel=(3e-5, 0, 1e-5, 0, 0, 0))
    rng = np.random.default_rng(32)
    ns = draw_ns(rng, p.NN)
    f0 = rng.standard_normal((2, 19, p.NN)) * 1e-4
    f0[1] = np.abs(f0[1]) + 0.5 * W19[:, None]
    f0 = f0.astype(dtype)
    sol = np.zeros(p.NN, np.uint8)
    f, mv, _ = run_gpu(p, f0, sol, ns, 24, 8, dtype)
    fo, mvo = run_oracle(p, f0, sol, ns, 24, 8)
    assert_close(f, mv, fo, mvo, dtype)


def test_gpu_walsh_matches_oracle_d2q9():
    p = po.Params(dims=2, LX=64, LY=48, LZ=1, tau=(0.9, 1.0), gaccel=(2e-5, -1e-5, 0, 0, 0, 0))
    rng = np.random.default_rng(33)
    sol = (rng.random(p.NN) < 0.3).astype(np.uint8)
    ns = np.where(sol == 1, 0.7, 0.0)          # the reference's 2D rule alone
    f0 = rng.standard_normal((1, 9, p.NN)) * 1e-4
    f, mv, _ = run_gpu(p, f0, sol, ns, 40, 10, np.float64)
    fo, mvo = run_oracle(p, f0, sol, ns, 40, 10)
    assert_close(f, mv, fo, mvo, np.float64)


def test_gpu_walsh_zero_fraction_is_the_plain_update():
    """ns = 0 on an all-fluid lattice: (1 - ns) = 1 and ns f = 0 exactly,
    so the Walsh kernel reproduces the plain kernel bit for bit in FP64."""
    p = po.Params(dims=3, LX=32, LY=30, LZ=28, tau=(0.8, 1.0), gaccel=(1e-5, 0, 2e-6, 0, 0, 0))
    rng = np.random.default_rng(34)
    f0 = rng.standard_normal((1, 19, p.NN)) * 1e-4
    sol = np.zeros(p.NN, np.uint8)
    f, mv, _ = run_gpu(p, f0, sol, np.zeros(p.NN), 20, 10, np.float64)
    lp = to_lbx(p, np.float64)
    lp.walsh = 0
    with lbx.Domain(lp, sol) as d:
        d.upload_f(f0)
        d.run(0, 20, 10)
        d.sync()
        fp, mvp = d.download_f(), d.download_mv()
    assert np.array_equal(f, fp) and np.array_equal(mv, mvp)


def test_gpu_walsh_full_size_step_pair_and_mass():
    """256^3 D3Q19 FP32 (the benchmark lattice) with a sphere-pack ns field:
    one odd/even pair against the oracle, then mass conservation over 20
    steps (streaming permutes, BGK and the blend conserve each node's sum)."""
    n = 256
    p = po.Params(dims=3, LX=n, LY=n, LZ=n, tau=(0.8, 1.0), gaccel=(1e-6, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(n, n, n, radius=6, porosity=0.4, seed=1234)
    rng = np.random.default_rng(35)
    ns = np.where(sol == 1, 1.0, rng.uniform(0.0, 0.2, p.NN))
    f0 = (rng.standard_normal((1, 19, p.NN)) * 1e-4).astype(np.float32)
    f, mv, _ = run_gpu(p, f0, sol, ns, 2, 2, np.float32)
    fo, mvo = run_oracle(p, f0, sol, ns, 2, 2)
    assert_close(f, mv, fo, mvo, np.float32)
    f0d = f0.astype(np.float64)
    with lbx.Domain(to_lbx(p, np.float64), sol) as d:
        d.set_ns(ns)
        d.upload_f(f0d)
        m0 = float(np.sum(f0d))
        d.run(0, 20, 20)
        d.sync()
        m1 = float(np.sum(d.download_f()))
    assert abs(m1 - m0) <= 1e-12 * float(np.sum(np.abs(f0d))), (m0, m1)


def test_gpu_walsh_set_ns_errors():
    p = lbx.Params(dims=3, LX=8, LY=8, LZ=8, precision=8)
    sol = np.zeros(p.NN, np.uint8)
    with lbx.Domain(p, sol) as d:
        with pytest.raises(lbx.LbxError) as ei:
            d.set_ns(np.zeros(p.NN))
        assert ei.value.code == lbx.LBX_ERR_STATE
    p.walsh = 1
    with lbx.Domain(p, sol) as d:
        for bad in (1.5, -0.1, np.nan):
            ns = np.zeros(p.NN)
            ns[17] = bad
            with pytest.raises(lbx.LbxError) as ei:
                d.set_ns(ns)
            assert ei.value.code == lbx.LBX_ERR_INVALID
        d.set_ns(np.full(p.NN, 0.5))
