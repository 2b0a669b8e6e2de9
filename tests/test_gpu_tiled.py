"""The tiled (temporal blocking) path of small 2D lattices (GPU).

lbx_run advances stretches of unchanging AA pairs of a 2D one-substance
lattice in rounds of K steps on tiles held in shared memory.  FP64 results
must be bit-identical to the per-step path and match the oracle (1e-12);
FP32 within the FP32 bound (1e-5).
"""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from _golden import rel_err

pytestmark = pytest.mark.gpu

LAYOUTS = {"dense": lbx.LBX_LAYOUT_DENSE, "compact": lbx.LBX_LAYOUT_COMPACT}
MODELS = {"shifted_inc": (1, 0), "plain_comp": (0, 1), "shifted_comp": (1, 1)}


def _case(LX, LY, faces=True, model="shifted_inc", seed=5, por=0.6, **kw):
    acc, comp = MODELS[model]
    face_kw = dict(pressure_s_in=(1, 0), pressure_n_out=(1, 0), rho_in=1.001,
                   rho_out=1.0) if faces else dict(gaccel=(1e-5, 2e-6, 0, 0, 0, 0))
    face_kw.update(kw)
    p = po.Params(dims=2, LX=LX, LY=LY, LZ=1, tau=(0.9, 1.0), accurate=acc,
                  compressible=comp, **face_kw)
    # discs along j with the first and last rows fluid (the faces fuse)
    sol = geometry.transpose_2d(geometry.disc_pack(LY, LX, radius=3, porosity=por, seed=seed),
                                LY, LX)
    rng = np.random.default_rng(seed)
    f0 = rng.standard_normal((1, 9, p.NN)) * 1e-4
    if not acc:
        # plain populations carry the density: f = w rho (1 + noise)
        w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
        f0 = w[None, :, None] * (1.0 + f0)
    return p, sol, f0


def _lbx(p, dtype, layout, kahan=0):
    kw = {k: getattr(p, k) for k in (
        "dims", "LX", "LY", "LZ", "nsubs", "accurate", "compressible", "tau", "gaccel",
        "pressure_n_in", "pressure_s_in", "pressure_n_out", "pressure_s_out", "rho_in",
        "rho_out", "bc_ramp_start", "bc_ramp_stop")}
    return lbx.Params(precision=np.dtype(dtype).itemsize, layout=LAYOUTS[layout],
                      kahan=kahan, **kw)


def _run(p, sol, f0, steps, frame_rate, dtype, layout, mode, kahan=0):
    with lbx.Domain(_lbx(p, dtype, layout, kahan), sol) as d:
        d.set_run_mode(mode)
        d.upload_f(f0.astype(dtype))
        before = d.launch_count()
        d.run(0, steps, frame_rate)
        d.sync()
        return d.download_f(), d.download_mv(), d.info(), d.launch_count() - before


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("model", sorted(MODELS))
@pytest.mark.parametrize("faces", [True, False])
def test_tiled_fp64_bit_identical_to_steps(layout, model, faces):
    """A ragged lattice (tiles overhang both edges), 2 x 45 steps with a frame
    between: the tiled run equals the per-step run bit for bit."""
    p, sol, f0 = _case(100, 70, faces=faces, model=model)
    ft, mvt, info, nt = _run(p, sol, f0, 90, 45, np.float64, layout, "tiled")
    fs, mvs, _, ns = _run(p, sol, f0, 90, 45, np.float64, layout, "steps")
    assert info["faces_fused"] == faces
    assert np.isfinite(ft).all() and np.isfinite(mvt).all()
    assert np.array_equal(ft, fs)
    assert np.array_equal(mvt, mvs)
    assert nt < ns                      # whole rounds ran as single launches


@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_tiled_fp64_matches_oracle(layout):
    p, sol, f0 = _case(64, 96, model="shifted_inc", seed=7)
    f, mv, _, _ = _run(p, sol, f0, 120, 60, np.float64, layout, "tiled")
    fo, mvo = po.run_oracle(p, f0.copy(), sol, 0, 120, 60)
    assert rel_err(f, fo) <= 1e-12
    fl = sol != 1
    for c in range(3):
        assert rel_err(mv[0, c], mvo[0, c], fl) <= 1e-12, c


@pytest.mark.parametrize("kahan", [0, 1])
@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_tiled_fp32_matches_oracle(layout, kahan):
    """FP32 between pressure faces: the tiled run agrees with the per-step
    path to FP32 rounding, and is as close to the FP64 oracle as the
    oracle's own FP32 run is (whose shifted face balance cancels at
    magnitude 1; the kernels form rho_bc - rho_A in double), or within
    1e-5 of it."""
    p, sol, f0 = _case(96, 48, model="shifted_inc", seed=11)
    p.kahan = kahan
    ft, mvt, _, _ = _run(p, sol, f0, 120, 120, np.float32, layout, "tiled", kahan=kahan)
    fs, mvs, _, _ = _run(p, sol, f0, 120, 120, np.float32, layout, "steps", kahan=kahan)
    f64, mv64 = po.run_oracle(p, f0.copy(), sol, 0, 120, 120)
    f32, mv32 = po.run_oracle(p, f0.astype(np.float32), sol, 0, 120, 120)
    fl = sol != 1
    assert rel_err(ft, fs) <= 1e-5
    assert rel_err(ft, f64) <= max(1e-5, 1.25 * rel_err(f32, f64))
    for c in range(3):
        assert rel_err(mvt[0, c], mvs[0, c], fl) <= 1e-5, c
        assert rel_err(mvt[0, c], mv64[0, c], fl) <= max(
            1e-5, 1.25 * rel_err(mv32[0, c], mv64[0, c], fl)), c


@pytest.mark.parametrize("shape", [(5, 3), (31, 17), (33, 15)])
def test_tiled_lattices_smaller_than_a_tile(shape):
    """Halos wider than the lattice wrap more than once; every copy of a node
    in a tile holds the same values, so the result is still exact."""
    LX, LY = shape
    p, sol, f0 = _case(LX, LY, faces=False, seed=3, por=0.8)
    ft, mvt, _, _ = _run(p, sol, f0, 48, 48, np.float64, "dense", "tiled")
    fs, mvs, _, _ = _run(p, sol, f0, 48, 48, np.float64, "dense", "steps")
    assert np.array_equal(ft, fs) and np.array_equal(mvt, mvs)


def test_tiled_skips_the_steps_whose_arguments_change():
    """A density ramp changes the face densities every step until it ends:
    those steps run one by one, the stretch after the ramp in rounds."""
    p, sol, f0 = _case(64, 48, seed=13, bc_ramp_start=5, bc_ramp_stop=30)
    ft, mvt, _, _ = _run(p, sol, f0, 100, 100, np.float64, "compact", "tiled")
    fs, mvs, _, _ = _run(p, sol, f0, 100, 100, np.float64, "compact", "steps")
    assert np.array_equal(ft, fs) and np.array_equal(mvt, mvs)
    fo, _ = po.run_oracle(p, f0.copy(), sol, 0, 100, 100)
    assert rel_err(ft, fo) <= 1e-12


def test_run_mode_is_checked():
    p, sol, _ = _case(16, 16)
    with lbx.Domain(_lbx(p, np.float64, "dense"), sol) as d:
        with pytest.raises(ValueError):
            d.set_run_mode("fast")
        assert lbx.load_library().lbx_set_run_mode(d._h, 7) == lbx.LBX_ERR_INVALID
        d.set_run_mode("auto")


@pytest.mark.parametrize("shape", [(128, 128), (416, 208)])
def test_tiled_plans_bit_identical_to_steps(shape):
    """128^2: tiles of equal work, one block each, waiting only for the
    tiles their halos read; 416 x 208: more 32 x 16 tiles (169) than the
    GPU has SMs, so blocks take several and meet at grid barriers."""
    LX, LY = shape
    p, sol, f0 = _case(LX, LY, seed=17)
    ft, mvt, _, nt = _run(p, sol, f0, 38, 38, np.float64, "compact", "tiled")
    fs, mvs, _, ns = _run(p, sol, f0, 38, 38, np.float64, "compact", "steps")
    assert np.isfinite(ft).all()
    assert np.array_equal(ft, fs) and np.array_equal(mvt, mvs)
    assert nt < ns


@pytest.mark.parametrize("shape", [(32, 16), (64, 8), (32, 48)])
def test_tiled_equal_work_edge_shapes(shape):
    """Lattices the tile columns divide: one tile whose halo wraps onto
    itself (it waits for its own counter), rows shorter than a tile's
    height, one column of three tiles."""
    LX, LY = shape
    p, sol, f0 = _case(LX, LY, seed=19)
    ft, mvt, info, nt = _run(p, sol, f0, 52, 52, np.float64, "compact", "tiled")
    fs, mvs, _, ns = _run(p, sol, f0, 52, 52, np.float64, "compact", "steps")
    assert info["faces_fused"]
    assert np.array_equal(ft, fs) and np.array_equal(mvt, mvs)
    assert nt < ns
