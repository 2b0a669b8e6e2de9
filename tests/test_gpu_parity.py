"""Parity of the sm_100a kernels with the reference (GPU).

Every case runs through the C ABI (liblbx.so via the lbx binding) and is
compared with either the committed golden fixtures -- outputs of the
reference's own kernel sources -- or the CPU oracle run live on the same
inputs.  Tolerances (norm-wise relative error, ||gpu - ref|| / ||ref||):
FP64 1e-12, FP32 1e-5.  Node classification is checked bit-exact.
"""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from _golden import golden_names, load, rel_err

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float64): 1e-12, np.dtype(np.float32): 1e-5}


def _pairs(f, mv, sol):
    """(name, array, mask) for populations and each macro variable plane."""
    fluid = sol.reshape(-1) != 1
    yield "f", f, None
    for s in range(mv.shape[0]):
        for c in range(mv.shape[1]):
            yield "mv[%d][%d]" % (s, c), mv[s, c], fluid


LAYOUTS = {"dense": lbx.LBX_LAYOUT_DENSE, "compact": lbx.LBX_LAYOUT_COMPACT}


def to_lbx(p: po.Params, dtype, layout="auto") -> lbx.Params:
    kw = {k: getattr(p, k) for k in (
        "dims", "LX", "LY", "LZ", "nsubs", "accurate", "compressible", "tau", "rho_A",
        "gaccel", "sink", "sigma_t_on", "sigma_t_off", "pressure_n_in", "pressure_s_in",
        "pressure_n_out", "pressure_s_out", "zeroconcgrad_n", "zeroconcgrad_s", "rho_in",
        "rho_out", "pfadd", "pfmul", "bc_ramp_start", "bc_ramp_stop", "pressure_n_table",
        "pressure_s_table", "pressure_t_in", "pressure_b_in", "pressure_t_out",
        "pressure_b_out", "constcon_t_in", "constcon_b_in", "zeroconcgrad_t",
        "zeroconcgrad_b", "rho_sigma_in", "kahan", "velocity_t_in", "velocity_t_out",
        "velocity_b_in", "velocity_b_out", "uz_in", "uz_out")}
    return lbx.Params(precision=np.dtype(dtype).itemsize,
                      layout=LAYOUTS.get(layout, lbx.LBX_LAYOUT_AUTO), **kw)


def run_gpu(p: po.Params, f0, sol, steps, frame_rate, dtype, layout="auto"):
    with lbx.Domain(to_lbx(p, dtype, layout), sol) as d:
        d.upload_f(f0)
        d.run(0, steps, frame_rate)
        d.sync()
        return d.download_f(), d.download_mv(), d.info()


def fusable(p: po.Params, sol) -> bool:
    m = sol.reshape(p.LY, p.LX) == 1
    north = any(p.pressure_n_in[:p.nsubs]) or any(p.pressure_n_out[:p.nsubs]) or \
        (p.nsubs == 2 and p.zeroconcgrad_n)
    south = any(p.pressure_s_in[:p.nsubs]) or any(p.pressure_s_out[:p.nsubs]) or \
        (p.nsubs == 2 and p.zeroconcgrad_s)
    for i in range(p.LX):
        up = [(i - 1) % p.LX, i, (i + 1) % p.LX]
        if north and not m[-1, i] and m[0, up].any():
            return False
        if south and not m[0, i] and m[-1, up].any():
            return False
    return True


def assert_close(f, mv, f_ref, mv_ref, sol, dtype, truth=None):
    """FP64: within 1e-12 of the reference.  FP32: within 1e-5 of the
    reference's FP32 result, or -- where that result itself is more than
    1e-5 from the FP64 result `truth` (the shifted pressure faces cancel at
    magnitude 1 in FP32, and unshifted populations lose ~1e-4 in u) -- as
    close to the FP64 result as the reference's FP32 result is, up to the
    spread of FP32 rounding (25%)."""
    tol = TOL[np.dtype(dtype)]
    fluid = sol.reshape(-1) != 1
    ours = dict((k, (a, m)) for k, a, m in _pairs(f, mv, sol))
    tp = dict((k, a) for k, a, _ in _pairs(*truth, sol)) if truth is not None else None
    for k, a_ref, m in _pairs(f_ref, mv_ref, sol):
        a, _ = ours[k]
        e = rel_err(a, a_ref, m)
        if e <= tol:
            continue
        assert tp is not None, "%s: %g" % (k, e)
        e_ref = rel_err(a_ref, tp[k], m)
        e_ours = rel_err(a, tp[k], m)
        assert e_ref > tol and e_ours <= 1.25 * e_ref, \
            "%s: %g from the reference; vs FP64 ours %g, reference %g" % (k, e, e_ours, e_ref)
    # solid nodes are never written
    assert np.array_equal(mv[..., ~fluid], mv_ref[..., ~fluid])


def fp64_truth(p, f0, sol, steps, fr):
    """The same run in FP64 (the oracle), for judging FP32 results."""
    f = f0.astype(np.float64)
    f, mv = po.run_oracle(p, f, sol, 0, steps, fr)
    return f, mv


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("name", golden_names(walsh=False))
def test_gpu_matches_reference_golden(name, layout):
    p, z = load(name)
    dtype = z["f0"].dtype
    steps, fr = int(z["steps"]), int(z["frame_rate"])
    f, mv, info = run_gpu(p, z["f0"], z["solids"], steps, fr, dtype, layout)
    assert info["layout"] == layout
    truth = fp64_truth(p, z["f0"], z["solids"], steps, fr) if dtype == np.float32 else None
    assert_close(f, mv, z["f"], z["mv"], z["solids"], dtype, truth)
    if p.dims == 2 and ("bc" in name or "table" in name):
        assert info["faces_fused"] == fusable(p, z["solids"])
    assert info["fluid_nodes"] == int(np.count_nonzero(z["solids"] != 1))


def _oracle(p, f0, sol, steps, fr):
    f = f0.copy()
    return po.run_oracle(p, f, sol, 0, steps, fr)


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("model", [(1, 0), (0, 1), (1, 1)])
def test_gpu_matches_oracle_d3q19_sphere_pack(dtype, model, layout):
    acc, comp = model
    p = po.Params(dims=3, LX=40, LY=36, LZ=32, accurate=acc, compressible=comp,
                  tau=(0.8, 1.0), gaccel=(1e-5, 2e-6, -1e-6, 0, 0, 0))
    sol = geometry.sphere_pack(40, 36, 32, radius=4, porosity=0.45, seed=11)
    rng = np.random.default_rng(2)
    f0 = rng.standard_normal((1, 19, p.NN)) * 1e-4
    if not acc:
        f0[0] += np.array([1 / 3] + [1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] * 2 + [1 / 36] * 8)[:, None]
    f0 = f0.astype(dtype)
    f, mv, _ = run_gpu(p, f0, sol, 30, 15, dtype, layout)
    fo, mvo = _oracle(p, f0, sol, 30, 15)
    assert_close(f, mv, fo, mvo, sol, dtype,
                 fp64_truth(p, f0, sol, 30, 15) if dtype == np.float32 else None)


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gpu_matches_oracle_d3q19_solute(dtype, layout):
    p = po.Params(dims=3, LX=33, LY=20, LZ=24, nsubs=2, tau=(0.9, 0.7), sink=1e-3,
                  gaccel=(2e-5, 0, 0, 0, 0, 0), sigma_t_on=5, sigma_t_off=1000)
    sol = geometry.sphere_pack(33, 20, 24, radius=3, porosity=0.5, seed=4)
    rng = np.random.default_rng(3)
    f0 = rng.standard_normal((2, 19, p.NN)) * 1e-4
    f0[1] = np.abs(f0[1]) * 10
    f0 = f0.astype(dtype)
    f, mv, _ = run_gpu(p, f0, sol, 24, 12, dtype, layout)
    fo, mvo = _oracle(p, f0, sol, 24, 12)
    assert_close(f, mv, fo, mvo, sol, dtype,
                 fp64_truth(p, f0, sol, 24, 12) if dtype == np.float32 else None)


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("fused", [True, False])
def test_gpu_matches_oracle_d2q9_pressure_faces(dtype, fused, layout):
    """The configuration of the 2D benchmark (flow between pressure faces) on
    a smaller lattice; `fused=False` plants solids across the periodic wrap
    so the stand-alone face kernels run."""
    LX, LY = 48, 64
    p = po.Params(dims=2, LX=LX, LY=LY, LZ=1, tau=(1.0, 1.0), pressure_s_in=(1, 0),
                  pressure_n_out=(1, 0), rho_in=1.001, rho_out=1.0)
    sol = geometry.transpose_2d(geometry.disc_pack(LY, LX, radius=4, porosity=0.6, seed=9),
                                LY, LX)
    if not fused:
        g = sol.reshape(LY, LX)
        g[0, 5] = 1
        g[-1, 20] = 1
    f0 = np.zeros((1, 9, p.NN), dtype=dtype)
    f, mv, info = run_gpu(p, f0, sol, 60, 20, dtype, layout)
    assert info["faces_fused"] == fused
    fo, mvo = _oracle(p, f0, sol, 60, 20)
    assert_close(f, mv, fo, mvo, sol, dtype,
                 fp64_truth(p, f0, sol, 60, 20) if dtype == np.float32 else None)


@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_gpu_d2q9_solute_faces_fp64(layout):
    p = po.Params(dims=2, LX=40, LY=30, LZ=1, nsubs=2, tau=(0.9, 0.8), sink=1e-3,
                  pressure_s_in=(1, 0), pressure_n_out=(1, 0), rho_in=1.002, rho_out=1.0,
                  zeroconcgrad_n=1, zeroconcgrad_s=1, bc_ramp_start=3, bc_ramp_stop=20)
    rng = np.random.default_rng(8)
    sol = (rng.random(p.NN) < 0.15).astype(np.uint8)
    f0 = rng.standard_normal((2, 9, p.NN)) * 1e-4
    f0[1] = np.abs(f0[1]) + 0.1
    f, mv, _ = run_gpu(p, f0, sol, 40, 10, np.float64, layout)
    fo, mvo = _oracle(p, f0, sol, 40, 10)
    assert_close(f, mv, fo, mvo, sol, np.float64)


@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_gpu_full_size_step_pair_matches_oracle(layout):
    """256^3 D3Q19 FP32 sphere pack (the benchmark lattice): one AA pair."""
    n = 256
    p = po.Params(dims=3, LX=n, LY=n, LZ=n, tau=(0.8, 1.0), gaccel=(1e-6, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(n, n, n, radius=6, porosity=0.4, seed=1234)
    rng = np.random.default_rng(0)
    f0 = (rng.standard_normal((1, 19, p.NN), dtype=np.float32) * np.float32(1e-4))
    f, mv, info = run_gpu(p, f0, sol, 2, 2, np.float32, layout)
    assert info["fluid_nodes"] == int(np.count_nonzero(sol != 1))
    fo, mvo = _oracle(p, f0, sol, 2, 2)
    assert_close(f, mv, fo, mvo, sol, np.float32, fp64_truth(p, f0, sol, 2, 2))


def test_gpu_mass_conserved_full_size():
    """Bounce-back and periodic streaming conserve mass: 200 steps at 256^3."""
    n = 256
    lp = lbx.Params(dims=3, LX=n, LY=n, LZ=n, precision=4, tau=(0.8, 1.0),
                    gaccel=(1e-6, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(n, n, n, radius=6, porosity=0.4, seed=1234)
    with lbx.Domain(lp, sol) as d:
        d.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        d.run(0, 199, 0)
        d.step(200, write_mv=True)
        r = d.reduce()
        assert r["status"] == lbx.LBX_OK and r["nonfinite"] == 0
        nf = int(np.count_nonzero(sol != 1))
        assert r["fluid_nodes"] == nf
        assert abs(r["mass"] - nf) / nf < 1e-6
        # flow develops along +x
        assert r["u_sum"][0] > 0 and abs(r["u_sum"][1]) < 0.05 * r["u_sum"][0]


def test_gpu_reduce_matches_numpy():
    p = lbx.Params(dims=3, LX=30, LY=20, LZ=10, precision=8, nsubs=2)
    rng = np.random.default_rng(1)
    sol = (rng.random(p.NN) < 0.3).astype(np.uint8)
    mv = rng.random((2, 4, p.NN)) + 0.5
    with lbx.Domain(p, sol) as d:
        d.upload_mv(mv)
        r = d.reduce()
    fl = sol != 1
    assert r["fluid_nodes"] == fl.sum()
    assert np.isclose(r["mass"], mv[0, 0, fl].sum(), rtol=1e-13)
    assert np.isclose(r["solute_mass"], mv[1, 0, fl].sum(), rtol=1e-13)
    for c in range(3):
        assert np.isclose(r["momentum"][c], (mv[0, 0, fl] * mv[0, 1 + c, fl]).sum(), rtol=1e-12)
    assert r["rho_min"] == mv[0, 0, fl].min() and r["rho_max"] == mv[0, 0, fl].max()


def test_gpu_reduce_flags_nonfinite():
    p = lbx.Params(dims=2, LX=8, LY=8, LZ=1, precision=4)
    mv = np.ones((1, 3, 64), np.float32)
    mv[0, 1, 10] = np.nan
    with lbx.Domain(p, np.zeros(64, np.uint8)) as d:
        d.upload_mv(mv)
        r = d.reduce()
    assert r["status"] == lbx.LBX_ERR_NUMERIC and r["nonfinite"] == 1


def test_gpu_init_equilibrium_matches_oracle():
    p = po.Params(dims=3, LX=16, LY=12, LZ=10, nsubs=2)
    rng = np.random.default_rng(6)
    rho = 1 + 0.01 * rng.random((2, p.NN))
    u = 0.01 * rng.standard_normal((3, 2, p.NN))
    fo = po.init_feq(p, rho, u[0], u[1], u[2])
    with lbx.Domain(to_lbx(p, np.float64), np.zeros(p.NN, np.uint8)) as d:
        for s in range(2):
            d.init_equilibrium(s, rho[s], u[0, s], u[1, s], u[2, s])
        f = d.download_f()
        mv = d.download_mv()
    assert rel_err(f, fo) < 1e-14
    # the macro variables hold the fields, as init_problem leaves them
    for s in range(2):
        assert np.array_equal(mv[s, 0], rho[s])
        for c in range(3):
            assert np.array_equal(mv[s, 1 + c], u[c, s])


@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_gpu_init_equilibrium_2d_then_steps(layout):
    """2D FP32 over solids: the state formed from rho, u equals the oracle's
    feq, the macro variables hold the fields, and steps from it match the
    oracle run from the same populations."""
    p = po.Params(dims=2, LX=40, LY=28, LZ=1, tau=(0.9, 1), gaccel=(1e-5, 0, 0, 0, 0, 0))
    sol = geometry.transpose_2d(geometry.disc_pack(28, 40, radius=3, porosity=0.6, seed=4),
                                28, 40)
    rng = np.random.default_rng(8)
    rho = (1 + 0.01 * rng.random(p.NN)).astype(np.float32)
    u = (0.01 * rng.standard_normal((2, p.NN))).astype(np.float32)
    fo = po.init_feq(p, rho[None], u[0][None], u[1][None], None)
    with lbx.Domain(to_lbx(p, np.float32, layout), sol) as d:
        d.init_equilibrium(0, rho, u[0], u[1])
        f0 = d.download_f()
        mv = d.download_mv()
        d.run(0, 20, 20)
        f = d.download_f()
    assert rel_err(f0, fo) < 1e-6
    assert np.array_equal(mv[0, 0], rho) and np.array_equal(mv[0, 1], u[0])
    assert np.array_equal(mv[0, 2], u[1])
    fr, _ = _oracle(p, f0.astype(np.float32), sol, 20, 20)
    fr64, _ = _oracle(p, f0.astype(np.float64), sol, 20, 20)
    assert rel_err(f, fr64) <= max(1e-5, 1.25 * rel_err(fr, fr64))


def test_gpu_rejects_out_of_order_steps():
    p = lbx.Params(dims=3, LX=8, LY=8, LZ=8, precision=4)
    with lbx.Domain(p, np.zeros(512, np.uint8)) as d:
        with pytest.raises(lbx.LbxError) as ei:
            d.step(2)
        assert ei.value.code == lbx.LBX_ERR_STATE
        d.step(1)
        with pytest.raises(lbx.LbxError):
            d.step(3)
        d.step(2)


def test_gpu_caller_stream():
    torch = pytest.importorskip("torch")
    p = po.Params(dims=3, LX=20, LY=18, LZ=16, tau=(0.9, 1), gaccel=(1e-5, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(20, 18, 16, radius=3, porosity=0.5, seed=2)
    f0 = (np.random.default_rng(1).standard_normal((1, 19, p.NN)) * 1e-4)
    s = torch.cuda.Stream()
    with lbx.Domain(to_lbx(p, np.float64), sol) as d:
        d.upload_f(f0)
        d.set_stream(s.cuda_stream)
        d.run(0, 10, 10)
        s.synchronize()
        d.set_stream(None)
        f = d.download_f()
        assert d.launch_count() >= 10
    fo, _ = _oracle(p, f0, sol, 10, 10)
    assert rel_err(f, fo) < 1e-12


@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_gpu_cfg1_full_run_matches_oracle(layout):
    """The 2D benchmark case in full: 256^2 D2Q9 FP64 between Zou-He pressure
    faces, 2000 steps from rest, against the oracle (1e-12)."""
    from lbx import configs
    lp, mask = configs.cfg1_params(8, LAYOUTS[layout])
    with lbx.Domain(lp, mask) as d:
        d.init_equilibrium(0, 1.0, 0.0, 0.0)
        d.run(0, 1999, 0)
        d.step(2000, write_mv=True)
        f, mv, info = d.download_f(), d.download_mv(), d.info()
    assert info["faces_fused"] and info["layout"] == layout
    p = po.Params(dims=2, LX=256, LY=256, LZ=1, tau=(1.0, 1.0), pressure_s_in=(1, 0),
                  pressure_n_out=(1, 0), rho_in=1.001, rho_out=1.0)
    # the macro variables init_equilibrium leaves (rho = 1, u = 0), which
    # the steps never overwrite at solid nodes
    mv0 = np.zeros((1, 3, p.NN))
    mv0[0, 0] = 1.0
    fo, mvo = po.run_oracle(p, np.zeros((1, 9, p.NN)), mask, 0, 2000, 2000, mv=mv0)
    assert_close(f, mv, fo, mvo, mask, np.float64)
    # pressure-driven flow along j, from the rho_in face to the rho_out face
    fl = mask != 1
    assert mv[0, 2, fl].mean() > 0
    rho = mv[0, 0].reshape(256, 256)
    flg = fl.reshape(256, 256)
    assert rho[1, flg[1]].mean() > rho[-2, flg[-2]].mean()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gpu_compact_thin_wide_lattice(dtype):
    """A lattice only three planes deep with ~111k fluid nodes per plane: the
    periodic wrap in z touches every node and compact indices of z
    neighbours lie ~111k apart."""
    LX, LY, LZ = 512, 256, 3
    p = po.Params(dims=3, LX=LX, LY=LY, LZ=LZ, tau=(0.7, 1.0),
                  gaccel=(2e-6, 1e-6, 0, 0, 0, 0))
    rng = np.random.default_rng(12)
    sol = (rng.random(p.NN) < 0.15).astype(np.uint8)
    f0 = (rng.standard_normal((1, 19, p.NN)) * 1e-4).astype(dtype)
    f, mv, info = run_gpu(p, f0, sol, 12, 6, dtype, "compact")
    fo, mvo = _oracle(p, f0, sol, 12, 6)
    assert_close(f, mv, fo, mvo, sol, dtype,
                 fp64_truth(p, f0, sol, 12, 6) if dtype == np.float32 else None)


@pytest.mark.parametrize("nsubs", [1, 2])
@pytest.mark.parametrize("dims,shape", [(3, (1, 5, 7)), (3, (2, 9, 5)), (3, (3, 11, 3)),
                                        (2, (1, 37, 1)), (2, (2, 19, 1))])
def test_gpu_compact_narrow_x_extents(dims, shape, nsubs):
    """Lattices one to three nodes wide in x with nodes 0 and N - 1 fluid:
    every node sits on an x edge (the odd step's wrapped x neighbours) and
    the neighbour lookups read the first and last words of the fluid-rank
    table.  FP64, compact layout, against the oracle."""
    LX, LY, LZ = shape
    p = po.Params(dims=dims, LX=LX, LY=LY, LZ=LZ, nsubs=nsubs, tau=(0.9, 0.7),
                  sink=1e-3 if nsubs == 2 else 0.0, sigma_t_on=2, sigma_t_off=1000,
                  gaccel=(2e-5, -1e-5, 3e-6 if dims == 3 else 0.0, 0, 0, 0))
    rng = np.random.default_rng(LX * 100 + LY + nsubs)
    sol = (rng.random(p.NN) < 0.3).astype(np.uint8)
    sol[0] = sol[-1] = 0
    Q = 19 if dims == 3 else 9
    f0 = rng.standard_normal((nsubs, Q, p.NN)) * 1e-4
    if nsubs == 2:
        f0[1] = np.abs(f0[1]) * 10
    f, mv, info = run_gpu(p, f0, sol, 12, 6, np.float64, "compact")
    assert info["layout"] == "compact"
    fo, mvo = _oracle(p, f0, sol, 12, 6)
    assert_close(f, mv, fo, mvo, sol, np.float64)


@pytest.mark.parametrize("nsubs", [1, 2])
def test_gpu_upload_into_a_stepped_domain(nsubs):
    """Uploading populations after steps replaces them: all of one
    substance equals a fresh domain bit for bit; one substance of two keeps
    the other's stepped state (the oracle, stepped and replaced the same
    way).  Compact layout, FP64."""
    p = po.Params(dims=3, LX=18, LY=14, LZ=12, nsubs=nsubs, tau=(0.9, 0.7),
                  sink=1e-3 if nsubs == 2 else 0.0, sigma_t_on=2, sigma_t_off=1000,
                  gaccel=(2e-5, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(18, 14, 12, radius=3, porosity=0.5, seed=5)
    rng = np.random.default_rng(8)
    f0 = rng.standard_normal((nsubs, 19, p.NN)) * 1e-4
    f1 = rng.standard_normal((nsubs, 19, p.NN)) * 1e-4
    if nsubs == 2:
        f0[1] = np.abs(f0[1]) * 10
        f1[1] = np.abs(f1[1]) * 10
    lp = to_lbx(p, np.float64, "compact")
    with lbx.Domain(lp, sol) as d:
        d.upload_f(f0)
        d.run(0, 6, 6)
        if nsubs == 1:
            d.upload_f(f1)
        else:
            d.upload_f(f1[1], subs=1)
        d.run(6, 6, 6)
        d.sync()
        f = d.download_f()
    if nsubs == 1:
        with lbx.Domain(lp, sol) as d:
            d.upload_f(f1)
            d.run(0, 6, 6)
            d.sync()
            np.testing.assert_array_equal(f, d.download_f())
    else:
        fo, _ = po.run_oracle(p, f0.copy(), sol, 0, 6, 6)
        fo[1] = f1[1]
        fo, _ = po.run_oracle(p, fo, sol, 6, 6, 6)
        assert rel_err(f, fo) < 1e-12


@pytest.mark.parametrize("nsubs", [1, 2])
def test_gpu_init_into_a_stepped_domain(nsubs):
    """lbx_init_equilibrium after steps replaces the substance's state: one
    substance equals a fresh domain's init bit for bit (solid nodes and
    macro variables included) and steps on identically; one substance of
    two keeps the other's stepped state (the oracle, stepped and replaced
    the same way).  Compact layout, FP64."""
    p = po.Params(dims=3, LX=18, LY=14, LZ=12, nsubs=nsubs, tau=(0.9, 0.7),
                  sink=1e-3 if nsubs == 2 else 0.0, sigma_t_on=2, sigma_t_off=1000,
                  gaccel=(2e-5, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(18, 14, 12, radius=3, porosity=0.5, seed=6)
    rng = np.random.default_rng(9)
    f0 = rng.standard_normal((nsubs, 19, p.NN)) * 1e-4
    if nsubs == 2:
        f0[1] = np.abs(f0[1]) * 10
    s = nsubs - 1                     # the substance re-initialised
    rho = (0.01 if s else 1.0) + 0.001 * rng.random(p.NN)
    lp = to_lbx(p, np.float64, "compact")

    def init(d):
        d.init_equilibrium(s, rho)    # at rest: u filled on the device
    with lbx.Domain(lp, sol) as d:
        d.upload_f(f0)
        d.run(0, 6, 6)
        init(d)
        fi, mvi = d.download_f(), d.download_mv()
        d.run(0, 6, 6)
        d.sync()
        f = d.download_f()
    if nsubs == 1:
        with lbx.Domain(lp, sol) as d:
            init(d)
            np.testing.assert_array_equal(fi, d.download_f())
            np.testing.assert_array_equal(mvi, d.download_mv())
            d.run(0, 6, 6)
            d.sync()
            np.testing.assert_array_equal(f, d.download_f())
    else:
        fo, _ = po.run_oracle(p, f0.copy(), sol, 0, 6, 6)
        z = np.zeros((2, p.NN))
        fo[1] = po.init_feq(p, np.stack([rho, rho]), z, z, z)[1]
        assert rel_err(fi, fo) < 1e-14
        assert np.array_equal(mvi[1, 0], rho) and not mvi[1, 1:].any()
        fo, _ = po.run_oracle(p, fo, sol, 0, 6, 6)
        assert rel_err(f, fo) < 1e-12
