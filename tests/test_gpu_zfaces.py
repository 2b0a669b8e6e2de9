"""Top/bottom (z) face boundaries and the breakthrough record (GPU) against
the CPU oracle.  The reference has no device code for these faces; the
oracle states the rules (2D kernels carried to z), so parity here is with
that restatement."""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from test_gpu_parity import assert_close, fp64_truth, to_lbx

pytestmark = pytest.mark.gpu


def _flow_solute(LX, LY, LZ, por, seed, **faces):
    p = po.Params(dims=3, LX=LX, LY=LY, LZ=LZ, nsubs=2, tau=(0.9, 0.7),
                  rho_in=1.001, rho_out=1.0, rho_sigma_in=1.0, **faces)
    sol = geometry.sphere_pack(LX, LY, LZ, radius=3, porosity=por, seed=seed)
    rho = np.stack([np.ones(p.NN), np.zeros(p.NN)])
    z = np.zeros((2, p.NN))
    return p, sol, po.init_feq(p, rho, z, z, z)


CASES = {
    # cfg3's boundary set: flow up from the bottom, C = 1 at the inlet
    "inlet_bottom": dict(pressure_b_in=(1, 0), pressure_t_out=(1, 0), constcon_b_in=1,
                         zeroconcgrad_t=1),
    # the mirrored set: flow down from the top
    "inlet_top": dict(pressure_t_in=(1, 0), pressure_b_out=(1, 0), constcon_t_in=1,
                      zeroconcgrad_b=1),
    # Zou-He velocity inflow at the top, pressure outflow at the bottom
    "velocity_top_in": dict(velocity_t_in=(1, 0), uz_in=-0.01, pressure_b_out=(1, 0),
                            constcon_t_in=1, zeroconcgrad_b=1),
    # velocity on both faces, the solute's too; a pressure face overridden
    # by the velocity face configured after it on the same face
    "velocity_both": dict(velocity_t_in=(1, 1), velocity_b_out=(1, 0), uz_in=-0.006,
                          uz_out=-0.004, pressure_t_in=(1, 0), zeroconcgrad_b=1),
    "velocity_bottom_in": dict(velocity_b_in=(1, 0), velocity_t_out=(1, 0), uz_in=0.008,
                               uz_out=0.007, constcon_b_in=1, zeroconcgrad_t=1),
}


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("case", sorted(CASES))
def test_gpu_z_faces_match_oracle(case, dtype, layout):
    p, sol, f0 = _flow_solute(20, 18, 24, 0.55, 5, **CASES[case])
    f0 = f0.astype(dtype)
    with lbx.Domain(to_lbx(p, dtype, layout), sol) as d:
        d.upload_f(f0)
        d.run(0, 40, 20)
        d.sync()
        f, mv = d.download_f(), d.download_mv()
    fo, mvo = po.run_oracle(p, f0.copy(), sol, 0, 40, 20)
    assert_close(f, mv, fo, mvo, sol, dtype,
                 fp64_truth(p, f0, sol, 40, 20) if dtype == np.float32 else None)


@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_gpu_z_faces_solid_wrap_neighbours(layout):
    """Solid nodes in the plane across the periodic wrap from a face: the
    deposits of those unknowns fall back to the node's own slot."""
    p, sol, f0 = _flow_solute(16, 14, 12, 0.6, 9, **CASES["inlet_bottom"])
    sol = sol.reshape(12, 14, 16)
    sol[-1, ::3, ::2] = 1          # top plane: upstream of the bottom face
    sol[0, 1::4, 1::3] = 1         # and some bottom-face nodes themselves
    sol = sol.reshape(-1)
    with lbx.Domain(to_lbx(p, np.float64, layout), sol) as d:
        d.upload_f(f0)
        d.run(0, 30, 15)
        d.sync()
        f, mv = d.download_f(), d.download_mv()
    fo, mvo = po.run_oracle(p, f0.copy(), sol, 0, 30, 15)
    assert_close(f, mv, fo, mvo, sol, np.float64)


@pytest.mark.parametrize("where", ["top", "bottom", "interior"])
@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gpu_breakthrough_record_matches_oracle(dtype, layout, where):
    """The record of a face plane (written only by the compact layout's
    face-plane launch, and reduced beside the interior launches) and of an
    interior plane (reduced after both)."""
    p, sol, f0 = _flow_solute(20, 18, 16, 0.55, 7, **CASES["inlet_bottom"])
    p.sigma_t_on, p.sigma_t_off = 3, 10 ** 6
    plane = {"top": p.LZ - 1, "bottom": 0, "interior": p.LZ // 2}[where]
    f0 = f0.astype(dtype)
    steps = 60
    with lbx.Domain(to_lbx(p, dtype, layout), sol) as d:
        d.upload_f(f0)
        d.btc_start(plane, 100)
        d.run(0, steps, 0)
        btc, ux = d.btc_read(ux=True)
    _, _, btc_o, ux_o = po.run_oracle_btc(p, f0.copy(), sol, 0, steps, plane)
    assert btc.shape == (steps,)
    assert np.isnan(btc[:2]).all() and np.isnan(btc_o[:2]).all()   # solute off at t=1,2
    live = ~np.isnan(btc_o)
    tol = 1e-12 if dtype == np.float64 else 1e-5
    scale = np.abs(btc_o[live]).max()
    assert scale > 0
    assert np.abs(btc[live] - btc_o[live]).max() <= tol * scale
    uscale = np.abs(ux_o).max()
    assert uscale > 0 and np.abs(ux - ux_o).max() <= tol * uscale


def test_gpu_breakthrough_record_through_graph_replay():
    """Long frame-free runs replay captured step pairs; the record still
    advances one slot per step and equals step-by-step stepping."""
    p, sol, f0 = _flow_solute(16, 16, 12, 0.6, 3, **CASES["inlet_bottom"])
    lp = to_lbx(p, np.float64, "compact")
    out = []
    for replay in (True, False):
        with lbx.Domain(lp, sol) as d:
            d.upload_f(f0)
            d.btc_start(p.LZ - 1, 50)
            if replay:
                d.run(0, 40, 0)
            else:
                for t in range(1, 41):
                    d.step(t)
            out.append(d.btc_read())
    assert out[0].shape == (40,)
    np.testing.assert_array_equal(out[0], out[1])


def test_z_faces_rejected_in_2d_and_thin_lattices():
    bad = [lbx.Params(dims=2, LX=8, LY=8, LZ=1, pressure_t_in=(1, 0)),
           lbx.Params(dims=3, LX=8, LY=8, LZ=2, pressure_b_in=(1, 0)),
           lbx.Params(dims=2, LX=8, LY=8, LZ=1, velocity_t_in=(1, 0), uz_in=-0.01),
           lbx.Params(dims=3, LX=8, LY=8, LZ=8, velocity_b_out=(1, 0), uz_out=1.0)]
    for lp in bad:
        with pytest.raises(lbx.LbxError):
            lbx.Domain(lp, np.zeros(lp.NN, np.uint8))


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gpu_constcon_profile_matches_oracle(dtype, layout):
    """A per-node inlet concentration on the bottom face."""
    p, sol, f0 = _flow_solute(18, 16, 14, 0.6, 11, **CASES["inlet_bottom"])
    prof = np.random.default_rng(5).uniform(0.0, 1.0, p.LX * p.LY)
    p.constcon_profile_b = prof
    f0 = f0.astype(dtype)
    with lbx.Domain(to_lbx(p, dtype, layout), sol) as d:
        d.set_face_profile(False, prof)
        d.upload_f(f0)
        d.run(0, 30, 30)
        d.sync()
        f, mv = d.download_f(), d.download_mv()
    fo, mvo = po.run_oracle(p, f0.copy(), sol, 0, 30, 30)
    assert_close(f, mv, fo, mvo, sol, dtype,
                 fp64_truth(p, f0, sol, 30, 30) if dtype == np.float32 else None)
    # the inlet plane holds the profile after an even step
    C = mvo[1, 0].reshape(p.LZ, p.LY, p.LX)[0].reshape(-1)
    fl = (sol.reshape(p.LZ, -1)[0] != 1)
    assert np.abs(C[fl] - prof[fl]).max() < (1e-12 if dtype == np.float64 else 1e-6)


def test_gpu_flow_only_record_has_ux():
    """A flow-only lattice records u_x means (C channel NaN)."""
    p = po.Params(dims=3, LX=16, LY=12, LZ=10, tau=(0.8, 1.0), gaccel=(1e-5, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(16, 12, 10, radius=2, porosity=0.6, seed=2)
    f0 = np.zeros((1, 19, p.NN))
    with lbx.Domain(to_lbx(p, np.float64, "compact"), sol) as d:
        d.upload_f(f0)
        d.btc_start(4, 20)
        d.run(0, 20, 0)
        c, ux = d.btc_read(ux=True)
    _, _, _, ux_o = po.run_oracle_btc(p, f0.copy(), sol, 0, 20, 4)
    assert np.isnan(c).all()
    assert np.abs(ux - ux_o).max() <= 1e-12 * np.abs(ux_o).max()


@pytest.mark.parametrize("model,prec", [((1, 0), 8), ((1, 1), 8), ((1, 0), 4)])
def test_gpu_velocity_face_imposes_the_momentum(model, prec):
    """Every fluid node of a velocity face leaves the step with momentum
    J = rho u_z(bc) and zero tangential momentum (mv holds u = J / den + tau g
    with den = rho_A for shifted incompressible populations, rho otherwise;
    no force here)."""
    acc, comp = model
    LX, LY, LZ = 24, 20, 32
    lp = lbx.Params(dims=3, LX=LX, LY=LY, LZ=LZ, precision=prec, accurate=acc,
                    compressible=comp, tau=(0.8, 1.0), velocity_t_in=(1, 0), uz_in=-0.02,
                    pressure_b_out=(1, 0), rho_out=1.0)
    sol = geometry.sphere_pack(LX, LY, LZ, radius=3, porosity=0.6, seed=12)
    with lbx.Domain(lp, sol) as d:
        d.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        d.run(0, 60, 60)
        d.sync()
        mv = d.download_mv()[0].astype(np.float64).reshape(4, LZ, LY, LX)
    top = sol.reshape(LZ, LY, LX)[-1] != 1
    rho, ux, uy, uz = (mv[c, -1][top] for c in range(4))
    den = np.ones_like(rho) if comp == 0 else rho
    tol = 1e-12 if prec == 8 else 2e-6
    assert np.allclose(uz * den, rho * -0.02, rtol=tol, atol=0)
    assert np.max(np.abs(ux)) < 0.05 and np.max(np.abs(uy)) < 0.05


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("prec", [8, 4])
def test_gpu_pressure_faces_impose_the_density(layout, prec):
    """Every fluid node of a Zou-He pressure face leaves an even step with
    the imposed density: the rule sets the unknowns so that the node's
    populations sum to rho_in (bottom) / rho_out (top), and the even step
    collides those populations in place, so its rho is that sum (the shifted
    sums plus rho_A).  After an odd step the node holds populations pulled
    from its neighbours, whose sum is not pinned.  Checked in a developed run
    of the flow + solute lattice, both z faces, solid neighbours included."""
    LX, LY, LZ = 24, 20, 32
    lp = lbx.Params(dims=3, LX=LX, LY=LY, LZ=LZ, nsubs=2, precision=prec, tau=(0.9, 0.7),
                    pressure_b_in=(1, 0), pressure_t_out=(1, 0), rho_in=1.0012,
                    rho_out=0.9995, constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0,
                    layout=lbx.LBX_LAYOUT_DENSE if layout == "dense" else lbx.LBX_LAYOUT_COMPACT)
    sol = geometry.sphere_pack(LX, LY, LZ, radius=3, porosity=0.6, seed=14)
    with lbx.Domain(lp, sol) as d:
        d.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        d.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
        d.run(0, 200, 200)             # ends on an even (in-place) step
        d.sync()
        mv = d.download_mv()[0].astype(np.float64).reshape(4, LZ, LY, LX)
    tol = 1e-12 if prec == 8 else 2e-6
    for k, rho_bc in ((0, 1.0012), (LZ - 1, 0.9995)):
        fluid = sol.reshape(LZ, LY, LX)[k] != 1
        rho = mv[0, k][fluid]
        assert fluid.any()
        assert np.abs(rho - rho_bc).max() <= tol * rho_bc, (k, np.abs(rho - rho_bc).max())
    # the flow is developed: the interior density lies between the two
    inner = mv[0, LZ // 2][sol.reshape(LZ, LY, LX)[LZ // 2] != 1]
    assert 0.9995 < inner.mean() < 1.0012


@pytest.mark.parametrize("case", ["inlet_bottom", "velocity_top_in", "velocity_both"])
def test_gpu_z_faces_fused_equal_standalone(case):
    """With fluid planes across the z wrap the compact layout applies the z
    faces inside a step launch over the two face planes (no stand-alone
    face-plane kernel); the dense layout keeps the stand-alone face kernels.
    FP64 results are bit-identical."""
    p, sol, f0 = _flow_solute(18, 16, 12, 0.6, 13, **CASES[case])
    m3 = sol.reshape(12, 16, 18)
    m3[0] = 0
    m3[-1] = 0
    sol = m3.reshape(-1)
    if case == "inlet_bottom":
        p.constcon_profile_b = np.random.default_rng(2).uniform(0, 1, p.LX * p.LY)
    out = {}
    for layout in ("dense", "compact"):
        with lbx.Domain(to_lbx(p, np.float64, layout), sol) as d:
            if p.constcon_profile_b is not None:
                d.set_face_profile(False, p.constcon_profile_b)
            d.upload_f(f0)
            n0 = d.launch_count()
            for t in range(1, 31):
                d.step(t, write_mv=(t == 30))
            launches = d.launch_count() - n0
            d.sync()
            out[layout] = (d.download_f(), d.download_mv(), launches)
    assert np.array_equal(out["dense"][0], out["compact"][0])
    assert np.array_equal(out["dense"][1], out["compact"][1])
    # dense: face plane + flow + solute per step; compact: the two face
    # planes (every substance) and the interior, flow and solute in one
    # launch on odd steps, two on even steps
    assert out["compact"][2] == 2 * 15 + 3 * 15 and out["dense"][2] == 3 * 30
    fo, mvo = po.run_oracle(p, f0.copy(), sol, 0, 30, 30)
    assert_close(out["compact"][0], out["compact"][1], fo, mvo, sol, np.float64)


def test_gpu_z_faces_side_stream_on_every_path():
    """The compact layout's face-plane launch (and the record of a face
    plane) run on a second stream, forked from and joined back into the
    step's stream.  Step by step, replayed from captured graphs, on a
    caller's stream and on the CUDA default stream (direct launches), FP64
    results and the record are bit-identical, and equal to the oracle."""
    torch = pytest.importorskip("torch")
    p, sol, f0 = _flow_solute(18, 16, 12, 0.6, 21, **CASES["inlet_bottom"])
    m3 = sol.reshape(12, 16, 18)
    m3[0] = 0
    m3[-1] = 0
    sol = m3.reshape(-1)
    steps = 40
    out = {}
    for how in ("steps", "graphs", "caller_stream", "default_stream"):
        with lbx.Domain(to_lbx(p, np.float64, "compact"), sol) as d:
            s = torch.cuda.Stream() if how == "caller_stream" else None
            if s is not None:
                d.set_stream(s.cuda_stream)
            if how == "default_stream":
                d.set_stream(None)
            d.upload_f(f0)
            d.btc_start(p.LZ - 1, steps)
            if how == "steps":
                for t in range(1, steps + 1):
                    d.step(t, write_mv=(t == steps))
            else:
                d.run(0, steps, steps)
            if s is not None:
                s.synchronize()
                d.set_stream(None)
            d.sync()
            out[how] = (d.download_f(), d.download_mv(), d.btc_read(ux=True))
    for how in ("graphs", "caller_stream", "default_stream"):
        assert np.array_equal(out[how][0], out["steps"][0]), how
        assert np.array_equal(out[how][1], out["steps"][1]), how
        for c in range(2):
            assert np.array_equal(out[how][2][c], out["steps"][2][c], equal_nan=True), how
    fo, mvo, btc_o, ux_o = po.run_oracle_btc(p, f0.copy(), sol, 0, steps, p.LZ - 1,
                                             frame_rate=steps)
    assert_close(out["steps"][0], out["steps"][1], fo, mvo, sol, np.float64)
    live = ~np.isnan(btc_o)
    assert np.abs(out["steps"][2][0][live] - btc_o[live]).max() <= \
        1e-12 * np.abs(btc_o[live]).max()
