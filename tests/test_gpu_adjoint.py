"""Discrete adjoint (GPU): gradients of plane objectives against central
finite differences of the FP64 forward solve and against the forward-mode
(tangent) derivative of the same FP64 model."""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry

pytestmark = pytest.mark.gpu


def _setup(LX=16, LY=14, LZ=8, por=0.6, seed=21, faces_fluid=True, nsubs=2):
    mask = geometry.sphere_pack(LX, LY, LZ, radius=2, porosity=por, seed=seed)
    if faces_fluid:
        m3 = mask.reshape(LZ, LY, LX)
        m3[0] = 0
        m3[-1] = 0
    kw = dict(dims=3, LX=LX, LY=LY, LZ=LZ, nsubs=nsubs, tau=(0.8, 0.75),
              gaccel=(2e-4, 0, 0, 0, 0, 0), sigma_t_on=0, sigma_t_off=1 << 30,
              layout=lbx.LBX_LAYOUT_COMPACT)
    if nsubs == 2:
        kw.update(constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0)
    profile = np.random.default_rng(seed).uniform(0.0, 1.0, LX * LY)
    return kw, mask, profile


def _J(kw, mask, profile, prec, steps, K, obj, grads=False):
    lp = lbx.Params(precision=prec, **kw)
    with lbx.Domain(lp, mask) as d:
        if kw.get("nsubs", 1) == 2:
            d.set_face_profile(False, profile)
        d.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        if kw.get("nsubs", 1) == 2:
            d.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
        J = d.adjoint_forward(0, steps, K, *obj)
        g = d.adjoint_backward(profile_b=kw.get("nsubs", 1) == 2) if grads else None
    return J, g


def _fd(kw, mask, profile, steps, obj, which, h):
    def with_param(delta):
        k2 = dict(kw)
        prof = profile
        if not isinstance(which, str):
            prof = profile + delta * which
        elif which == "gx":
            g = list(kw["gaccel"]); g[0] += delta; k2["gaccel"] = tuple(g)
        elif which == "tau":
            t = list(kw["tau"]); t[0] += delta; k2["tau"] = tuple(t)
        elif which == "tau_s":
            t = list(kw["tau"]); t[1] += delta; k2["tau"] = tuple(t)
        return _J(k2, mask, prof, 8, steps, steps, obj)[0]
    return (with_param(h) - with_param(-h)) / (2 * h)


# J is linear in the inlet profile (the solute is passive and linear given
# the flow), so profile differences take a large step: no truncation error,
# and far less rounding noise than h = 1e-6.
H_PROFILE = 1e-3
STEPS = 60
OBJS = {"outlet_c": (7, 31, 60, 1.0, 0.0), "outlet_ux": (7, 31, 60, 0.0, 1.0)}


@pytest.mark.parametrize("objective", sorted(OBJS))
def test_gpu_adjoint_fp64_matches_finite_differences(objective):
    kw, mask, prof = _setup()
    obj = OBJS[objective]
    J, g = _J(kw, mask, prof, 8, STEPS, 7, obj, grads=True)
    assert J != 0.0
    v = np.random.default_rng(3).standard_normal(prof.size)
    v /= np.linalg.norm(v)
    checks = [("gx", g["d_gaccel"][0], 1e-6 * kw["gaccel"][0]),
              ("tau", g["d_tau"], 1e-6 * kw["tau"][0]),
              ("tau_s", g["d_tau_s"], 1e-6 * kw["tau"][1]),
              (v, float(g["d_profile_b"] @ v), H_PROFILE)]
    for which, adj, h in checks:
        fd = _fd(kw, mask, prof, STEPS, obj, which, h)
        name = which if isinstance(which, str) else "profile"
        scale = max(abs(fd), abs(adj))
        if scale < 1e-14 * abs(J):          # no dependence (e.g. u_x on tau_s)
            continue
        assert abs(adj - fd) <= 1e-6 * scale, (objective, name, adj, fd)


def _oracle_case(kw, mask, prof):
    """The oracle's parameters and initial state for the same run."""
    p = po.Params(dims=3, LX=kw["LX"], LY=kw["LY"], LZ=kw["LZ"], nsubs=kw["nsubs"],
                  tau=tuple(kw["tau"]), gaccel=tuple(kw["gaccel"]),
                  sigma_t_on=kw["sigma_t_on"], sigma_t_off=kw["sigma_t_off"],
                  constcon_b_in=kw.get("constcon_b_in", 0),
                  zeroconcgrad_t=kw.get("zeroconcgrad_t", 0),
                  rho_sigma_in=kw.get("rho_sigma_in", 1.0),
                  constcon_profile_b=prof if kw["nsubs"] == 2 else None)
    ns = kw["nsubs"]
    rho = np.stack([np.ones(p.NN)] + [np.zeros(p.NN)] * (ns - 1))
    z = np.zeros((ns, p.NN))
    return p, po.init_feq(p, rho, z, z, z)


@pytest.mark.parametrize("objective", sorted(OBJS))
def test_gpu_adjoint_fp64_matches_tangent(objective):
    """adjoint . v against the forward-mode derivative along v of the same
    FP64 discrete model (the oracle run in complex arithmetic, exact to
    rounding), for g_x, tau, tau_s, a random inlet-profile direction and a
    random direction over all of them at once."""
    kw, mask, prof = _setup()
    obj = OBJS[objective]
    J, g = _J(kw, mask, prof, 8, STEPS, 7, obj, grads=True)
    p, f0 = _oracle_case(kw, mask, prof)
    rng = np.random.default_rng(17)
    v = rng.standard_normal(prof.size)
    a = rng.standard_normal(3)
    dirs = {
        "gx": (dict(d_gaccel=(1, 0, 0, 0, 0, 0)), g["d_gaccel"][0]),
        "tau": (dict(d_tau=(1, 0)), g["d_tau"]),
        "tau_s": (dict(d_tau=(0, 1)), g["d_tau_s"]),
        "profile": (dict(d_profile_b=v), float(g["d_profile_b"] @ v)),
        "all": (dict(d_gaccel=(a[0], 0, 0, 0, 0, 0), d_tau=(a[1], a[2]), d_profile_b=v),
                a[0] * g["d_gaccel"][0] + a[1] * g["d_tau"] + a[2] * g["d_tau_s"]
                + float(g["d_profile_b"] @ v)),
    }
    for name, (kwd, adj) in dirs.items():
        Jt, tan = po.tangent_objective(p, f0, mask, STEPS, *obj, **kwd)
        assert Jt == pytest.approx(J, rel=1e-12, abs=0)
        # directions the objective does not depend on (u_x on the solute's
        # parameters) give exactly 0 in the tangent; the adjoint's sums of
        # exact zeros stay 0 there too
        tol = 1e-10 * max(abs(tan), abs(adj)) + 1e-15 * abs(J)
        assert abs(adj - tan) <= tol, (objective, name, adj, tan)


@pytest.mark.parametrize("objective", sorted(OBJS))
def test_gpu_adjoint_fp32_matches_fp64_finite_differences(objective):
    kw, mask, prof = _setup()
    obj = OBJS[objective]
    _, g = _J(kw, mask, prof, 4, STEPS, 10, obj, grads=True)
    for which, adj, h in (("gx", g["d_gaccel"][0], 1e-6 * kw["gaccel"][0]),
                          ("tau", g["d_tau"], 1e-6 * kw["tau"][0]),
                          ("tau_s", g["d_tau_s"], 1e-6 * kw["tau"][1])):
        fd = _fd(kw, mask, prof, STEPS, obj, which, h)
        scale = max(abs(fd), abs(adj))
        if scale == 0.0 or (objective == "outlet_ux" and which == "tau_s"):
            continue
        assert abs(adj - fd) <= 1e-4 * scale, (objective, which, adj, fd)


def test_gpu_adjoint_independent_of_checkpoint_interval():
    kw, mask, prof = _setup()
    obj = (7, 31, 60, 1.0, 0.5)
    res = [_J(kw, mask, prof, 8, STEPS, K, obj, grads=True)[1] for K in (1, 7, 60)]
    for g in res[1:]:
        for k in ("d_tau", "d_tau_s"):
            assert abs(g[k] - res[0][k]) <= 1e-12 * abs(res[0][k])
        assert abs(g["d_gaccel"][0] - res[0]["d_gaccel"][0]) <= 1e-12 * abs(res[0]["d_gaccel"][0])
        np.testing.assert_allclose(g["d_profile_b"], res[0]["d_profile_b"], rtol=1e-11, atol=0)


def test_gpu_adjoint_flow_only_matches_finite_differences():
    kw, mask, prof = _setup(nsubs=1)
    obj = (5, 20, 40, 0.0, 1.0)
    J, g = _J(kw, mask, prof, 8, 40, 9, obj, grads=True)
    for which, adj, h in (("gx", g["d_gaccel"][0], 1e-6 * kw["gaccel"][0]),
                          ("tau", g["d_tau"], 1e-6 * kw["tau"][0])):
        fd = _fd(kw, mask, prof, 40, obj, which, h)
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), abs(adj)), (which, adj, fd)


def test_gpu_adjoint_solid_face_neighbours():
    """Solids on the face planes: deposits behind solids follow the forward's
    slot rules in the adjoint too."""
    kw, mask, prof = _setup(faces_fluid=False, por=0.55, seed=8)
    obj = (7, 31, 60, 1.0, 0.0)
    _, g = _J(kw, mask, prof, 8, STEPS, 6, obj, grads=True)
    v = np.random.default_rng(9).standard_normal(prof.size)
    v /= np.linalg.norm(v)
    for which, adj, h in (("tau_s", g["d_tau_s"], 1e-6 * kw["tau"][1]),
                          (v, float(g["d_profile_b"] @ v), H_PROFILE)):
        fd = _fd(kw, mask, prof, STEPS, obj, which, h)
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), abs(adj))


def test_gpu_adjoint_autograd_function():
    torch = pytest.importorskip("torch")
    from _lbx_autograd import PlaneObjective
    kw, mask, prof = _setup()
    setup = dict(params={k: v for k, v in kw.items() if k not in ("gaccel", "tau")} | {"precision": 8},
                 mask=mask, steps=STEPS, K=7, plane=7, t_first=31, w_c=1.0, w_ux=0.0)
    x = [torch.tensor(kw["gaccel"][0], dtype=torch.float64, requires_grad=True),
         torch.tensor(kw["tau"][0], dtype=torch.float64, requires_grad=True),
         torch.tensor(kw["tau"][1], dtype=torch.float64, requires_grad=True),
         torch.tensor(prof, dtype=torch.float64, requires_grad=True)]
    J = PlaneObjective.apply(*x, setup)
    grads = torch.autograd.grad(J, x)
    _, g = _J(kw, mask, prof, 8, STEPS, 7, (7, 31, 60, 1.0, 0.0), grads=True)
    assert float(grads[0]) == pytest.approx(g["d_gaccel"][0], rel=1e-12)
    assert float(grads[1]) == pytest.approx(g["d_tau"], rel=1e-12)
    assert float(grads[2]) == pytest.approx(g["d_tau_s"], rel=1e-12)
    np.testing.assert_allclose(grads[3].numpy(), g["d_profile_b"], rtol=1e-11, atol=1e-30)


def test_gpu_adjoint_rejects_unsupported():
    kw, mask, prof = _setup()
    for bad in (dict(layout=lbx.LBX_LAYOUT_DENSE), dict(accurate=0, compressible=1),
                dict(pressure_b_in=(1, 0))):
        lp = lbx.Params(precision=8, **{**kw, **bad})
        with lbx.Domain(lp, mask) as d:
            with pytest.raises(lbx.LbxError):
                d.adjoint_forward(0, 10, 5, 7, 1, 10, 1.0, 0.0)
