"""The forward-mode (tangent) derivative of the oracle (CPU).

The oracle's complex-step build runs the FP64 model with tau, tau_s, g_x and
the inlet profile given imaginary parts i h v; the imaginary part of the
plane objective is then h times dJ/dp . v, exact to rounding.  Here it is
checked against central differences of the real FP64 oracle, and its real
part against the real run bit for bit.  tests/test_gpu_adjoint.py compares
the product's discrete adjoint with it.
"""
import dataclasses

import numpy as np
import pytest

import pyoracle as po
from lbx import geometry

OBJ = (5, 21, 40, 1.0, 0.5)        # plane, t_first, t_last, w_c, w_ux


def case():
    LX, LY, LZ = 12, 10, 8
    mask = geometry.sphere_pack(LX, LY, LZ, radius=2, porosity=0.6, seed=4)
    m3 = mask.reshape(LZ, LY, LX)
    m3[0] = 0
    m3[-1] = 0
    prof = np.random.default_rng(4).uniform(0, 1, LX * LY)
    p = po.Params(dims=3, LX=LX, LY=LY, LZ=LZ, nsubs=2, tau=(0.8, 0.75),
                  gaccel=(2e-4, 0, 0, 0, 0, 0), sigma_t_on=0, sigma_t_off=1 << 30,
                  constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0,
                  constcon_profile_b=prof)
    rho = np.stack([np.ones(p.NN), np.zeros(p.NN)])
    z = np.zeros((2, p.NN))
    return p, mask, po.init_feq(p, rho, z, z, z)


def J64(p, f0, mask):
    plane, t1, t2, wc, wu = OBJ
    _, _, btc, bux = po.run_oracle_btc(p, f0.copy(), mask, 0, t2, plane)
    return wc * np.mean(btc[t1 - 1:t2]) + wu * np.mean(bux[t1 - 1:t2])


@pytest.mark.parametrize("which", ["gx", "tau", "tau_s", "profile"])
def test_complex_step_tangent_matches_central_differences(which):
    p, mask, f0 = case()
    v = np.random.default_rng(9).standard_normal(p.LX * p.LY)
    kw = {"gx": dict(d_gaccel=(1, 0, 0, 0, 0, 0)), "tau": dict(d_tau=(1, 0)),
          "tau_s": dict(d_tau=(0, 1)), "profile": dict(d_profile_b=v)}[which]
    J, dJ = po.tangent_objective(p, f0, mask, OBJ[2], *OBJ, **kw)
    assert J == J64(p, f0, mask)

    def shifted(e):
        if which == "gx":
            return dataclasses.replace(p, gaccel=(p.gaccel[0] + e,) + tuple(p.gaccel[1:]))
        if which == "tau":
            return dataclasses.replace(p, tau=(p.tau[0] + e, p.tau[1]))
        if which == "tau_s":
            return dataclasses.replace(p, tau=(p.tau[0], p.tau[1] + e))
        return dataclasses.replace(p, constcon_profile_b=p.constcon_profile_b + e * v)
    h = {"gx": 1e-9, "tau": 1e-6, "tau_s": 1e-6, "profile": 1e-3}[which]
    fd = (J64(shifted(h), f0, mask) - J64(shifted(-h), f0, mask)) / (2 * h)
    assert dJ != 0.0
    assert abs(dJ - fd) <= 1e-5 * abs(dJ), (dJ, fd)


def test_complex_step_is_linear_in_the_direction():
    p, mask, f0 = case()
    _, a = po.tangent_objective(p, f0, mask, OBJ[2], *OBJ, d_tau=(1, 0))
    _, b = po.tangent_objective(p, f0, mask, OBJ[2], *OBJ, d_gaccel=(1, 0, 0, 0, 0, 0))
    _, ab = po.tangent_objective(p, f0, mask, OBJ[2], *OBJ, d_tau=(2, 0),
                                 d_gaccel=(-3, 0, 0, 0, 0, 0))
    assert abs(ab - (2 * a - 3 * b)) <= 1e-12 * (abs(2 * a) + abs(3 * b))
