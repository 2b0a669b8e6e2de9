"""Parity at the full geometry of the two-substance and batched configurations
(GPU), where the small-lattice tests cannot reach large-lattice indexing.

* The coupled flow + solute lattice of 192 x 192 x 384 nodes (sphere pack of
  radius 5 to porosity 0.35, tau 0.9 / tau_s 0.7), driven by Zou-He pressure
  on the z faces (rho_in 1.0005 at the bottom, rho_out 1.0 at the top) with
  C = 1 held at the bottom plane and a zero-gradient top, 20 steps against
  the oracle in FP32 and FP64, with the plane record of a plane near the
  inlet.  This drives the two-substance compact kernels' row-window lookups
  and the face-plane kernels over a 14.2M-node lattice.
* A batch of 12 samples whose cubic-ish edges span 32 to 96 nodes (a 96^3
  sample included), tau in [0.6, 1.2], porosity in [0.3, 0.7], sphere radii
  3 to 6, in every batch mode, each sample against the oracle.
The z faces have no reference device code, so their parity is with the
oracle's restatement of the 2D rules carried to z.
"""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from lbx.batch import Batch
from _golden import rel_err
from test_gpu_parity import assert_close, to_lbx

pytestmark = pytest.mark.gpu

CFG3 = dict(LX=192, LY=192, LZ=384, radius=5, porosity=0.35, seed=31)


def cfg3_case():
    c = CFG3
    p = po.Params(dims=3, LX=c["LX"], LY=c["LY"], LZ=c["LZ"], nsubs=2, tau=(0.9, 0.7),
                  pressure_b_in=(1, 0), pressure_t_out=(1, 0), rho_in=1.0005, rho_out=1.0,
                  constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0)
    sol = geometry.sphere_pack(c["LX"], c["LY"], c["LZ"], c["radius"], c["porosity"], c["seed"])
    # the bottom plane is the inlet: keep it fluid, as a column feeding the pack
    sol.reshape(c["LZ"], c["LY"], c["LX"])[0] = 0
    rho = np.stack([np.ones(p.NN), np.zeros(p.NN)])
    z = np.zeros((2, p.NN))
    return p, sol, po.init_feq(p, rho, z, z, z)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gpu_cfg3_full_geometry_matches_oracle(dtype):
    p, sol, f0 = cfg3_case()
    f0 = f0.astype(dtype)
    steps, plane = 20, 4
    with lbx.Domain(to_lbx(p, dtype, "compact"), sol) as d:
        assert d.info()["layout"] == "compact"
        d.upload_f(f0)
        d.btc_start(plane, 64)
        d.run(0, steps, steps)
        btc = d.btc_read()
        f, mv = d.download_f(), d.download_mv()
    fo, mvo, btc_o, _ = po.run_oracle_btc(p, f0, sol, 0, steps, plane, frame_rate=steps)
    assert_close(f, mv, fo, mvo, sol, dtype)
    # the solute front has reached the recorded plane
    assert np.nanmax(btc_o) > 1e-6
    tol = 1e-12 if dtype == np.float64 else 1e-5
    live = ~np.isnan(btc_o)
    assert np.array_equal(live, ~np.isnan(btc))
    assert np.abs(btc[live] - btc_o[live]).max() <= tol * np.abs(btc_o[live]).max()


def cfg4_samples(prec):
    """12 samples, edges spanning 32..96 (both ends included), per-sample
    tau, porosity, radius and seed as the batched configuration draws them."""
    rng = np.random.default_rng(404)
    edges = [32, 96, 40, 88, 48, 80, 56, 72, 64, 33, 95, 61]
    params, masks = [], []
    for i, e in enumerate(edges):
        L = (e, max(32, e - 3 * (i % 3)), max(32, e - 5 * (i % 2)))
        tau = float(rng.uniform(0.6, 1.2))
        por = float(rng.uniform(0.3, 0.7))
        r = int(rng.integers(3, 7))
        masks.append(geometry.sphere_pack(L[0], L[1], L[2], r, por, 5000 + i))
        params.append(lbx.Params(dims=3, LX=L[0], LY=L[1], LZ=L[2], precision=prec,
                                 tau=(tau, 1.0), gaccel=(1e-6, 0, 0, 0, 0, 0)))
    return params, masks


@pytest.mark.parametrize("mode", ["fused", "persistent", "sequential"])
def test_gpu_cfg4_batch_edges_32_to_96_match_oracle(mode):
    params, masks = cfg4_samples(4)
    assert min(p.LX for p in params) == 32 and max(p.LX for p in params) == 96
    rng = np.random.default_rng(2)
    f0 = [(rng.standard_normal((19, p.NN)) * 1e-4).astype(np.float32) for p in params]
    steps = 12
    with Batch(params, masks) as b:
        for i in range(len(params)):
            b.upload_f(i, f0[i])
        b.run(0, steps, steps, mode=mode)
        b.sync()
        out = [(b.download_f(i), b.download_mv(i)) for i in range(len(params))]
    for i, p in enumerate(params):
        q = po.Params(dims=3, LX=p.LX, LY=p.LY, LZ=p.LZ, tau=tuple(p.tau),
                      gaccel=tuple(p.gaccel))
        fo, mvo = po.run_oracle(q, f0[i].reshape(1, 19, -1).copy(), masks[i], 0, steps, steps)
        fl = masks[i] != 1
        assert rel_err(out[i][0], fo[0]) <= 1e-5, (i, rel_err(out[i][0], fo[0]))
        for c in range(4):
            e = rel_err(out[i][1][c], mvo[0, c], fl)
            assert e <= 2e-5, (i, c, e)
