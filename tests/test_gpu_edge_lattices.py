"""Lattices at the edge of the node rule (GPU): no fluid node at all, and a
single fluid node boxed in by solids.

The reference's kernels skip solid nodes (src/k_stream_collide_stream.c,
src/k_collide.c: `if (!is_solid)`), so a lattice without fluid nodes is
never written, and a lone fluid node bounces every population back.  Both
layouts, 2D (per-step and tiled runs, with pressure faces) and 3D (with z
faces and the outlet-plane record), against the oracle.
"""
import numpy as np
import pytest

import lbx
import pyoracle as po
from _golden import rel_err
from test_gpu_parity import to_lbx

pytestmark = pytest.mark.gpu


def _params(dims, nsubs=1, faces=False):
    if dims == 2:
        kw = dict(pressure_s_in=(1, 0), pressure_n_out=(1, 0), rho_in=1.001,
                  rho_out=1.0) if faces else dict(gaccel=(1e-5, 0, 0, 0, 0, 0))
        return po.Params(dims=2, LX=64, LY=32, LZ=1, tau=(0.9, 1.0), **kw)
    kw = dict(pressure_b_in=(1, 0), pressure_t_out=(1, 0), rho_in=1.001, rho_out=1.0,
              constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0) if faces else \
        dict(gaccel=(1e-5, 0, 0, 0, 0, 0))
    return po.Params(dims=3, LX=12, LY=10, LZ=8, nsubs=nsubs, tau=(0.9, 0.7), **kw)


def _run(p, sol, f0, steps, layout, mode="auto", record=None):
    with lbx.Domain(to_lbx(p, np.float64, layout), sol) as d:
        if p.dims == 2:
            d.set_run_mode(mode)
        d.upload_f(f0)
        if record is not None:
            d.btc_start(record, steps)
        d.run(0, steps, steps)
        d.sync()
        out = (d.download_f(), d.download_mv(), d.reduce(), d.info())
        if record is not None:
            out = out + (d.btc_read(ux=True),)
        return out


CASES = [(2, 1, False, "steps"), (2, 1, True, "steps"), (2, 1, True, "tiled"),
         (3, 1, False, "auto"), (3, 2, True, "auto")]


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dims,nsubs,faces,mode", CASES)
def test_gpu_lattice_without_fluid_nodes(dims, nsubs, faces, mode, layout):
    """Every node solid: nothing is written, reductions count no fluid node."""
    p = _params(dims, nsubs, faces)
    sol = np.ones(p.NN, np.uint8)
    f0 = np.random.default_rng(1).standard_normal((p.nsubs, p.Q, p.NN))
    res = _run(p, sol, f0, 20, layout, mode, record=p.LZ - 1 if dims == 3 else None)
    f, mv, red, info = res[:4]
    assert info["fluid_nodes"] == 0
    assert np.array_equal(f, f0)
    assert not mv.any()
    assert red["status"] == lbx.LBX_OK
    assert red["fluid_nodes"] == 0 and red["mass"] == 0.0 and red["nonfinite"] == 0
    fo, _ = po.run_oracle(p, f0.copy(), sol, 0, 20, 20)
    assert np.array_equal(fo, f0)


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dims,nsubs,faces,mode", CASES)
def test_gpu_single_fluid_node(dims, nsubs, faces, mode, layout):
    """One fluid node among solids bounces every population back: the run
    equals the oracle's at 1e-12, and only that node's slots change."""
    p = _params(dims, nsubs, faces)
    sol = np.ones(p.NN, np.uint8)
    c = (p.LX // 2) + p.LX * ((p.LY // 2) + p.LY * (p.LZ // 2 if dims == 3 else 0))
    sol[c] = 0
    rng = np.random.default_rng(2)
    f0 = rng.standard_normal((p.nsubs, p.Q, p.NN)) * 1e-3
    if nsubs == 2:
        f0[1] = np.abs(f0[1])
    f, mv, red, info = _run(p, sol, f0, 20, layout, mode)[:4]
    assert info["fluid_nodes"] == 1 and red["fluid_nodes"] == 1
    fo, mvo = po.run_oracle(p, f0.copy(), sol, 0, 20, 20)
    assert rel_err(f, fo) <= 1e-12
    others = np.ones(p.NN, bool)
    others[c] = False
    assert np.array_equal(f[..., others], f0[..., others])
    for s in range(p.nsubs):
        for k in range(1 + dims):
            assert abs(mv[s, k, c] - mvo[s, k, c]) <= 1e-12 * max(1.0, abs(mvo[s, k, c]))
