"""The largest lattices (GPU): 64-bit population offsets.

The compact kernels keep slot offsets in 32 bits while 19 x P < 2^32 (P the
fluid count rounded up to 32); a lattice with more than 226M fluid nodes
takes the 64-bit form.  A 624^3 lattice (243M nodes, 1% solids) runs three
steps on the compact layout (64-bit offsets) and on the dense layout (32-bit
node indices, 64-bit plane offsets) from the same non-uniform state; both
compute each node's update in the same arithmetic, so the macro variables
must agree bit for bit.  About 45 GB of device memory per domain, one
domain at a time.
"""
import numpy as np
import pytest

import lbx

pytestmark = pytest.mark.gpu

N_EDGE = 624


def _state(n):
    k = np.arange(n, dtype=np.float32)
    ux = (0.02 * np.sin(2 * np.pi * k / n)).astype(np.float32)      # shear wave along z
    i = np.arange(n, dtype=np.float32)
    rho = (1.0 + 1e-3 * np.cos(2 * np.pi * i / n)).astype(np.float32)  # density wave along x
    rho_f = np.broadcast_to(rho[None, None, :], (n, n, n)).reshape(-1)
    ux_f = np.broadcast_to(ux[:, None, None], (n, n, n)).reshape(-1)
    return rho_f, ux_f


def _run(layout, mask, rho, ux):
    n = N_EDGE
    p = lbx.Params(dims=3, LX=n, LY=n, LZ=n, precision=4, tau=(0.8, 1.0),
                   gaccel=(1e-6, 0, 0, 0, 0, 0), layout=layout)
    with lbx.Domain(p, mask) as d:
        assert d.info()["layout"] == {lbx.LBX_LAYOUT_DENSE: "dense",
                                      lbx.LBX_LAYOUT_COMPACT: "compact"}[layout]
        d.init_equilibrium(0, rho, ux, 0.0, 0.0)
        d.run(0, 3, 3)
        d.sync()
        fluid = d.info()["fluid_nodes"]
        return d.download_mv()[0], fluid


def test_gpu_64bit_offsets_equal_dense_layout():
    n = N_EDGE
    rng = np.random.default_rng(77)
    mask = (rng.random(n ** 3) < 0.01).astype(np.uint8)
    rho, ux = _state(n)
    mv_c, fluid = _run(lbx.LBX_LAYOUT_COMPACT, mask, rho, ux)
    assert 19 * ((fluid + 31) // 32 * 32) >= 2 ** 32      # the 64-bit offset path
    mv_d, _ = _run(lbx.LBX_LAYOUT_DENSE, mask, rho, ux)
    fl = mask != 1
    for c in range(4):
        assert np.array_equal(mv_c[c][fl], mv_d[c][fl]), c
    assert np.all(np.isfinite(mv_c[:, fl]))
