"""The device side of the start-up path against the reference's own (GPU).

lbx_init_equilibrium (the device form of the feq loop of init_problem,
src/latman.c:1786-1840) fed with lbh_initial_rho's densities must give,
bit for bit, the populations the reference's read_params + init_problem
made of the same params.in (tests/golden/init/, see tests/test_init_pin.py),
on every node: the reference initialises solid nodes too, and the compact
layout returns them exactly as set.  The macro variables then hold what
init_problem leaves in them (rho, u = 0), whether u is passed as zeros
(dense runs) or left out and filled on the device (compact runs).
"""
import numpy as np
import pytest

import lbx
from lbx import host
from test_init_pin import NAMES, load_init, same_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", [lbx.LBX_LAYOUT_DENSE, lbx.LBX_LAYOUT_COMPACT])
@pytest.mark.parametrize("name", NAMES)
def test_gpu_init_equilibrium_matches_reference_init_problem(name, layout, tmp_path):
    z, hp, dims, nsubs, dt, p = load_init(name, tmp_path)
    rho = [host_rho.astype(dt) for host_rho in
           (host.initial_rho(hp, dims, nsubs, s) for s in range(nsubs))]
    mask = (np.random.default_rng(len(name)).random(p.NN) < 0.3).astype(np.uint8)
    lp = lbx.Params(dims=dims, LX=p.LX, LY=p.LY, LZ=p.LZ, nsubs=nsubs,
                    precision=np.dtype(dt).itemsize, accurate=p.accurate,
                    compressible=p.compressible, layout=layout)
    with lbx.Domain(lp, mask) as d:
        for s in range(nsubs):
            if layout == lbx.LBX_LAYOUT_DENSE:
                d.init_equilibrium(s, rho[s], 0.0, 0.0, 0.0 if dims == 3 else None)
            else:
                d.init_equilibrium(s, rho[s])   # u = 0 filled on the device
        d.sync()
        f = d.download_f()
        mv = d.download_mv()
    assert same_bits(f, z["f"])
    # and the macro variables init_problem leaves: rho, and u at rest
    assert same_bits(mv, z["mv"])
