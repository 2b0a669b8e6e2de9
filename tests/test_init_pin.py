"""The start-up path against the reference's own (CPU).

The reference starts a run with read_params (src/params.h:40-660, which
derives the cube bounds' defaults and, with two substances, swaps
rho_A[1] = rho_B[0]) and init_problem (src/latman.c:1270-2063: rho per
initial_condition, u = 0, f = feq, shifted for the flow lattice of an
ACCURATE build).  The fixtures in tests/golden/init/ hold what the
reference's own code made of each params.in (tests/golden/make_golden.py
init).  Here the host library's reader and lbh_initial_rho, followed by the
oracle's restatement of the equilibrium, must reproduce them bit for bit;
the device side of the same path is tests/test_gpu_init_pin.py.
"""
import glob
import os

import numpy as np
import pytest

import pyoracle as po
from lbx import host

INIT_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "init")
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(INIT_DIR, "*.npz")))


def load_init(name, tmp_path):
    """(fixture, host params, dims, nsubs, dtype, oracle Params) of one case."""
    z = np.load(os.path.join(INIT_DIR, name + ".npz"), allow_pickle=False)
    path = str(tmp_path / "params.in")
    with open(path, "w") as fh:
        fh.write(str(z["params_in"]))
    variant = str(z["variant"])
    dims = 2 if variant.startswith("d2q9") else 3
    nsubs = z["f"].shape[0]
    hp = host.read_params(path, dims=dims, nsubs=nsubs)
    letters = variant.split("_")[0].replace("d3q19", "").replace("d2q9", "")
    accurate = 0 if "p" in letters else 1
    compressible = 1 if ("p" in letters or "c" in letters) else 0
    p = po.Params(dims=dims, LX=hp.LX, LY=hp.LY, LZ=hp.LZ, nsubs=nsubs, accurate=accurate,
                  compressible=compressible)
    return z, hp, dims, nsubs, z["f"].dtype, p


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and \
        np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_init_fixtures_present():
    assert len(NAMES) >= 12
    ics = {n.split("_")[1] for n in NAMES}
    assert ics == {"ic0", "ic2"}


@pytest.mark.parametrize("name", NAMES)
def test_host_initial_rho_and_oracle_feq_match_reference(name, tmp_path):
    z, hp, dims, nsubs, dt, p = load_init(name, tmp_path)
    rho = np.stack([host.initial_rho(hp, dims, nsubs, s) for s in range(nsubs)])
    # rho is formed in double on the host and stored in the run's precision,
    # as the reference's `real` params are
    assert same_bits(rho.astype(dt), z["mv"][:, 0]), "initial density"
    assert not np.any(z["mv"][:, 1:]), "the reference starts at rest"
    zero = np.zeros_like(rho)
    f = po.init_feq(p, rho.astype(dt), zero, zero, zero if dims == 3 else None, dtype=dt)
    assert same_bits(f, z["f"]), "equilibrium populations"


@pytest.mark.parametrize("ic", [1, 3, 4])
def test_initial_conditions_the_reference_exits_on_are_rejected(ic, tmp_path):
    """The reference compiles only cases 0 and 2 of init_problem; 1 and 3
    sit inside #if 0 and every other value reaches its `Unhandled case`
    exit (src/latman.c:1340-1376, :1507-1630)."""
    z, hp, dims, nsubs, dt, p = load_init("d3q19_ic2_f64", tmp_path)
    hp.initial_condition = ic
    with pytest.raises(host.HostError, match="not supported"):
        host.initial_rho(hp, dims, nsubs, 0)
