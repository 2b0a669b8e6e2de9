"""PEST point sampling on the GPU: lbx_pest_set / lbx_pest_read against the
oracle's restatement (pinned to the reference's own sampling code on the
CPU), on both layouts, and the C driver's PEST files against the
reference's sampling run through the harness.  Tolerances (relative, per
value): FP64 1e-12, FP32 1e-5.
"""
import os
import subprocess

import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import host
from _host_files import write_params
from test_gpu_driver import BASE, DRIVER

pytestmark = pytest.mark.gpu

TOL = {8: 1e-12, 4: 1e-5}


def close(a, b, tol):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-30) + 1e-300)


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dims,prec", [(2, 8), (3, 4)])
def test_gpu_pest_matches_oracle(dims, prec, layout):
    LX, LY, LZ = (40, 30, 1) if dims == 2 else (24, 20, 16)
    p = po.Params(dims=dims, LX=LX, LY=LY, LZ=LZ, nsubs=2, tau=(0.9, 0.8), sink=1e-3,
                  sigma_t_on=2, sigma_t_off=60, gaccel=(1e-4, 3e-5, 0, 0, 0, 0))
    rng = np.random.default_rng(21)
    dtype = np.float32 if prec == 4 else np.float64
    f0 = rng.standard_normal((2, p.Q, p.NN)) * 1e-3
    f0[1] = np.abs(f0[1]) + 0.1
    f0 = f0.astype(dtype)
    sol = (rng.random(p.NN) < 0.2).astype(np.uint8)
    times = np.array([1, 2, 2, 7, 8, 8, 8, 15, 30, 31, 200])
    nodes = rng.integers(0, LX * LY, size=times.size)      # plane 0, as the reference indexes
    lp = lbx.Params(dims=dims, LX=LX, LY=LY, LZ=LZ, nsubs=2, precision=prec, tau=(0.9, 0.8),
                    sink=1e-3, sigma_t_on=2, sigma_t_off=60, gaccel=(1e-4, 3e-5, 0, 0, 0, 0),
                    layout={"dense": lbx.LBX_LAYOUT_DENSE,
                            "compact": lbx.LBX_LAYOUT_COMPACT}[layout])
    steps = 40
    with lbx.Domain(lp, sol) as d:
        d.upload_f(f0)
        d.pest_set(times, nodes)
        d.run(0, steps, 10)              # graph-replayed stretches break at sample times
        got = d.pest_read()
    _, _, c, ux, uy, taken = po.pest_samples(p, f0.copy(), sol, 0, steps, times, nodes)
    assert got["taken"] == taken == 10
    for k, (a, b) in (("conc", (got["conc"], c)), ("ux", (got["ux"], ux)),
                      ("uy", (got["uy"], uy))):
        assert close(a[:taken], b[:taken], TOL[prec]), k
        assert np.all(np.isnan(a[taken:]))


def test_gpu_pest_blocked_by_a_passed_time_and_errors():
    p = lbx.Params(dims=2, LX=16, LY=12, nsubs=2, precision=8)
    sol = np.zeros(p.NN, np.uint8)
    with lbx.Domain(p, sol) as d:
        d.pest_set([0, 3], [5, 6])       # time 0 never comes: nothing after it is taken
        d.run(0, 10, 0)
        assert d.pest_read()["taken"] == 0
        for t, n in (([2, 1], [0, 0]), ([1], [p.NN])):
            with pytest.raises(lbx.LbxError) as ei:
                d.pest_set(t, n)
            assert ei.value.code == lbx.LBX_ERR_INVALID
    p1 = lbx.Params(dims=2, LX=16, LY=12, nsubs=1, precision=8)
    with lbx.Domain(p1, sol) as d:
        with pytest.raises(lbx.LbxError):
            d.pest_set([1], [0])


def test_gpu_driver_pest_files_match_reference(tmp_path):
    """The driver with PEST inputs (2D, two substances, FP64) against the
    reference's sampling around its own kernels from the same initial state."""
    variant = "d2q9s_pest_f64"
    if not po.reference_available(variant):
        pytest.skip("reference harness not built")
    run, ref = str(tmp_path / "run"), str(tmp_path / "ref")
    LX, LY = 24, 18
    vals = dict(BASE, LX=LX, LY=LY, LZ=1, NumFrames=2, FrameRate=10, sink=1e-3,
                sigma_t_on=1, sigma_t_off=100, rho_sigma=1.0,
                **{"gforce[0][0]": 5e-5, "tau[1]": 0.8})
    times, xs, ys = [1, 4, 4, 9, 10, 17, 20], [2, 5, 23, 0, 11, 7, 3], [1, 17, 9, 0, 4, 12, 6]
    mask = (np.random.default_rng(5).random(LX * LY) < 0.15).astype(np.uint8)
    for d in (run, ref):
        os.makedirs(os.path.join(d, "in"))
        write_params(os.path.join(d, "in", "params.in"), vals)
        host.write_bmp_mask(os.path.join(d, "in", "%dx%d.bmp" % (LX, LY)), LX, LY, mask)
        for name, v in (("timestep", times), ("x_coord", xs), ("y_coord", ys)):
            with open(os.path.join(d, "in", name + "_file.in"), "w") as fh:
                fh.write("\n".join(map(str, v)) + "\n")
    r = subprocess.run([DRIVER, "--subs", "2", "--frames", "summary"], cwd=run,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    hp = host.read_params(os.path.join(run, "in", "params.in"), 2, 2)
    p = po.Params(dims=2, LX=LX, LY=LY, LZ=1, nsubs=2, tau=(hp.tau[0].d, hp.tau[1].d),
                  rho_A=(hp.rho_A[0].d, hp.rho_A[1].d),
                  gaccel=tuple(hp.gforce[s][c].d for s in range(2) for c in range(3)),
                  sink=hp.sink.d, sigma_t_on=hp.sigma_t_on, sigma_t_off=hp.sigma_t_off,
                  bc_ramp_start=hp.bc_ramp_start, bc_ramp_stop=hp.bc_ramp_stop)
    rho = np.stack([host.initial_rho(hp, 2, 2, s) for s in range(2)])
    z = np.zeros((2, p.NN))
    f = po.init_feq(p, rho, z, z, None)
    po.reference_pest(variant, p, f, mask, 0, 20, ref)
    for name in ("conc_order", "conc_data", "vel_data"):
        a = open(os.path.join(ref, "out", name + "_proc0000.dat")).read().split()
        b = open(os.path.join(run, "out", name + "_proc0000.dat")).read().split()
        if name == "conc_order":
            assert a == b
        else:
            assert close([float(x) for x in b], [float(x) for x in a], 1e-12), name
