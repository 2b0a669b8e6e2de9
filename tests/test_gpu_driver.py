"""The C host driver (bin/lbgpu_b200, the reference's main) end to end.

Each case writes the reference's input files (in/params.in, the solid mask,
the Walsh fraction file), runs the driver in a scratch directory and
compares its last frame of .dat files -- binary reals, zero where the mask
byte is non-zero -- with the CPU oracle run from the same initial state
(equilibrium at the initial density, u = 0).  Tolerances (norm-wise
relative): FP64 1e-12, FP32 1e-5.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

import pyoracle as po
from lbx import geometry, host
from _golden import rel_err
from _host_files import write_params

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "lbgpu-prime-dev_b200", "bin", "lbgpu_b200")
TOL = {8: 1e-12, 4: 1e-5}


def run_driver(tmp, args):
    r = subprocess.run([DRIVER] + args, cwd=tmp, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def oracle_last_frame(hp, dims, prec, mask, steps, fr, **kw):
    """The oracle's macro variables at the last frame, with the driver's
    parameters and initial state."""
    rv = (lambda x: x.f) if prec == 4 else (lambda x: x.d)
    p = po.Params(dims=dims, LX=hp.LX, LY=hp.LY, LZ=hp.LZ,
                  tau=(rv(hp.tau[0]), rv(hp.tau[1])), rho_A=(rv(hp.rho_A[0]), rv(hp.rho_A[1])),
                  gaccel=tuple(rv(hp.gforce[s][c]) for s in range(2) for c in range(3)),
                  rho_in=rv(hp.rho_in), rho_out=rv(hp.rho_out),
                  bc_ramp_start=hp.bc_ramp_start, bc_ramp_stop=hp.bc_ramp_stop, **kw)
    dtype = np.float32 if prec == 4 else np.float64
    rho = host.initial_rho(hp, dims, 1, 0).astype(dtype).astype(np.float64)
    z = np.zeros(p.NN)
    f = po.init_feq(p, rho[None], z[None], z[None], z[None], dtype=dtype)
    f, mv = po.run_oracle(p, f, mask, 0, steps, fr)
    return mv


def read_frame(tmp, name, frame, prec):
    path, = glob.glob(os.path.join(tmp, "out", "cuda_%s*_frame%04d.dat" % (name, frame)))
    return np.fromfile(path, dtype=np.float32 if prec == 4 else np.float64)


def check_frame(tmp, mv, mask, dims, frame, prec):
    solid = mask != 0
    for c, name in enumerate(["rho", "u_x", "u_y", "u_z"][:dims + 1]):
        a = read_frame(tmp, name, frame, prec)
        assert np.all(a[solid] == 0)
        e = rel_err(a[~solid], mv[0, c][~solid])
        assert e <= TOL[prec], "%s: %g" % (name, e)


BASE = {"NumFrames": 3, "FrameRate": 10, "tau[0]": 0.9, "tau[1]": 1.0, "rho_A[0]": 1.0,
        "rho_A[1]": 1.0, "bc_ramp_start": -1, "bc_ramp_stop": -1, "sigma_t_on": -1,
        "sigma_t_off": -1, "initial_condition": 0, "x0": -1, "r0": -1}


def test_gpu_driver_2d_pressure_faces(tmp_path):
    """The reference's default build (2D, FP64, shifted) between Zou-He
    pressure faces, with a disc-pack .bmp mask."""
    tmp = str(tmp_path)
    os.makedirs(os.path.join(tmp, "in"))
    LX, LY = 40, 32
    write_params(os.path.join(tmp, "in", "params.in"),
                 dict(BASE, LX=LX, LY=LY, LZ=1, rho_in=1.002, rho_out=1.0,
                      **{"pressure_s_in[0]": 1, "pressure_n_out[0]": 1}))
    mask = geometry.transpose_2d(geometry.disc_pack(LY, LX, radius=3, porosity=0.6, seed=4),
                                 LY, LX)
    host.write_bmp_mask(os.path.join(tmp, "in", "%dx%d.bmp" % (LX, LY)), LX, LY, mask)
    run_driver(tmp, [])
    hp = host.read_params(os.path.join(tmp, "in", "params.in"), 2, 1)
    mv = oracle_last_frame(hp, 2, 8, mask, 30, 10, pressure_s_in=(1, 0),
                           pressure_n_out=(1, 0))
    check_frame(tmp, mv, mask, 2, 3, 8)
    frames, = glob.glob(os.path.join(tmp, "out", "cuda_frames*.dat"))
    rows = [ln.split() for ln in open(frames) if ln.split() and ln.split()[0].isdigit()]
    assert [int(r[0]) for r in rows] == [0, 10, 20, 30]


@pytest.mark.parametrize("prec", [8, 4])
def test_gpu_driver_3d_walsh_from_file(tmp_path, prec):
    """--walsh in 3D with ns_flag 1: the fraction field is byte / 255 of
    in/ns<LX>x<LY>x<LZ>.raw; every node is updated."""
    tmp = str(tmp_path)
    os.makedirs(os.path.join(tmp, "in"))
    LX, LY, LZ = 20, 18, 16
    write_params(os.path.join(tmp, "in", "params.in"),
                 dict(BASE, LX=LX, LY=LY, LZ=LZ, ns_flag=1, **{"gforce[0][0]": 2e-5}))
    mask = np.zeros(LX * LY * LZ, np.uint8)
    host.write_raw_mask(os.path.join(tmp, "in", "%dx%dx%d.raw" % (LX, LY, LZ)), mask)
    rng = np.random.default_rng(41)
    raw = rng.integers(0, 256, LX * LY * LZ).astype(np.uint8)
    raw.tofile(os.path.join(tmp, "in", "ns%dx%dx%d.raw" % (LX, LY, LZ)))
    run_driver(tmp, ["--dims", "3", "--precision", str(prec), "--walsh"])
    hp = host.read_params(os.path.join(tmp, "in", "params.in"), 3, 1)
    mv = oracle_last_frame(hp, 3, prec, mask, 30, 10, walsh=1, ns=raw / 255.0)
    check_frame(tmp, mv, mask, 3, 3, prec)


def test_gpu_driver_2d_walsh_mask_rule(tmp_path):
    """--walsh in 2D: ns = the params.in value where the mask is solid, 0
    elsewhere (the field the reference's 2D runs upload)."""
    tmp = str(tmp_path)
    os.makedirs(os.path.join(tmp, "in"))
    LX, LY = 36, 30
    write_params(os.path.join(tmp, "in", "params.in"),
                 dict(BASE, LX=LX, LY=LY, LZ=1, ns=0.6, **{"gforce[0][0]": 1e-5}))
    mask = geometry.transpose_2d(geometry.disc_pack(LY, LX, radius=3, porosity=0.7, seed=5),
                                 LY, LX)
    host.write_bmp_mask(os.path.join(tmp, "in", "%dx%d.bmp" % (LX, LY)), LX, LY, mask)
    run_driver(tmp, ["--walsh"])
    hp = host.read_params(os.path.join(tmp, "in", "params.in"), 2, 1)
    mv = oracle_last_frame(hp, 2, 8, mask, 30, 10, walsh=1, ns=np.where(mask == 1, 0.6, 0.0))
    check_frame(tmp, mv, mask, 2, 3, 8)


def oracle_frames(hp, dims, prec, mask, nframes, fr, **kw):
    """The oracle's macro variables at frames 0..nframes, starting from the
    driver's initial state (solid nodes keep their initial values, as on
    the device)."""
    rv = (lambda x: x.f) if prec == 4 else (lambda x: x.d)
    p = po.Params(dims=dims, LX=hp.LX, LY=hp.LY, LZ=hp.LZ,
                  tau=(rv(hp.tau[0]), rv(hp.tau[1])), rho_A=(rv(hp.rho_A[0]), rv(hp.rho_A[1])),
                  gaccel=tuple(rv(hp.gforce[s][c]) for s in range(2) for c in range(3)),
                  rho_in=rv(hp.rho_in), rho_out=rv(hp.rho_out),
                  bc_ramp_start=hp.bc_ramp_start, bc_ramp_stop=hp.bc_ramp_stop, **kw)
    dtype = np.float32 if prec == 4 else np.float64
    rho = host.initial_rho(hp, dims, 1, 0).astype(dtype)
    z = np.zeros(p.NN)
    f = po.init_feq(p, rho.astype(np.float64)[None], z[None], z[None], z[None], dtype=dtype)
    mv = np.zeros((1, 1 + dims, p.NN), dtype=dtype)
    mv[0, 0] = rho
    out = [mv.copy()]
    for k in range(nframes):
        f, mv = po.run_oracle(p, f, mask, k * fr, fr, fr, mv=mv)
        out.append(mv.copy())
    return out


@pytest.mark.parametrize("dims,prec", [(3, 8), (2, 4)])
def test_gpu_driver_frame_files_match_reference_output_frame(tmp_path, dims, prec):
    """Every file the driver writes per frame against the reference's own
    output_frame (built by the harness) fed with the oracle's macro variables
    at the same frames: the same file names; .dat and .txt values within the
    parity bar; byte images within one level (a value on a rounding edge);
    summary columns to the printed 7 decimals (FP32 means within the
    reference's float running sums)."""
    variant = ("d3q19" if dims == 3 else "d2q9") + ("_f64" if prec == 8 else "_f32")
    if not po.reference_available(variant):
        pytest.skip("reference harness not built")
    tmp = str(tmp_path / "run")
    os.makedirs(os.path.join(tmp, "in"))
    LX, LY, LZ = (12, 10, 8) if dims == 3 else (20, 14, 1)
    N = LX * LY * LZ
    write_params(os.path.join(tmp, "in", "params.in"),
                 dict(BASE, LX=LX, LY=LY, LZ=LZ, NumFrames=3, FrameRate=6,
                      **{"gforce[0][0]": 3e-5, "gforce[0][1]": -1e-5}))
    rng = np.random.default_rng(51)
    mask = rng.choice([0, 1, 255], size=N, p=[0.75, 0.2, 0.05]).astype(np.uint8)
    if dims == 3:
        host.write_raw_mask(os.path.join(tmp, "in", "%dx%dx%d.raw" % (LX, LY, LZ)), mask)
    else:
        mask = np.where(mask == 255, 0, mask).astype(np.uint8)   # a BMP holds 0/1 only
        host.write_bmp_mask(os.path.join(tmp, "in", "%dx%d.bmp" % (LX, LY)), LX, LY, mask)
    run_driver(tmp, ["--dims", str(dims), "--precision", str(prec)])
    hp = host.read_params(os.path.join(tmp, "in", "params.in"), dims, 1)
    ref = str(tmp_path / "ref")
    for k, mv in enumerate(oracle_frames(hp, dims, prec, mask, 3, 6)):
        assert po.reference_output_frame(variant, LX, LY, LZ, mv, mask, 6 * k, k, 6, ref)
    names = sorted(os.listdir(os.path.join(ref, "out")))
    assert names == sorted(os.listdir(os.path.join(tmp, "out")))
    dtype = np.float32 if prec == 4 else np.float64
    tol = TOL[prec]
    for name in names:
        a_path, b_path = os.path.join(ref, "out", name), os.path.join(tmp, "out", name)
        if name.endswith(".raw"):
            a = np.fromfile(a_path, np.uint8).astype(int)
            b = np.fromfile(b_path, np.uint8).astype(int)
            d = np.minimum(np.abs(a - b), 256 - np.abs(a - b))
            assert d.max() <= 1 and np.mean(d != 0) < 0.02, name
        elif "_frames" in name:
            ra = [ln.split() for ln in open(a_path) if ln.split() and ln.split()[0].isdigit()]
            rb = [ln.split() for ln in open(b_path) if ln.split() and ln.split()[0].isdigit()]
            assert len(ra) == len(rb) == 4
            for x, y in zip(ra, rb):
                for kk, (u, v) in enumerate(zip(x, y)):
                    u, v = float(u), float(v)
                    slack = 1e-5 * abs(u) if kk in (14, 15, 16, 20) else 2e-7
                    assert abs(u - v) <= slack + (1e-6 if prec == 4 else 0.0), (name, kk, u, v)
        elif name.endswith(".dat"):
            assert rel_err(np.fromfile(b_path, dtype), np.fromfile(a_path, dtype)) <= tol, name
        else:
            a = np.array(open(a_path).read().split(), dtype=np.float64)
            b = np.array(open(b_path).read().split(), dtype=np.float64)
            assert rel_err(b, a) <= tol, name


def test_gpu_driver_zfaces_velocity_inflow(tmp_path):
    """--zfaces in 3D: the z-face boundaries of params.in (here Zou-He
    velocity inflow on the top plane, pressure outflow on the bottom)."""
    tmp = str(tmp_path)
    os.makedirs(os.path.join(tmp, "in"))
    LX, LY, LZ = 18, 16, 20
    write_params(os.path.join(tmp, "in", "params.in"),
                 dict(BASE, LX=LX, LY=LY, LZ=LZ, uz_in=-0.01, rho_out=1.0,
                      **{"velocity_t_in[0]": 1, "pressure_b_out[0]": 1}))
    mask = geometry.sphere_pack(LX, LY, LZ, radius=3, porosity=0.6, seed=17)
    host.write_raw_mask(os.path.join(tmp, "in", "%dx%dx%d.raw" % (LX, LY, LZ)), mask)
    run_driver(tmp, ["--dims", "3", "--zfaces", "--frames", "dat"])
    hp = host.read_params(os.path.join(tmp, "in", "params.in"), 3, 1)
    assert hp.velocity_t_in[0] == 1 and hp.pressure_b_out[0] == 1
    mv = oracle_last_frame(hp, 3, 8, mask, 30, 10, velocity_t_in=(1, 0), uz_in=hp.uz_in.d,
                           pressure_b_out=(1, 0))
    check_frame(tmp, mv, mask, 3, 3, 8)
