"""The product against the reference's own CUDA kernels, on the same GPU.

oracle/_ref/refgpu_<variant> is the reference's k_stream_collide_stream and
k_collide, unmodified, compiled for sm_100a and launched as its serial main
launches them (oracle/refgpu_harness.cu; built by oracle/ref_build.py where
the reference tree is available).  The product's results must match the
reference GPU build's on the same inputs (the reference's nvcc build may
contract products into FMAs, so FP64 agrees to 1e-12 rather than bit for
bit), and the reference's kernels are timed on the 256^3 benchmark lattice
as the like-for-like context of the product's rate (written to the file
named by $LBX_REFGPU_REPORT when set).
"""
import json
import os
import subprocess

import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from _golden import rel_err

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(po.__file__)), "_ref")


def _binary(variant):
    path = os.path.join(REF_DIR, "refgpu_%s" % variant)
    if not os.path.exists(path):
        pytest.skip("the reference's GPU build is absent (reference tree absent at build)")
    return path


def run_reference_gpu(variant, mask, f0, shape, block, tau, g, steps, tmp_path):
    LX, LY, LZ = shape
    Q, D = (9, 2) if LZ == 1 else (19, 3)
    mpath, fin, fout = (str(tmp_path / x) for x in ("mask.raw", "f_in.bin", "f_out.bin"))
    np.ascontiguousarray(mask, dtype=np.uint8).tofile(mpath)
    np.ascontiguousarray(f0).tofile(fin)
    subprocess.run([_binary(variant), str(LX), str(LY), str(LZ)] + [str(b) for b in block] +
                   [repr(tau)] + [repr(x) for x in g] + [str(steps), mpath, fin, fout],
                   check=True, timeout=300)
    out = np.fromfile(fout, dtype=f0.dtype)
    N = LX * LY * LZ
    return out[:Q * N].reshape(Q, N), out[Q * N:].reshape(1 + D, N)


@pytest.mark.parametrize("layout", ["dense", "compact"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gpu_matches_reference_gpu_kernels(dtype, layout, tmp_path):
    LX, LY, LZ = 32, 24, 16
    tau, g = 0.8, (2e-5, -4e-6, 3e-6)
    mask = geometry.sphere_pack(LX, LY, LZ, radius=3, porosity=0.55, seed=17)
    f0 = (np.random.default_rng(5).standard_normal((19, LX * LY * LZ)) * 1e-4).astype(dtype)
    steps = 10
    variant = "d3q19_f64" if dtype == np.float64 else "d3q19_f32"
    fr, mvr = run_reference_gpu(variant, mask, f0, (LX, LY, LZ), (16, 2, 2), tau, g, steps,
                                tmp_path)
    lp = lbx.Params(dims=3, LX=LX, LY=LY, LZ=LZ, precision=np.dtype(dtype).itemsize,
                    tau=(tau, 1.0), gaccel=(g[0], g[1], g[2], 0, 0, 0),
                    layout=lbx.LBX_LAYOUT_DENSE if layout == "dense" else lbx.LBX_LAYOUT_COMPACT)
    with lbx.Domain(lp, mask) as d:
        d.upload_f(f0.reshape(1, 19, -1))
        d.run(0, steps, steps)
        d.sync()
        f, mv = d.download_f()[0], d.download_mv()[0]
    tol = 1e-12 if dtype == np.float64 else 1e-5
    fluid = mask != 1
    assert rel_err(f, fr) <= tol
    for c in range(4):
        assert rel_err(mv[c], mvr[c], fluid) <= (tol if dtype == np.float64 else 2e-5), c


def test_gpu_time_reference_kernels_256(tmp_path):
    """The reference's kernels on the benchmark lattice (256^3 sphere pack,
    FP32, tau 0.8, gx 1e-6), over a few of its block shapes; the best is the
    context figure."""
    binary = _binary("d3q19_f32")
    mask = geometry.sphere_pack(256, 256, 256, 6, 0.4, 1234)
    mpath = str(tmp_path / "mask.raw")
    mask.astype(np.uint8).tofile(mpath)
    runs = []
    for block in ((32, 4, 1), (64, 2, 1), (128, 1, 1), (16, 8, 2), (256, 1, 1)):
        out = subprocess.run([binary, "256", "256", "256"] + [str(b) for b in block] +
                             ["0.8", "1e-06", "0", "0", "20", mpath, "-", "-", "time"],
                             check=True, capture_output=True, text=True, timeout=300)
        runs.append(json.loads(out.stdout.strip().splitlines()[-1]))
    best = max(runs, key=lambda r: r["mlups"])
    assert best["mlups"] > 0
    report = os.environ.get("LBX_REFGPU_REPORT")
    if report:
        with open(report, "w") as fh:
            json.dump({"best": best, "runs": runs}, fh, indent=1)


@pytest.mark.parametrize("run_mode", ["steps", "tiled"])
@pytest.mark.parametrize("layout", ["dense", "compact"])
def test_gpu_matches_reference_gpu_kernels_2d(layout, run_mode, tmp_path):
    """D2Q9 FP64 (the 2D case's precision), periodic with a body force,
    discs: the product (per-step launches and the tiled run) against the
    reference's kernels on the GPU."""
    LX, LY = 96, 64
    tau, g = 0.9, (2e-5, -5e-6, 0.0)
    mask = geometry.transpose_2d(geometry.disc_pack(LY, LX, radius=4, porosity=0.6, seed=21),
                                 LY, LX)
    f0 = np.random.default_rng(8).standard_normal((9, LX * LY)) * 1e-4
    steps = 40
    fr, mvr = run_reference_gpu("d2q9_f64", mask, f0, (LX, LY, 1), (32, 4, 1), tau, g, steps,
                                tmp_path)
    lp = lbx.Params(dims=2, LX=LX, LY=LY, LZ=1, precision=8, tau=(tau, 1.0),
                    gaccel=(g[0], g[1], 0, 0, 0, 0),
                    layout=lbx.LBX_LAYOUT_DENSE if layout == "dense" else lbx.LBX_LAYOUT_COMPACT)
    with lbx.Domain(lp, mask) as d:
        d.set_run_mode(run_mode)
        d.upload_f(f0.reshape(1, 9, -1))
        d.run(0, steps, steps)
        d.sync()
        f, mv = d.download_f()[0], d.download_mv()[0]
    fluid = mask != 1
    assert rel_err(f, fr) <= 1e-12
    for c in range(3):
        assert rel_err(mv[c], mvr[c], fluid) <= 1e-12, c


def test_gpu_time_reference_kernels_2d_256(tmp_path):
    """The reference's kernels on the 2D case's lattice (256^2 discs, FP64,
    tau 1.0; periodic with a body force, since the harness runs no face
    rows) over a few block shapes, beside the product on the same lattice
    (its default run mode) over 2000 steps."""
    torch = pytest.importorskip("torch")
    binary = _binary("d2q9_f64")
    from lbx import configs
    lp, mask = configs.cfg1_params(8)
    mpath = str(tmp_path / "mask.raw")
    mask.astype(np.uint8).tofile(mpath)
    runs = []
    for block in ((32, 4, 1), (64, 2, 1), (128, 1, 1), (256, 1, 1), (16, 16, 1)):
        out = subprocess.run([binary, "256", "256", "1"] + [str(b) for b in block] +
                             ["1.0", "1e-06", "0", "0", "2000", mpath, "-", "-", "time"],
                             check=True, capture_output=True, text=True, timeout=300)
        runs.append(json.loads(out.stdout.strip().splitlines()[-1]))
    best = max(runs, key=lambda r: r["mlups"])
    p = lbx.Params(dims=2, LX=256, LY=256, LZ=1, precision=8, tau=(1.0, 1.0),
                   gaccel=(1e-6, 0, 0, 0, 0, 0))
    with lbx.Domain(p, mask) as d:
        s = torch.cuda.Stream()
        d.set_stream(s.cuda_stream)
        d.init_equilibrium(0, 1.0, 0.0, 0.0)
        d.run(0, 40, 0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        d.run(40, 2000, 0)
        e1.record(s)
        s.synchronize()
        product = 256 * 256 * 2000 / (e0.elapsed_time(e1) / 1e3) / 1e6
    assert best["mlups"] > 0 and product > 0
    report = os.environ.get("LBX_REFGPU_REPORT_2D")
    if report:
        with open(report, "w") as fh:
            json.dump({"best": best, "runs": runs, "product_mlups": product}, fh, indent=1)

