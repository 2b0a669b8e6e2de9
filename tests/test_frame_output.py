"""The per-frame files of the reference's output_frame (CPU).

lbh_write_frame (the host library) against the reference's own
output_frame, compute_* and writers (src/lbio.c, src/compute.c) built by
the harness, on the same macro variables and mask: the .dat, .txt and .raw
files byte for byte, the cuda_frames summary line for line (header exact;
FP64 values to the printed 7 decimals; FP32 means and the max/mean ratios
within the reference's float running-sum error, since the library sums in
FP64).
"""
import glob
import os

import numpy as np
import pytest

import pyoracle as po
from lbx import host

CASES = [("d2q9_f64", 2, 1, 8), ("d3q19_f64", 3, 1, 8), ("d3q19_f32", 3, 1, 4),
         ("d3q19s_f64", 3, 2, 8)]


def make_mv(rng, dims, nsubs, N, dtype):
    mv = rng.standard_normal((nsubs, 1 + dims, N)) * 1e-3
    mv[:, 0] += 1.0
    mv[:, 1:, 5] = 0.0                       # |u| = 0 somewhere
    return mv.astype(dtype)


def files(d):
    return sorted(os.path.basename(p) for p in glob.glob(os.path.join(d, "out", "*")))


def summary_rows(path):
    with open(path) as fh:
        lines = fh.read().split("\n")
    return lines[:3], [ln.split() for ln in lines[3:] if ln.strip()]


@pytest.mark.parametrize("variant,dims,nsubs,rs", CASES)
def test_frame_files_match_reference(tmp_path, variant, dims, nsubs, rs):
    if not po.reference_available(variant):
        pytest.skip("reference harness not built")
    LX, LY, LZ = (7, 5, 1) if dims == 2 else (6, 5, 4)
    N = LX * LY * LZ
    rng = np.random.default_rng(77)
    dtype = np.float32 if rs == 4 else np.float64
    sol = rng.choice([0, 1, 255], size=N, p=[0.7, 0.2, 0.1]).astype(np.uint8)
    ref, ours = str(tmp_path / "ref"), str(tmp_path / "ours")
    os.makedirs(os.path.join(ours, "out"))
    for time, frame in ((0, 0), (10, 1), (20, 2)):
        mv = make_mv(rng, dims, nsubs, N, dtype)
        if frame == 2:
            mv[:, 2] = 3e-4                  # constant u_y: a_max == a_min in the images
        assert po.reference_output_frame(variant, LX, LY, LZ, mv, sol, time, frame, 10, ref)
        stats = [po.frame_stats(mv[s], sol, dims) for s in range(nsubs)]
        host.write_frame(os.path.join(ours, "out"), dims, LX, LY, LZ, time, frame, mv, stats,
                         sol)
    assert files(ref) == files(ours)
    for name in files(ref):
        a = open(os.path.join(ref, "out", name), "rb").read()
        b = open(os.path.join(ours, "out", name), "rb").read()
        if "_frames" not in name:
            assert a == b, name
            continue
        ha, ra = summary_rows(os.path.join(ref, "out", name))
        hb, rb = summary_rows(os.path.join(ours, "out", name))
        assert ha == hb
        assert len(ra) == len(rb) == 3
        for x, y in zip(ra, rb):
            assert len(x) == len(y) == 21, (x, y)
            for k, (u, v) in enumerate(zip(x, y)):
                if u == v:
                    continue
                # FP32 means (and the ratios built on them) may differ in the
                # last printed digit
                assert rs == 4 and k in (11, 12, 13, 14, 15, 16, 19, 20), (name, k, u, v)
                # the reference's float running sum over ~100 nodes is within
                # ~100 float ulps of the exact mean
                tol = 1e-5 * abs(float(u)) if k in (14, 15, 16, 20) else \
                    1e-6 * max(1.0, abs(float(u)))
                assert abs(float(u) - float(v)) <= tol, (k, u, v)


def test_txt_rows_planes_and_parallel_formatting(tmp_path):
    """The text dump's layout at a size that spreads over every host core."""
    LX, LY, LZ = 33, 17, 9
    a = np.random.default_rng(3).standard_normal(LX * LY * LZ)
    a[4] = -0.0
    p = str(tmp_path / "t.txt")
    mv = np.stack([a, a, a, a])[None]
    st = po.frame_stats(mv[0], np.zeros(a.size, np.uint8), 3)
    host.write_frame(str(tmp_path), 3, LX, LY, LZ, 0, 0, mv, [st], np.zeros(a.size, np.uint8),
                     host.FRAME_TXT)
    got = open(glob.glob(str(tmp_path / "cuda_rho*.txt"))[0]).read()
    want = []
    n = 0
    for k in range(LZ):
        for j in range(LY):
            want.append("".join(" %18.16f" % a[n + i] for i in range(LX)) + "\n")
            n += LX
        want.append("\n")
    assert got == "".join(want)
