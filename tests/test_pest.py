"""PEST point sampling (CPU): the host reader and writer and the oracle's
restatement against the reference's own read_PEST_in_files,
write_PEST_out_data and write_PEST_out_file (src/latman.c:899-1232), built
by the harness around the reference's kernels.

The reader keeps what the reference keeps (file order, out-of-lattice
samples dropped, the count rule that drops a last value with no newline);
the three output files are byte-identical when fed the oracle's samples.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from lbx import host


def write_inputs(d, times, xs, ys, trailing_newline=True):
    os.makedirs(os.path.join(d, "in"), exist_ok=True)
    for name, vals in (("timestep", times), ("x_coord", xs), ("y_coord", ys)):
        text = "\n".join(str(v) for v in vals) + ("\n" if trailing_newline else "")
        with open(os.path.join(d, "in", name + "_file.in"), "w") as fh:
            fh.write(text)


CASES = [
    # times, xs, ys, trailing newline
    ([3, 3, 5, 8], [1, 4, 2, 7], [2, 0, 5, 1], True),
    ([3, 3, 5, 8], [1, 4, 2, 7], [2, 0, 5, 1], False),        # last value uncounted
    ([2, 4, 4, 9, 9], [1, 40, 3, 0, -1], [1, 2, 99, 0, 3], True),   # out-of-lattice samples
    ([], [], [], True),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_reader_keeps_what_the_reference_keeps(tmp_path, case):
    if not po.reference_available("d2q9s_pest_f64"):
        pytest.skip("reference harness not built")
    times, xs, ys, nl = CASES[case]
    d = str(tmp_path)
    write_inputs(d, times, xs, ys, nl)
    LX, LY = 8, 6
    ref = po.reference_pest_inputs("d2q9s_pest_f64", LX, LY, 1, d)
    order, time, node = host.read_pest(os.path.join(d, "in"), LX, LY)
    assert np.array_equal(order, ref[0]) and np.array_equal(time, ref[1])
    assert np.array_equal(node, ref[3] * LX + ref[2])


def test_reader_errors(tmp_path):
    d = str(tmp_path)
    assert host.pest_count(os.path.join(d, "in")) == -1
    write_inputs(d, [4, 2], [0, 0], [0, 0])
    with pytest.raises(host.HostError):
        host.read_pest(os.path.join(d, "in"), 4, 4)
    write_inputs(d, [1, 2, 3], [0, 0], [0, 0, 0])
    with pytest.raises(host.HostError):
        host.read_pest(os.path.join(d, "in"), 4, 4)


@pytest.mark.parametrize("variant,dims,dtype", [("d2q9s_pest_f64", 2, np.float64),
                                                ("d3q19s_pest_f32", 3, np.float32)])
def test_samples_and_files_match_reference(tmp_path, variant, dims, dtype):
    if not po.reference_available(variant):
        pytest.skip("reference harness not built")
    LX, LY, LZ = (10, 8, 1) if dims == 2 else (8, 7, 6)
    p = po.Params(dims=dims, LX=LX, LY=LY, LZ=LZ, nsubs=2, tau=(0.9, 0.8), sink=1e-3,
                  sigma_t_on=2, sigma_t_off=30, gaccel=(1e-4, 3e-5, 0, 0, 0, 0))
    rng = np.random.default_rng(9)
    Q = p.Q
    f = rng.standard_normal((2, Q, p.NN)) * 1e-3
    f[1] = np.abs(f[1]) + 0.1
    f = f.astype(dtype)
    sol = (rng.random(p.NN) < 0.15).astype(np.uint8)
    times = [1, 2, 2, 5, 8, 8, 8, 13, 40]          # 40: beyond the run, never taken
    xs = [1, 3, 3, 9, 0, 5, 2, 4, 1]
    ys = [2, 0, 5, 1, 6, 3, 3, 6, 0]
    ref_dir, our_dir = str(tmp_path / "ref"), str(tmp_path / "ours")
    for d in (ref_dir, our_dir):
        write_inputs(d, times, [min(x, LX - 1) for x in xs], [min(y, LY - 1) for y in ys])
    steps = 20
    po.reference_pest(variant, p, f.copy(), sol, 0, steps, ref_dir)
    order, time, node = host.read_pest(os.path.join(our_dir, "in"), LX, LY)
    _, _, c, ux, uy, taken = po.pest_samples(p, f.copy(), sol, 0, steps, time, node)
    assert taken == 8
    os.makedirs(os.path.join(our_dir, "out"))
    host.write_pest(os.path.join(our_dir, "out"), c, ux, uy, order, np.dtype(dtype).itemsize)
    for name in ("conc_data", "vel_data", "conc_order"):
        a = open(os.path.join(ref_dir, "out", name + "_proc0000.dat")).read()
        b = open(os.path.join(our_dir, "out", name + "_proc0000.dat")).read()
        if name == "conc_order":
            assert a == b
            continue
        # the untaken sample: the reference prints its never-written field
        la, lb = a.split("\n"), b.split("\n")
        assert la[:taken] == lb[:taken], name
        assert len(la) == len(lb)
