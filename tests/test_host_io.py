"""The host C library's file interface against the reference (CPU only).

Node classification must be bit-exact: the BMP decoder (black -> 1, rows as
stored), the raw decoder (bytes verbatim) and the device rule (solid iff the
byte is 1).  The positional params.in reader must put every value in the
field the reference's read_params puts it.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from lbx import host
from _host_files import write_params

REF_IN = os.path.join(po.reference_root(), "in")


VALUES = {
    "LX": 37, "LY": 21, "LZ": 5, "BX": 1, "BY": 1, "BZ": 1, "NumFrames": 4,
    "FrameRate": 30, "tau[0]": 0.85, "gforce[0][0]": 2.5e-6, "tau[1]": 0.7,
    "rho_A[0]": 1.0, "rho_B[0]": 0.75, "sigma_t_on": 3, "sigma_t_off": -1,
    "sink": 1e-5, "pfmul": 0.25, "pfadd": 1.0, "rho_in": 1.0012, "rho_out": 0.9991,
    "bc_ramp_start": 10, "bc_ramp_stop": 200, "pressure_n_in[0]": 2,
    "pressure_s_in[0]": 1, "zeroconcgrad_n": 1, "initial_condition": 2,
    "x0": -1, "r0": -1, "x1": 4, "x2": 9, "y1": -1, "y2": -1, "z1": 0, "z2": 3,
    "rel_y1": 0.25, "rel_y2": -1.0, "cut": -1.0,
}


def test_params_reader_derived_values(tmp_path):
    path = str(tmp_path / "params.in")
    write_params(path, VALUES)
    p = host.read_params(path, dims=3, nsubs=2)
    assert (p.LX, p.LY, p.LZ, p.NumFrames, p.FrameRate) == (37, 21, 5, 4, 30)
    assert p.NumNodes == 37 * 21 * 5 and p.NumTimeSteps == 120
    assert p.tau[0].d == 0.85 and p.tau[0].f == np.float32(0.85)
    assert p.gforce[0][0].d == 2.5e-6 and p.tau[1].d == 0.7
    assert p.sigma_t_off == 120                 # < 0 -> NumTimeSteps
    assert p.rho_A[1].d == 0.75                 # rho_A[1] = rho_B[0]
    assert p.x0 == 37 // 2 and p.r0 == 5        # defaults from the extents
    assert p.y1 == round(0.25 * 21) and p.y2 == 21 // 2
    assert p.cut.d == 0.3
    assert p.pressure_n_in[0] == 2 and p.pressure_s_in[0] == 1 and p.zeroconcgrad_n == 1


def test_params_reader_matches_reference_reader(tmp_path):
    path = str(tmp_path / "params.in")
    write_params(path, VALUES)
    ref = po.reference_read_params(path)
    if ref is None:
        pytest.skip("reference harness not built")
    p = host.read_params(path, dims=2, nsubs=1)
    mine = {"LX": p.LX, "LY": p.LY, "LZ": 1, "NumFrames": p.NumFrames,
            "FrameRate": p.FrameRate, "initial_condition": p.initial_condition,
            "bc_ramp_start": p.bc_ramp_start, "bc_ramp_stop": p.bc_ramp_stop,
            "pressure_n_in[0]": p.pressure_n_in[0], "pressure_s_in[0]": p.pressure_s_in[0],
            "tau[0]": p.tau[0].d, "rho_A[0]": p.rho_A[0].d, "rho_B[0]": p.rho_B[0].d,
            "rho_in": p.rho_in.d, "rho_out": p.rho_out.d, "sink": p.sink.d,
            "gforce[0][0]": p.gforce[0][0].d, "pfmul": p.pfmul.d}
    assert mine == ref


@pytest.mark.skipif(not os.path.isdir(REF_IN), reason="reference inputs absent")
def test_params_reader_reads_the_reference_input():
    p = host.read_params(os.path.join(REF_IN, "params.in"), dims=2, nsubs=1)
    ref = po.reference_read_params(os.path.join(REF_IN, "params.in"))
    assert p.LX > 0 and p.NumTimeSteps == p.NumFrames * p.FrameRate
    if ref is not None:
        assert (p.LX, p.LY, p.FrameRate, p.bc_ramp_stop) == \
            (ref["LX"], ref["LY"], ref["FrameRate"], ref["bc_ramp_stop"])
        assert p.tau[0].d == ref["tau[0]"] and p.rho_in.d == ref["rho_in"]


def test_params_reader_rejects_short_file(tmp_path):
    path = str(tmp_path / "params.in")
    with open(path, "w") as fh:
        fh.write("LX 10\nLY 10\n")
    with pytest.raises(host.HostError, match="ends before"):
        host.read_params(path)


@pytest.mark.parametrize("shape", [(9, 9), (13, 7), (64, 40), (3, 3)])
def test_bmp_decode_bit_exact(tmp_path, shape):
    LX, LY = shape
    rng = np.random.default_rng(LX * 100 + LY)
    mask = (rng.random(LX * LY) < 0.4).astype(np.uint8)
    path = str(tmp_path / ("%dx%d.bmp" % (LX, LY)))
    host.write_bmp_mask(path, LX, LY, mask)
    assert np.array_equal(host.read_bmp_mask(path, LX, LY), mask)
    ref = po.reference_read_bmp(path, LX, LY)
    if ref is not None:
        assert np.array_equal(ref, mask)


def test_bmp_non_black_colours_are_fluid(tmp_path):
    """Only (0,0,0) is solid; a dark grey pixel is fluid."""
    LX, LY = 5, 4
    path = str(tmp_path / "5x4.bmp")
    host.write_bmp_mask(path, LX, LY, np.zeros(20, np.uint8))
    raw = bytearray(open(path, "rb").read())
    row = (3 * LX + 3) // 4 * 4
    raw[54 + 0] = raw[54 + 1] = raw[54 + 2] = 0          # (0,0) black
    raw[54 + row + 3] = 1                                   # (1,1) near-black
    raw[54 + row + 4] = raw[54 + row + 5] = 0
    open(path, "wb").write(bytes(raw))
    m = host.read_bmp_mask(path, LX, LY)
    assert m[0] == 1 and m[LX + 1] == 0 and m.sum() == 1
    ref = po.reference_read_bmp(path, LX, LY)
    if ref is not None:
        assert np.array_equal(ref, m)


def test_bmp_rejects_wrong_size_and_depth(tmp_path):
    path = str(tmp_path / "m.bmp")
    host.write_bmp_mask(path, 6, 6, np.zeros(36, np.uint8))
    with pytest.raises(host.HostError, match="size"):
        host.read_bmp_mask(path, 7, 6)
    raw = bytearray(open(path, "rb").read())
    raw[28] = 8
    open(path, "wb").write(bytes(raw))
    with pytest.raises(host.HostError, match="24-bit"):
        host.read_bmp_mask(path, 6, 6)


def test_raw_decode_verbatim(tmp_path):
    rng = np.random.default_rng(4)
    mask = rng.choice([0, 1, 255, 7], size=6 * 5 * 4).astype(np.uint8)
    path = str(tmp_path / "6x5x4.raw")
    host.write_raw_mask(path, mask)
    assert np.array_equal(host.read_raw_mask(path, mask.size), mask)
    ref = po.reference_read_raw(path, 6, 5, 4)
    if ref is not None:
        assert np.array_equal(ref, mask)
    with pytest.raises(host.HostError, match="fewer"):
        host.read_raw_mask(path, mask.size + 1)


@pytest.mark.skipif(not os.path.isdir(REF_IN), reason="reference inputs absent")
@pytest.mark.parametrize("name,shape", [("3x3.bmp", (3, 3)), ("9x9.bmp", (9, 9)),
                                        ("3x3x3.raw", (3, 3, 3)), ("9x9x9.raw", (9, 9, 9))])
def test_reference_fixtures_decode_identically(name, shape):
    """The reference's own tiny mask fixtures, through both decoders."""
    path = os.path.join(REF_IN, name)
    if name.endswith(".bmp"):
        mine = host.read_bmp_mask(path, *shape)
        ref = po.reference_read_bmp(path, *shape)
    else:
        mine = host.read_raw_mask(path, int(np.prod(shape)))
        ref = po.reference_read_raw(path, *shape)
    if ref is None:
        pytest.skip("reference harness not built")
    assert np.array_equal(mine, ref)
    if name == "9x9x9.raw":
        # its solids are stored as 255: the device rule (== 1) makes them fluid
        assert (mine == 255).any() and not (mine == 1).any()


def test_initial_density_cube_and_uniform(tmp_path):
    path = str(tmp_path / "params.in")
    write_params(path, dict(VALUES, LX=10, LY=8, LZ=1, x1=2, x2=4, y1=1, y2=3))
    p = host.read_params(path, dims=2, nsubs=1)
    rho = host.initial_rho(p, 2, 1, 0).reshape(8, 10)
    assert (rho[1:4, 2:5] == 0.75).all() and rho[0, 0] == 1.0
    p.initial_condition = 0
    assert (host.initial_rho(p, 2, 1, 0) == 1.0).all()
    p.initial_condition = 7
    with pytest.raises(host.HostError):
        host.initial_rho(p, 2, 1, 0)


def test_solid_rule_device_keeps_bytes_nonzero_maps_to_one():
    from lbx import host
    m = np.array([0, 1, 255, 2, 0, 1], np.uint8)
    d = m.copy()
    assert host.apply_solid_rule(d, host.SOLID_DEVICE) == 2
    assert np.array_equal(d, m)
    z = m.copy()
    assert host.apply_solid_rule(z, host.SOLID_NONZERO) == 2
    assert np.array_equal(z, [0, 1, 1, 1, 0, 1])
    assert host.apply_solid_rule(z, host.SOLID_DEVICE) == 0


def test_walsh_ns_from_mask_and_file(tmp_path):
    """The mask rule of process_ns (ns where the byte is 1, 0 elsewhere, so
    255 bytes stay 0 as the device rule reads them) and the byte / 255 rule
    of read_ns; ns outside [0, 1] and a short file are errors."""
    m = np.array([0, 1, 255, 1, 0, 2], np.uint8)
    assert np.array_equal(host.walsh_ns(0.3, host.NS_MASK, mask=m), [0, 0.3, 0, 0.3, 0, 0])
    with pytest.raises(host.HostError):
        host.walsh_ns(1.5, host.NS_MASK, mask=m)
    raw = np.array([0, 255, 51, 128, 7], np.uint8)
    path = str(tmp_path / "ns5x1x1.raw")
    raw.tofile(path)
    assert np.array_equal(host.walsh_ns(0.0, host.NS_FILE, N=5, path=path), raw / 255.0)
    with pytest.raises(host.HostError):
        host.walsh_ns(0.0, host.NS_FILE, N=6, path=path)
