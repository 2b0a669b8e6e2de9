"""ctypes binding of the host C library lib/liblbh.so (host/lbh.h).

The reference's file interface: the positional params.in reader, the 24-bit
BMP and raw solid-mask decoders/writers, the initial density field and the
frame file names.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "liblbh.so")


class Real(C.Structure):
    _fields_ = [("d", C.c_double), ("f", C.c_float)]


def _ints(n):
    return C.c_int * n


class HostParams(C.Structure):
    """Mirror of lbh_params (host/lbh.h), field for field."""
    _fields_ = [
        ("LX", C.c_int), ("LY", C.c_int), ("LZ", C.c_int), ("BX", C.c_int), ("BY", C.c_int),
        ("BZ", C.c_int), ("length_scale", C.c_int), ("NumFrames", C.c_int),
        ("FrameRate", C.c_int),
        ("tau", Real * 2), ("gforce", (Real * 3) * 2), ("end_grav", _ints(2)),
        ("buoyancy", C.c_int), ("incompressible", C.c_int), ("simple_diffusion", C.c_int),
        ("rho_A", Real * 2), ("rho_B", Real * 2),
        ("rho_sigma", Real), ("rho_sigma_in", Real), ("rho_sigma_out", Real),
        ("u_sigma", Real), ("u_sigma_in", Real), ("u_sigma_out", Real),
        ("sigma_t_on", C.c_int), ("sigma_t_off", C.c_int), ("sigma_start", C.c_int),
        ("sigma_stop", C.c_int), ("sigma_btc_rate", C.c_int), ("sigma_btc_spot", C.c_int),
        ("GZL", C.c_int), ("PressureBC", C.c_int), ("AllBoundaryPeriodic", C.c_int),
        ("sink", Real), ("pfmul", Real), ("pfadd", Real), ("rho_in", Real), ("rho_out", Real),
        ("ux_in", Real), ("ux_out", Real), ("uy_in", Real), ("uy_out", Real),
        ("uz_in", Real), ("uz_out", Real), ("big_V0", Real), ("big_V0_solid", Real * 2),
        ("ns_flag", C.c_int), ("ns", Real),
        ("ic_poisseuille", C.c_int), ("bc_poisseuille", C.c_int),
        ("bc_slip_north", C.c_int), ("bc_sigma_slip", C.c_int),
        ("bc_ramp_start", C.c_int), ("bc_ramp_stop", C.c_int),
    ] + [(n, _ints(2)) for n in (
        "pressure_t_in", "pressure_b_in", "pressure_t_out", "pressure_b_out",
        "velocity_t_in", "velocity_b_in", "velocity_t_out", "velocity_b_out",
        "pressure_n_in", "pressure_s_in", "pressure_n_out", "pressure_s_out",
        "velocity_n_in", "velocity_s_in", "velocity_n_out", "velocity_s_out",
        "pressure_e_in", "pressure_w_in", "pressure_e_out", "pressure_w_out",
        "velocity_e_in", "velocity_w_in", "velocity_e_out", "velocity_w_out")] + [
        ("constcon", _ints(24)),
        ("zeroconcgrad_t", C.c_int), ("zeroconcgrad_b", C.c_int),
        ("zeroconcgrad_n", C.c_int), ("zeroconcgrad_s", C.c_int),
        ("zeroconcgrad_e", C.c_int), ("zeroconcgrad_w", C.c_int),
        ("zeroconcgrad_full", C.c_int),
        ("plot_scale_dynamic", C.c_int), ("use_colormap", C.c_int),
        ("initial_condition", C.c_int),
        ("x0", C.c_int), ("y0", C.c_int), ("z0", C.c_int), ("r0", C.c_int), ("cut", Real),
        ("x1", C.c_int), ("x2", C.c_int), ("y1", C.c_int), ("y2", C.c_int),
        ("z1", C.c_int), ("z2", C.c_int),
        ("rel_x1", Real), ("rel_x2", Real), ("rel_y1", Real), ("rel_y2", Real),
        ("rel_z1", Real), ("rel_z2", Real),
        ("dump_rho", C.c_int), ("dump_u", C.c_int), ("dump_force", C.c_int),
        ("dump_vor", C.c_int),
        ("NumNodes", C.c_longlong), ("NumTimeSteps", C.c_int),
    ]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("liblbh.so missing: make -C lbgpu-prime-dev_b200")
        lib = C.CDLL(LIB_PATH)
        lib.lbh_read_params.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(HostParams),
                                        C.c_char_p, C.c_int]
        lib.lbh_read_bmp_mask.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                          C.c_char_p, C.c_int]
        lib.lbh_read_raw_mask.argtypes = [C.c_char_p, C.c_longlong, C.c_void_p,
                                          C.c_char_p, C.c_int]
        lib.lbh_write_bmp_mask.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p]
        lib.lbh_write_raw_mask.argtypes = [C.c_char_p, C.c_longlong, C.c_void_p]
        lib.lbh_initial_rho.argtypes = [C.POINTER(HostParams), C.c_int, C.c_int, C.c_int,
                                        C.c_void_p]
        lib.lbh_apply_solid_rule.argtypes = [C.c_void_p, C.c_longlong, C.c_int]
        lib.lbh_apply_solid_rule.restype = C.c_longlong
        lib.lbh_write_frame.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(C.c_void_p), C.POINTER(FrameStats),
                                        C.c_void_p, C.c_uint]
        lib.lbh_pest_count.argtypes = [C.c_char_p]
        lib.lbh_read_pest.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]
        lib.lbh_write_pest.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_int]
        lib.lbh_walsh_ns.argtypes = [C.c_double, C.c_int, C.c_void_p, C.c_longlong,
                                     C.c_char_p, C.c_void_p, C.c_char_p, C.c_int]
        _lib = lib
    return _lib


class FrameStats(C.Structure):
    """Mirror of lbh_frame_stats (and of the ABI's lbx_frame_stats)."""
    _fields_ = [("nodes", C.c_longlong), ("max_rho", C.c_double), ("min_rho", C.c_double),
                ("ave_rho", C.c_double), ("max_u", C.c_double * 3), ("min_u", C.c_double * 3),
                ("ave_u", C.c_double * 3)]

    @classmethod
    def from_dict(cls, d):
        st = cls()
        st.nodes = d["nodes"]
        st.max_rho, st.min_rho, st.ave_rho = d["max_rho"], d["min_rho"], d["ave_rho"]
        for c in range(3):
            st.max_u[c], st.min_u[c], st.ave_u[c] = d["max_u"][c], d["min_u"][c], d["ave_u"][c]
        return st


FRAME_SUMMARY, FRAME_RAW, FRAME_DAT, FRAME_TXT, FRAME_ALL = 1, 2, 4, 8, 15


class HostError(RuntimeError):
    pass


def read_params(path: str, dims: int = 2, nsubs: int = 1) -> HostParams:
    p = HostParams()
    err = C.create_string_buffer(512)
    if load().lbh_read_params(path.encode(), dims, nsubs, C.byref(p), err, 512):
        raise HostError(err.value.decode())
    return p


def read_bmp_mask(path: str, LX: int, LY: int) -> np.ndarray:
    out = np.zeros(LX * LY, np.uint8)
    err = C.create_string_buffer(512)
    if load().lbh_read_bmp_mask(path.encode(), LX, LY, out.ctypes.data, err, 512):
        raise HostError(err.value.decode())
    return out


def read_raw_mask(path: str, N: int) -> np.ndarray:
    out = np.zeros(N, np.uint8)
    err = C.create_string_buffer(512)
    if load().lbh_read_raw_mask(path.encode(), N, out.ctypes.data, err, 512):
        raise HostError(err.value.decode())
    return out


SOLID_DEVICE, SOLID_NONZERO = 0, 1


def apply_solid_rule(mask: np.ndarray, rule: int) -> int:
    """lbh_apply_solid_rule in place on a uint8 mask; returns how many bytes
    are neither 0 nor 1."""
    assert mask.dtype == np.uint8 and mask.flags.c_contiguous
    return int(load().lbh_apply_solid_rule(mask.ctypes.data, mask.size, rule))


NS_MASK, NS_FILE = 0, 1


def walsh_ns(ns_value: float, source: int, mask: np.ndarray = None, N: int = None,
             path: str = "") -> np.ndarray:
    """lbh_walsh_ns: the Walsh fraction field from the mask (ns_value where
    the byte is 1, else 0) or from an N-byte file (byte / 255)."""
    if mask is not None:
        mask = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        N = mask.size
    out = np.zeros(N, np.float64)
    err = C.create_string_buffer(512)
    if load().lbh_walsh_ns(ns_value, source, mask.ctypes.data if mask is not None else None,
                           N, path.encode(), out.ctypes.data, err, 512):
        raise HostError(err.value.decode())
    return out


def write_frame(outdir: str, dims: int, LX: int, LY: int, LZ: int, time: int, frame: int,
                mv: np.ndarray, stats, mask: np.ndarray, flags: int = FRAME_ALL):
    """lbh_write_frame: every per-frame file of the reference for the macro
    variables mv ([nsubs][1+D][N], float32 or float64) with their statistics
    (FrameStats or dicts, one per substance)."""
    mv = np.ascontiguousarray(mv)
    nsubs = mv.shape[0]
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    ptrs = (C.c_void_p * nsubs)(*[mv[s].ctypes.data for s in range(nsubs)])
    st = (FrameStats * nsubs)(*[x if isinstance(x, FrameStats) else FrameStats.from_dict(x)
                                for x in stats])
    if load().lbh_write_frame(outdir.encode(), dims, nsubs, LX, LY, LZ, time, frame,
                              mv.dtype.itemsize, ptrs, st, m.ctypes.data, flags):
        raise HostError("cannot write the frame files in " + outdir)


def pest_count(dir_: str) -> int:
    """lbh_pest_count: samples in dir/timestep_file.in (-1: none)."""
    return int(load().lbh_pest_count(dir_.encode()))


def read_pest(dir_: str, LX: int, LY: int):
    """lbh_read_pest: (order, time, node) of the kept samples."""
    n = pest_count(dir_)
    if n < 0:
        raise HostError("no PEST sample times in " + dir_)
    a = [np.zeros(max(n, 1), np.int32) for _ in range(3)]
    err = C.create_string_buffer(512)
    kept = load().lbh_read_pest(dir_.encode(), LX, LY, n, a[0].ctypes.data, a[1].ctypes.data,
                                a[2].ctypes.data, err, 512)
    if kept < 0:
        raise HostError(err.value.decode())
    return tuple(x[:kept] for x in a)


def write_pest(outdir: str, conc, ux, uy, order, real_size: int):
    """lbh_write_pest: the three PEST output files."""
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (conc, ux, uy)]
    o = np.ascontiguousarray(order, dtype=np.int32)
    if load().lbh_write_pest(outdir.encode(), len(o), *[x.ctypes.data for x in arrs],
                             o.ctypes.data, real_size):
        raise HostError("cannot write the PEST files in " + outdir)


def write_bmp_mask(path: str, LX: int, LY: int, mask: np.ndarray):
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    if load().lbh_write_bmp_mask(path.encode(), LX, LY, m.ctypes.data):
        raise HostError("cannot write " + path)


def write_raw_mask(path: str, mask: np.ndarray):
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    if load().lbh_write_raw_mask(path.encode(), m.size, m.ctypes.data):
        raise HostError("cannot write " + path)


def initial_rho(p: HostParams, dims: int, nsubs: int, subs: int) -> np.ndarray:
    out = np.zeros(p.NumNodes, np.float64)
    if load().lbh_initial_rho(C.byref(p), dims, nsubs, subs, out.ctypes.data):
        raise HostError("initial_condition %d is not supported" % p.initial_condition)
    return out


def params_layout():
    """[(name, is_real)] of params.in fields in file order (src/params.h:40-660)."""
    lib = load()
    lib.lbh_params_field.restype = C.c_char_p
    lib.lbh_params_field.argtypes = [C.c_int, C.POINTER(C.c_int)]
    out = []
    for k in range(lib.lbh_params_field_count()):
        r = C.c_int()
        out.append((lib.lbh_params_field(k, C.byref(r)).decode(), bool(r.value)))
    return out
