"""Python binding of the lbx C ABI (include/lbx.h) over ctypes.

The binding is a thin host-side mirror of the reference's device-facing
calls: construct the device lattice, upload the populations, step at the
reference's odd/even times, download the macro variables.  All compute runs
in the CUDA library ``lib/liblbx.so``; there is no CPU fallback and importing
this module fails if the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field, fields
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "liblbx.so")

LBX_OK, LBX_ERR_INVALID, LBX_ERR_CUDA, LBX_ERR_NOMEM, LBX_ERR_STATE, LBX_ERR_NUMERIC = range(6)
LBX_WRITE_MV = 1
LBX_LAYOUT_AUTO, LBX_LAYOUT_DENSE, LBX_LAYOUT_COMPACT = 0, 1, 2
LBX_RUN_AUTO, LBX_RUN_STEPS, LBX_RUN_TILED = 0, 1, 2

_D2 = C.c_double * 2
_D6 = C.c_double * 6
_I2 = C.c_int * 2


class _CParams(C.Structure):
    _fields_ = [
        ("dims", C.c_int), ("LX", C.c_int), ("LY", C.c_int), ("LZ", C.c_int),
        ("nsubs", C.c_int), ("precision", C.c_int),
        ("accurate", C.c_int), ("compressible", C.c_int),
        ("tau", _D2), ("rho_A", _D2), ("gaccel", _D6), ("sink", C.c_double),
        ("sigma_t_on", C.c_int), ("sigma_t_off", C.c_int),
        ("pressure_n_in", _I2), ("pressure_s_in", _I2),
        ("pressure_n_out", _I2), ("pressure_s_out", _I2),
        ("zeroconcgrad_n", C.c_int), ("zeroconcgrad_s", C.c_int),
        ("rho_in", C.c_double), ("rho_out", C.c_double),
        ("pfadd", C.c_double), ("pfmul", C.c_double),
        ("bc_ramp_start", C.c_int), ("bc_ramp_stop", C.c_int),
        ("pressure_n_table", C.POINTER(C.c_double)), ("pressure_n_len", C.c_int),
        ("pressure_s_table", C.POINTER(C.c_double)), ("pressure_s_len", C.c_int),
        ("device", C.c_int), ("layout", C.c_int),
        ("pressure_t_in", _I2), ("pressure_b_in", _I2),
        ("pressure_t_out", _I2), ("pressure_b_out", _I2),
        ("constcon_t_in", C.c_int), ("constcon_b_in", C.c_int),
        ("zeroconcgrad_t", C.c_int), ("zeroconcgrad_b", C.c_int),
        ("rho_sigma_in", C.c_double),
        ("kahan", C.c_int),
        ("walsh", C.c_int),
        ("velocity_t_in", _I2), ("velocity_t_out", _I2), ("velocity_b_in", _I2),
        ("velocity_b_out", _I2), ("uz_in", C.c_double), ("uz_out", C.c_double),
    ]


class _CObjective(C.Structure):
    _fields_ = [("plane", C.c_int), ("t_first", C.c_int), ("t_last", C.c_int),
                ("w_c", C.c_double), ("w_ux", C.c_double)]


class _CGradient(C.Structure):
    _fields_ = [("J", C.c_double), ("d_gaccel", C.c_double * 3), ("d_tau", C.c_double),
                ("d_tau_s", C.c_double)]


class _CFrameStats(C.Structure):
    _fields_ = [("nodes", C.c_longlong), ("max_rho", C.c_double), ("min_rho", C.c_double),
                ("ave_rho", C.c_double), ("max_u", C.c_double * 3), ("min_u", C.c_double * 3),
                ("ave_u", C.c_double * 3)]

    def as_dict(self) -> dict:
        return dict(nodes=self.nodes, max_rho=self.max_rho, min_rho=self.min_rho,
                    ave_rho=self.ave_rho, max_u=list(self.max_u), min_u=list(self.min_u),
                    ave_u=list(self.ave_u))


class _CFrame(C.Structure):
    _fields_ = [("time", C.c_int), ("nsubs", C.c_int), ("mv", C.c_void_p * 2),
                ("stats", _CFrameStats * 2)]


class _CReductions(C.Structure):
    _fields_ = [
        ("mass", C.c_double), ("solute_mass", C.c_double),
        ("momentum", C.c_double * 3), ("u_sum", C.c_double * 3),
        ("rho_min", C.c_double), ("rho_max", C.c_double),
        ("fluid_nodes", C.c_longlong), ("nonfinite", C.c_int),
    ]


# Every symbol include/lbx.h declares, with its ctypes signature.
_SIGNATURES = {
    "lbx_params_default": (None, [C.POINTER(_CParams)]),
    "lbx_create": (C.c_int, [C.POINTER(_CParams), C.c_void_p, C.POINTER(C.c_void_p)]),
    "lbx_destroy": (C.c_int, [C.c_void_p]),
    "lbx_upload_f": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lbx_download_f": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lbx_upload_mv": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lbx_download_mv": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 4),
    "lbx_init_equilibrium": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 4),
    "lbx_step": (C.c_int, [C.c_void_p, C.c_int, C.c_uint]),
    "lbx_step_pair": (C.c_int, [C.c_void_p, C.c_int, C.c_uint]),
    "lbx_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "lbx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lbx_set_run_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "lbx_sync": (C.c_int, [C.c_void_p]),
    "lbx_reduce": (C.c_int, [C.c_void_p, C.POINTER(_CReductions)]),
    "lbx_frame_stats_compute": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_CFrameStats)]),
    "lbx_pest_set": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "lbx_pest_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int)]),
    "lbx_frame_enqueue": (C.c_int, [C.c_void_p, C.c_int]),
    "lbx_frame_wait": (C.c_int, [C.c_void_p, C.POINTER(_CFrame)]),
    "lbx_reduce_mv_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int,
                                       C.c_int, C.c_int, C.c_void_p,
                                       C.POINTER(_CReductions)]),
    "lbx_device_f": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "lbx_device_mv": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "lbx_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                           C.POINTER(C.c_int)]),
    "lbx_launch_count": (C.c_longlong, [C.c_void_p]),
    "lbx_batch_create": (C.c_int, [C.c_int, C.POINTER(_CParams), C.c_void_p,
                                   C.POINTER(C.c_void_p)]),
    "lbx_batch_destroy": (C.c_int, [C.c_void_p]),
    "lbx_batch_upload_f": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lbx_batch_download_f": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lbx_batch_download_mv": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 4),
    "lbx_batch_init_equilibrium": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 4),
    "lbx_batch_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "lbx_batch_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
    "lbx_batch_set_layout": (C.c_int, [C.c_void_p, C.c_int]),
    "lbx_batch_get_layout": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "lbx_batch_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lbx_batch_sync": (C.c_int, [C.c_void_p]),
    "lbx_batch_reduce": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_CReductions)]),
    "lbx_batch_launch_count": (C.c_longlong, [C.c_void_p]),
    "lbx_btc_start": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "lbx_btc_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.c_int, C.POINTER(C.c_longlong)]),
    "lbx_set_face_profile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "lbx_set_ns": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "lbx_adjoint_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(_CObjective), C.POINTER(C.c_double)]),
    "lbx_adjoint_backward": (C.c_int, [C.c_void_p, C.POINTER(_CGradient),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "lbx_btc_stop": (C.c_int, [C.c_void_p]),
    "lbx_last_error": (C.c_char_p, []),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load liblbx.so and bind every exported symbol; raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            "liblbx.so not found at %s: build it with `make -C lbgpu-prime-dev_b200` "
            "(there is no CPU fallback)" % path)
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class LbxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("lbx error %d: %s" % (code, msg))
        self.code = code


def _check(rc: int):
    if rc != LBX_OK:
        raise LbxError(rc, _lib.lbx_last_error().decode())


@dataclass
class Params:
    """lbx_params; names and meanings follow the reference's params.in."""
    dims: int = 3
    LX: int = 1
    LY: int = 1
    LZ: int = 1
    nsubs: int = 1
    precision: int = 8
    accurate: int = 1
    compressible: int = 0
    tau: Sequence[float] = (1.0, 1.0)
    rho_A: Sequence[float] = (1.0, 1.0)
    gaccel: Sequence[float] = (0.0,) * 6
    sink: float = 0.0
    sigma_t_on: int = 0
    sigma_t_off: int = -1
    pressure_n_in: Sequence[int] = (0, 0)
    pressure_s_in: Sequence[int] = (0, 0)
    pressure_n_out: Sequence[int] = (0, 0)
    pressure_s_out: Sequence[int] = (0, 0)
    zeroconcgrad_n: int = 0
    zeroconcgrad_s: int = 0
    rho_in: float = 1.0
    rho_out: float = 1.0
    pfadd: float = 1.0
    pfmul: float = 0.1
    bc_ramp_start: int = -1
    bc_ramp_stop: int = -1
    pressure_n_table: Optional[np.ndarray] = None
    pressure_s_table: Optional[np.ndarray] = None
    device: int = 0
    layout: int = LBX_LAYOUT_AUTO
    # 3D z faces: top = plane k = LZ-1, bottom = plane k = 0
    pressure_t_in: Sequence[int] = (0, 0)
    pressure_b_in: Sequence[int] = (0, 0)
    pressure_t_out: Sequence[int] = (0, 0)
    pressure_b_out: Sequence[int] = (0, 0)
    constcon_t_in: int = 0
    constcon_b_in: int = 0
    zeroconcgrad_t: int = 0
    zeroconcgrad_b: int = 0
    rho_sigma_in: float = 1.0
    kahan: int = 0
    walsh: int = 0          # partial bounce-back by a per-node fraction (set_ns)
    # Zou-He velocity on the z faces (u_z = uz_in on *_in, uz_out on *_out)
    velocity_t_in: Sequence[int] = (0, 0)
    velocity_t_out: Sequence[int] = (0, 0)
    velocity_b_in: Sequence[int] = (0, 0)
    velocity_b_out: Sequence[int] = (0, 0)
    uz_in: float = 0.0
    uz_out: float = 0.0

    @property
    def Q(self) -> int:
        return 9 if self.dims == 2 else 19

    @property
    def NN(self) -> int:
        return self.LX * self.LY * self.LZ

    @property
    def dtype(self):
        return np.float64 if self.precision == 8 else np.float32

    def _to_c(self, keep: list) -> _CParams:
        st = _CParams()
        for name, _ in _CParams._fields_:
            if name.endswith("_len"):
                continue
            v = getattr(self, name)
            if name.endswith("_table"):
                if v is not None:
                    arr = np.ascontiguousarray(v, dtype=np.float64)
                    keep.append(arr)
                    setattr(st, name, arr.ctypes.data_as(C.POINTER(C.c_double)))
                    setattr(st, name.replace("_table", "_len"), len(arr))
                continue
            if isinstance(v, (tuple, list)):
                fld = getattr(st, name)
                for i, x in enumerate(v):
                    fld[i] = x
            else:
                setattr(st, name, v)
        return st


class Domain:
    """One device lattice (lbx_domain)."""

    def __init__(self, params: Params, solids: np.ndarray):
        load_library()
        self.p = params
        sol = np.ascontiguousarray(solids, dtype=np.uint8).reshape(-1)
        if sol.size != params.NN:
            raise ValueError("solids must hold LX*LY*LZ bytes")
        keep = []
        cp = params._to_c(keep)
        h = C.c_void_p()
        _check(_lib.lbx_create(C.byref(cp), sol.ctypes.data, C.byref(h)))
        self._h = h

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.lbx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- data --------------------------------------------------------------
    def upload_f(self, f: np.ndarray, subs: Optional[int] = None):
        """f: [nsubs, Q, N] (all substances) or [Q, N] with subs given."""
        p = self.p
        f = np.ascontiguousarray(f, dtype=p.dtype)
        if subs is None:
            f = f.reshape(p.nsubs, p.Q, p.NN)
            for s in range(p.nsubs):
                _check(_lib.lbx_upload_f(self._h, s, f[s].ctypes.data))
        else:
            _check(_lib.lbx_upload_f(self._h, subs, f.reshape(p.Q, p.NN).ctypes.data))

    def download_f(self) -> np.ndarray:
        p = self.p
        out = np.empty((p.nsubs, p.Q, p.NN), dtype=p.dtype)
        for s in range(p.nsubs):
            _check(_lib.lbx_download_f(self._h, s, out[s].ctypes.data))
        return out

    def upload_mv(self, mv: np.ndarray):
        p = self.p
        mv = np.ascontiguousarray(mv, dtype=p.dtype).reshape(p.nsubs, 1 + p.dims, p.NN)
        for s in range(p.nsubs):
            _check(_lib.lbx_upload_mv(self._h, s, mv[s].ctypes.data))

    def download_mv(self) -> np.ndarray:
        """[nsubs, 1+D, N]: rho, ux, uy[, uz] per substance."""
        p = self.p
        out = np.empty((p.nsubs, 1 + p.dims, p.NN), dtype=p.dtype)
        for s in range(p.nsubs):
            ptrs = [out[s, c].ctypes.data for c in range(1 + p.dims)]
            if p.dims == 2:
                ptrs.append(None)
            _check(_lib.lbx_download_mv(self._h, s, *ptrs))
        return out

    def frame_stats(self, subs: int) -> dict:
        """lbx_frame_stats_compute: the reference's frame statistics of one
        substance (host mask rule, FP64)."""
        st = _CFrameStats()
        _check(_lib.lbx_frame_stats_compute(self._h, subs, C.byref(st)))
        return st.as_dict()

    def pest_set(self, times, nodes):
        """lbx_pest_set: PEST samples (time-ordered) at dense node indices."""
        t = np.ascontiguousarray(times, dtype=np.int32)
        n = np.ascontiguousarray(nodes, dtype=np.int32)
        assert t.size == n.size
        _check(_lib.lbx_pest_set(self._h, int(t.size), t.ctypes.data, n.ctypes.data))
        self._pest_n = int(t.size)

    def pest_read(self) -> dict:
        """lbx_pest_read: C, u_x, u_y per sample (NaN where not taken)."""
        n = getattr(self, "_pest_n", 0)
        a = [np.zeros(max(n, 1)) for _ in range(3)]
        taken = C.c_int()
        _check(_lib.lbx_pest_read(self._h, *[x.ctypes.data for x in a], C.byref(taken)))
        return dict(conc=a[0][:n], ux=a[1][:n], uy=a[2][:n], taken=taken.value)

    def frame_enqueue(self, time: int):
        _check(_lib.lbx_frame_enqueue(self._h, time))

    def frame_wait(self, copy: bool = True) -> dict:
        """lbx_frame_wait: the oldest queued frame.  Its macro variables are
        copied out of the library's page-locked buffers, or with copy=False
        returned as views of them, valid until the second frame_enqueue after
        this call (the substances' blocks are adjacent in one buffer)."""
        fr = _CFrame()
        _check(_lib.lbx_frame_wait(self._h, C.byref(fr)))
        p = self.p
        n = fr.nsubs * (1 + p.dims) * p.NN
        buf = (C.c_char * (n * np.dtype(p.dtype).itemsize)).from_address(fr.mv[0])
        mv = np.frombuffer(buf, dtype=p.dtype, count=n).reshape(fr.nsubs, 1 + p.dims, p.NN)
        return dict(time=fr.time, mv=mv.copy() if copy else mv,
                    stats=[fr.stats[s].as_dict() for s in range(fr.nsubs)])

    def init_equilibrium(self, subs: int, rho, ux=None, uy=None, uz=None):
        """f = feq of rho, u (scalars or [N] arrays); a velocity component
        left None is zero, filled on the device (only rho is copied)."""
        p = self.p
        arrs = [None if x is None else
                np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=p.dtype), (p.NN,)))
                for x in (rho, ux, uy, uz if p.dims == 3 else None)]
        _check(_lib.lbx_init_equilibrium(self._h, subs, *[
            None if a is None else a.ctypes.data for a in arrs]))

    # -- stepping ----------------------------------------------------------
    def step(self, time: int, write_mv: bool = False):
        _check(_lib.lbx_step(self._h, time, LBX_WRITE_MV if write_mv else 0))

    def step_pair(self, time: int, write_mv: bool = False):
        _check(_lib.lbx_step_pair(self._h, time, LBX_WRITE_MV if write_mv else 0))

    def run(self, t0: int, nsteps: int, frame_rate: int = 0):
        _check(_lib.lbx_run(self._h, t0, nsteps, frame_rate))

    def set_stream(self, stream_handle: Optional[int]):
        """Queue work on a caller's cudaStream_t (an integer handle); 0 or
        None is the CUDA default stream."""
        _check(_lib.lbx_set_stream(self._h, stream_handle))

    RUN_MODES = {"auto": LBX_RUN_AUTO, "steps": LBX_RUN_STEPS, "tiled": LBX_RUN_TILED}

    def set_run_mode(self, mode: str):
        """How run() advances stretches of AA pairs with unchanging launch
        arguments: "auto" (default), "steps" (a launch per step, replayed
        from CUDA graphs) or "tiled" (temporal blocking in shared memory,
        2D one-substance lattices; see lbx_set_run_mode in lbx.h)."""
        if mode not in self.RUN_MODES:
            raise ValueError("run mode must be one of %s" % sorted(self.RUN_MODES))
        _check(_lib.lbx_set_run_mode(self._h, self.RUN_MODES[mode]))

    def sync(self):
        _check(_lib.lbx_sync(self._h))

    def reduce(self) -> dict:
        r = _CReductions()
        rc = _lib.lbx_reduce(self._h, C.byref(r))
        out = dict(mass=r.mass, solute_mass=r.solute_mass,
                   momentum=tuple(r.momentum), u_sum=tuple(r.u_sum),
                   rho_min=r.rho_min, rho_max=r.rho_max,
                   fluid_nodes=r.fluid_nodes, nonfinite=r.nonfinite)
        if rc not in (LBX_OK, LBX_ERR_NUMERIC):
            _check(rc)
        out["status"] = rc
        return out

    # -- introspection -----------------------------------------------------
    def device_f_ptr(self) -> int:
        ptr = C.c_void_p()
        _check(_lib.lbx_device_f(self._h, C.byref(ptr)))
        return ptr.value

    def device_mv_ptr(self) -> int:
        ptr = C.c_void_p()
        _check(_lib.lbx_device_mv(self._h, C.byref(ptr)))
        return ptr.value

    def info(self) -> dict:
        fl = C.c_longlong()
        fused = C.c_int()
        layout = C.c_int()
        _check(_lib.lbx_info(self._h, C.byref(fl), C.byref(fused), C.byref(layout)))
        return dict(fluid_nodes=fl.value, faces_fused=bool(fused.value),
                    layout={LBX_LAYOUT_DENSE: "dense", LBX_LAYOUT_COMPACT: "compact"}[layout.value])

    def launch_count(self) -> int:
        return int(_lib.lbx_launch_count(self._h))

    def btc_start(self, plane: int, capacity: int):
        """Record the means of the solute C and the flow u_x over the fluid
        nodes of `plane` (k in 3D, j in 2D) after every following step."""
        _check(_lib.lbx_btc_start(self._h, plane, capacity))

    def btc_read(self, ux: bool = False):
        """The recorded C means (the breakthrough curve); with ux=True the
        pair (C means, u_x means)."""
        n = C.c_longlong()
        _check(_lib.lbx_btc_read(self._h, None, None, 0, C.byref(n)))
        c = np.empty(max(int(n.value), 0), dtype=np.float64)
        u = np.empty_like(c)
        P = C.POINTER(C.c_double)
        got = C.c_longlong()
        _check(_lib.lbx_btc_read(self._h, c.ctypes.data_as(P), u.ctypes.data_as(P),
                                 c.size, C.byref(got)))
        k = min(c.size, int(got.value))
        return (c[:k], u[:k]) if ux else c[:k]

    def adjoint_forward(self, t0: int, nsteps: int, checkpoint_every: int, plane: int,
                        t_first: int, t_last: int, w_c: float = 1.0, w_ux: float = 0.0) -> float:
        """Run `nsteps` steps storing checkpoints; return the plane
        objective J (see lbx_adjoint_forward)."""
        ob = _CObjective(plane, t_first, t_last, w_c, w_ux)
        J = C.c_double()
        _check(_lib.lbx_adjoint_forward(self._h, t0, nsteps, checkpoint_every, C.byref(ob),
                                        C.byref(J)))
        return J.value

    def adjoint_backward(self, profile_b: bool = False, profile_t: bool = False) -> dict:
        """Gradients of the last adjoint_forward's J."""
        g = _CGradient()
        n = self.p.LX * self.p.LY
        pb = np.zeros(n) if profile_b else None
        pt = np.zeros(n) if profile_t else None
        P = C.POINTER(C.c_double)
        _check(_lib.lbx_adjoint_backward(self._h, C.byref(g),
                                         pb.ctypes.data_as(P) if pb is not None else None,
                                         pt.ctypes.data_as(P) if pt is not None else None))
        out = dict(J=g.J, d_gaccel=tuple(g.d_gaccel), d_tau=g.d_tau, d_tau_s=g.d_tau_s)
        if pb is not None:
            out["d_profile_b"] = pb
        if pt is not None:
            out["d_profile_t"] = pt
        return out

    def set_face_profile(self, top: bool, conc):
        """Per-node concentration (LX*LY, i fastest) of a constant-
        concentration face; None returns to rho_sigma_in."""
        if conc is None:
            _check(_lib.lbx_set_face_profile(self._h, 1 if top else 0, None))
            return
        a = np.ascontiguousarray(conc, dtype=np.float64).reshape(-1)
        if a.size != self.p.LX * self.p.LY:
            raise ValueError("profile must hold LX*LY values")
        _check(_lib.lbx_set_face_profile(self._h, 1 if top else 0,
                                         a.ctypes.data_as(C.POINTER(C.c_double))))

    def set_ns(self, ns):
        """Walsh runs: the per-node fraction ns (N values, dense node order,
        each in [0, 1])."""
        a = np.ascontiguousarray(ns, dtype=np.float64).reshape(-1)
        if a.size != self.p.NN:
            raise ValueError("ns must hold LX*LY*LZ values")
        _check(_lib.lbx_set_ns(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))

    def btc_stop(self):
        _check(_lib.lbx_btc_stop(self._h))


def exported_symbols() -> list:
    return list(_SIGNATURES)
