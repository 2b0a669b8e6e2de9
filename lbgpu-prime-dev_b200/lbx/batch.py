"""Binding of the batch API (lbx_batch_* in include/lbx.h): many independent
lattices of uneven size stepped together on one GPU."""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import (LbxError, Params, _CParams, _CReductions, _check, load_library)

LBX_BATCH_AUTO, LBX_BATCH_FUSED, LBX_BATCH_PERSISTENT, LBX_BATCH_SEQUENTIAL = 0, 1, 2, 3
MODES = {"auto": LBX_BATCH_AUTO, "fused": LBX_BATCH_FUSED,
         "persistent": LBX_BATCH_PERSISTENT, "sequential": LBX_BATCH_SEQUENTIAL}
LAYOUTS = {"largest_first": 0, "interleaved": 1, "given": 2}


class Batch:
    """lbx_batch: samples with their own extents, masks, tau and force."""

    def __init__(self, params: Sequence[Params], masks: Sequence[np.ndarray]):
        lib = load_library()
        self._lib = lib
        self.params = list(params)
        keep = []
        arr = (_CParams * len(params))()
        for i, p in enumerate(params):
            arr[i] = p._to_c(keep)
        self._masks = [np.ascontiguousarray(m, dtype=np.uint8).reshape(-1) for m in masks]
        for p, m in zip(params, self._masks):
            if m.size != p.NN:
                raise ValueError("mask size does not match LX*LY*LZ")
        ptrs = (C.c_void_p * len(masks))(*[m.ctypes.data for m in self._masks])
        h = C.c_void_p()
        _check(lib.lbx_batch_create(len(params), arr, ptrs, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lbx_batch_destroy(self._h)
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

    def upload_f(self, sample: int, f: np.ndarray):
        p = self.params[sample]
        f = np.ascontiguousarray(f, dtype=p.dtype).reshape(p.Q, p.NN)
        _check(self._lib.lbx_batch_upload_f(self._h, sample, f.ctypes.data))

    def download_f(self, sample: int) -> np.ndarray:
        p = self.params[sample]
        out = np.empty((p.Q, p.NN), dtype=p.dtype)
        _check(self._lib.lbx_batch_download_f(self._h, sample, out.ctypes.data))
        return out

    def download_mv(self, sample: int) -> np.ndarray:
        p = self.params[sample]
        out = np.empty((1 + p.dims, p.NN), dtype=p.dtype)
        ptrs = [out[c].ctypes.data for c in range(1 + p.dims)] + ([None] if p.dims == 2 else [])
        _check(self._lib.lbx_batch_download_mv(self._h, sample, *ptrs))
        return out

    def init_equilibrium(self, sample: int, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        p = self.params[sample]
        a = [np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=p.dtype), (p.NN,)))
             for x in (rho, ux, uy, uz)]
        _check(self._lib.lbx_batch_init_equilibrium(
            self._h, sample, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data,
            a[3].ctypes.data if p.dims == 3 else None))

    def run(self, t0: int, nsteps: int, frame_rate: int = 0, mode: str = "auto"):
        _check(self._lib.lbx_batch_run(self._h, t0, nsteps, frame_rate, MODES[mode]))

    def autotune(self, steps: int = 6):
        m, b = C.c_int(), C.c_int()
        _check(self._lib.lbx_batch_autotune(self._h, steps, C.byref(m), C.byref(b)))
        return {v: k for k, v in MODES.items()}[m.value], b.value

    def set_layout(self, layout: str):
        """Sample order of the compact population array: "largest_first"
        (default), "interleaved" or "given"; the state is kept."""
        if layout not in LAYOUTS:
            raise ValueError("layout must be one of %s" % sorted(LAYOUTS))
        _check(self._lib.lbx_batch_set_layout(self._h, LAYOUTS[layout]))

    def layout(self) -> str:
        v = C.c_int()
        _check(self._lib.lbx_batch_get_layout(self._h, C.byref(v)))
        return {k: x for x, k in LAYOUTS.items()}[v.value]

    def set_stream(self, handle):
        _check(self._lib.lbx_batch_set_stream(self._h, handle))

    def sync(self):
        _check(self._lib.lbx_batch_sync(self._h))

    def reduce(self, sample: int) -> dict:
        r = _CReductions()
        _check(self._lib.lbx_batch_reduce(self._h, sample, C.byref(r)))
        return dict(mass=r.mass, momentum=tuple(r.momentum), u_sum=tuple(r.u_sum),
                    rho_min=r.rho_min, rho_max=r.rho_max, fluid_nodes=r.fluid_nodes)

    def launch_count(self) -> int:
        return int(self._lib.lbx_batch_launch_count(self._h))
