"""ctypes access to the CPU oracle and to the reference-kernel harness.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

* ``run_oracle`` -- oracle/liblbx_oracle.so, the C restatement of the
  reference's GPU path (oracle/lbx_oracle.c).
* ``run_reference`` -- oracle/_ref/librefk_<variant>.so, the reference's own
  kernel sources compiled for the CPU (oracle/refk_harness.c).  Present only
  where the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liblbx_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")


def reference_root() -> str:
    """The reference project's checkout (present only where the reference-side
    checker is built): $LBX_REFERENCE_ROOT, else a directory named
    `reference` beside this repository."""
    env = os.environ.get("LBX_REFERENCE_ROOT")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


@dataclass
class Params:
    """Run parameters, named as in the reference's params.in."""
    dims: int = 3
    LX: int = 8
    LY: int = 8
    LZ: int = 8
    nsubs: int = 1
    accurate: int = 1
    compressible: int = 0
    tau: tuple = (1.0, 1.0)
    rho_A: tuple = (1.0, 1.0)
    gaccel: tuple = (0.0,) * 6
    sink: float = 0.0
    sigma_t_on: int = 0
    sigma_t_off: int = 1 << 30
    pressure_n_in: tuple = (0, 0)
    pressure_s_in: tuple = (0, 0)
    pressure_n_out: tuple = (0, 0)
    pressure_s_out: tuple = (0, 0)
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
    # 3D z faces (top = k = LZ-1, bottom = k = 0)
    pressure_t_in: tuple = (0, 0)
    pressure_b_in: tuple = (0, 0)
    pressure_t_out: tuple = (0, 0)
    pressure_b_out: tuple = (0, 0)
    constcon_t_in: int = 0
    constcon_b_in: int = 0
    zeroconcgrad_t: int = 0
    zeroconcgrad_b: int = 0
    rho_sigma_in: float = 1.0
    constcon_profile_t: Optional[np.ndarray] = None
    constcon_profile_b: Optional[np.ndarray] = None
    kahan: int = 0
    walsh: int = 0
    ns: Optional[np.ndarray] = None     # per-node Walsh fraction (walsh == 1)
    velocity_t_in: tuple = (0, 0)
    velocity_t_out: tuple = (0, 0)
    velocity_b_in: tuple = (0, 0)
    velocity_b_out: tuple = (0, 0)
    uz_in: float = 0.0
    uz_out: float = 0.0
    # complex-step runs only: imaginary parts of tau, gaccel and the inlet
    # profiles (h times a direction)
    d_tau: tuple = (0.0, 0.0)
    d_gaccel: tuple = (0.0,) * 6
    d_profile_t: Optional[np.ndarray] = None
    d_profile_b: Optional[np.ndarray] = None

    @property
    def Q(self) -> int:
        return 9 if self.dims == 2 else 19

    @property
    def NN(self) -> int:
        return self.LX * self.LY * self.LZ


_D2 = C.c_double * 2
_D6 = C.c_double * 6
_I2 = C.c_int * 2


class _OrcParams(C.Structure):
    _fields_ = [
        ("dims", C.c_int), ("LX", C.c_int), ("LY", C.c_int), ("LZ", C.c_int),
        ("nsubs", C.c_int), ("accurate", C.c_int), ("compressible", C.c_int),
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
        ("pressure_t_in", _I2), ("pressure_b_in", _I2),
        ("pressure_t_out", _I2), ("pressure_b_out", _I2),
        ("constcon_t_in", C.c_int), ("constcon_b_in", C.c_int),
        ("zeroconcgrad_t", C.c_int), ("zeroconcgrad_b", C.c_int),
        ("rho_sigma_in", C.c_double),
        ("constcon_profile_t", C.POINTER(C.c_double)),
        ("constcon_profile_b", C.POINTER(C.c_double)),
        ("kahan", C.c_int),
        ("walsh", C.c_int),
        ("ns", C.POINTER(C.c_double)),
        ("velocity_t_in", C.c_int * 2),
        ("velocity_t_out", C.c_int * 2),
        ("velocity_b_in", C.c_int * 2),
        ("velocity_b_out", C.c_int * 2),
        ("uz_in", C.c_double),
        ("uz_out", C.c_double),
        ("d_tau", _D2),
        ("d_gaccel", _D6),
        ("d_profile_t", C.POINTER(C.c_double)),
        ("d_profile_b", C.POINTER(C.c_double)),
    ]


class _RefParams(C.Structure):
    _fields_ = [
        ("LX", C.c_int), ("LY", C.c_int), ("LZ", C.c_int),
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
    ]


def _fill(st, p: Params, keep):
    for name, _ in st._fields_:
        if name.startswith("constcon_profile") or name.startswith("d_profile") or name == "ns":
            v = getattr(p, name)
            if v is not None and np.size(v) > 0:
                arr = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
                keep.append(arr)
                setattr(st, name, arr.ctypes.data_as(C.POINTER(C.c_double)))
            continue
        if name.endswith("_table"):
            tab = getattr(p, name)
            if tab is not None:
                arr = np.ascontiguousarray(tab, dtype=np.float64)
                keep.append(arr)
                setattr(st, name, arr.ctypes.data_as(C.POINTER(C.c_double)))
                setattr(st, name.replace("_table", "_len"), len(arr))
            continue
        if name.endswith("_len"):
            continue
        v = getattr(p, name)
        if isinstance(v, tuple):
            fld = getattr(st, name)
            for i, x in enumerate(v):
                fld[i] = x
        else:
            setattr(st, name, v)


_oracle = None


def _lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        lib = C.CDLL(ORACLE_SO)
        for sfx, ct in (("f64", C.c_double), ("f32", C.c_float)):
            fn = getattr(lib, "orc_run_" + sfx)
            fn.argtypes = [C.POINTER(_OrcParams), C.POINTER(ct), C.c_void_p,
                           C.POINTER(ct), C.c_int, C.c_int, C.c_int, C.c_int]
            fn.restype = C.c_int
            fn = getattr(lib, "orc_run_btc_" + sfx)
            fn.argtypes = [C.POINTER(_OrcParams), C.POINTER(ct), C.c_void_p,
                           C.POINTER(ct), C.c_int, C.c_int, C.c_int, C.c_int,
                           C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
            fn.restype = C.c_int
            fn = getattr(lib, "orc_init_feq_" + sfx)
            fn.argtypes = [C.POINTER(_OrcParams)] + [C.POINTER(ct)] * 4 + [C.POINTER(ct)]
            fn.restype = C.c_int
        lib.orc_run_btc_cs.argtypes = [C.POINTER(_OrcParams), C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.orc_run_btc_cs.restype = C.c_int
        _oracle = lib
    return _oracle


def _ct(dtype):
    return C.c_double if np.dtype(dtype) == np.float64 else C.c_float


def _sfx(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def run_oracle(p: Params, f: np.ndarray, solids: np.ndarray, t0: int,
               nsteps: int, frame_rate: int = 0, mv: Optional[np.ndarray] = None,
               threads: int = 0):
    """Advance f ([nsubs, Q, N], float64 or float32) in place; returns (f, mv)."""
    dtype = f.dtype
    assert f.flags.c_contiguous and f.size == p.nsubs * p.Q * p.NN
    sol = np.ascontiguousarray(solids, dtype=np.uint8).reshape(-1)
    assert sol.size == p.NN
    if mv is None:
        mv = np.zeros((p.nsubs, 1 + p.dims, p.NN), dtype=dtype)
    keep = []
    st = _OrcParams()
    _fill(st, p, keep)
    nt = threads or min(os.cpu_count() or 1, 64)
    rc = getattr(_lib(), "orc_run_" + _sfx(dtype))(
        C.byref(st), f.ctypes.data_as(C.POINTER(_ct(dtype))),
        sol.ctypes.data, mv.ctypes.data_as(C.POINTER(_ct(dtype))),
        t0, nsteps, frame_rate, nt)
    if rc != 0:
        raise ValueError("orc_run rejected the parameters")
    return f, mv


def run_oracle_btc(p: Params, f: np.ndarray, solids: np.ndarray, t0: int,
                   nsteps: int, plane: int, frame_rate: int = 0,
                   mv: Optional[np.ndarray] = None, threads: int = 0):
    """run_oracle plus the plane record of the plane k (3D) / row j (2D) =
    `plane`: the mean solute C over its fluid nodes after every step (NaN
    while the solute is inactive) and the mean flow u_x.  Returns
    (f, mv, btc, btc_ux)."""
    dtype = f.dtype
    assert f.flags.c_contiguous and f.size == p.nsubs * p.Q * p.NN
    sol = np.ascontiguousarray(solids, dtype=np.uint8).reshape(-1)
    if mv is None:
        mv = np.zeros((p.nsubs, 1 + p.dims, p.NN), dtype=dtype)
    btc = np.zeros(nsteps, dtype=np.float64)
    btc_ux = np.zeros(nsteps, dtype=np.float64)
    st = _OrcParams()
    keep = []
    _fill(st, p, keep)
    nt = threads or min(os.cpu_count() or 1, 64)
    P = C.POINTER(C.c_double)
    rc = getattr(_lib(), "orc_run_btc_" + _sfx(dtype))(
        C.byref(st), f.ctypes.data_as(C.POINTER(_ct(dtype))),
        sol.ctypes.data, mv.ctypes.data_as(C.POINTER(_ct(dtype))),
        t0, nsteps, frame_rate, nt, plane, btc.ctypes.data_as(P), btc_ux.ctypes.data_as(P))
    if rc != 0:
        raise ValueError("orc_run_btc rejected the parameters")
    return f, mv, btc, btc_ux


def init_feq(p: Params, rho: np.ndarray, ux: np.ndarray, uy: np.ndarray,
             uz: Optional[np.ndarray], dtype=np.float64) -> np.ndarray:
    """Equilibrium initial state; rho/u are [nsubs, N]."""
    f = np.zeros((p.nsubs, p.Q, p.NN), dtype=dtype)
    arrs = [np.ascontiguousarray(x, dtype=dtype).reshape(p.nsubs, p.NN)
            for x in (rho, ux, uy, uz if uz is not None else np.zeros_like(rho))]
    st = _OrcParams()
    keep = []
    _fill(st, p, keep)
    ct = C.POINTER(_ct(dtype))
    getattr(_lib(), "orc_init_feq_" + _sfx(dtype))(
        C.byref(st), *[a.ctypes.data_as(ct) for a in arrs], f.ctypes.data_as(ct))
    return f


_refs = {}


def reference_available(variant: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, "librefk_%s.so" % variant))


def run_reference(variant: str, p: Params, f: np.ndarray, solids: np.ndarray,
                  t0: int, nsteps: int, frame_rate: int = 0,
                  mv: Optional[np.ndarray] = None):
    """Same contract as run_oracle, through the reference's own kernels."""
    if variant not in _refs:
        lib = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % variant))
        lib.refk_run.restype = C.c_int
        lib.refk_real_size.restype = C.c_int
        _refs[variant] = lib
    lib = _refs[variant]
    rs = lib.refk_real_size()
    assert f.dtype.itemsize == rs, "variant precision mismatch"
    assert lib.refk_num_dims() == p.dims and lib.refk_num_subs() == p.nsubs
    assert lib.refk_accurate() == p.accurate
    assert lib.refk_compressible() == p.compressible
    sol = np.ascontiguousarray(solids, dtype=np.uint8).reshape(-1)
    if mv is None:
        mv = np.zeros((p.nsubs, 1 + p.dims, p.NN), dtype=f.dtype)
    keep = []
    st = _RefParams()
    _fill(st, p, keep)
    lib.refk_walsh.restype = C.c_int
    assert lib.refk_walsh() == (1 if getattr(p, "walsh", 0) else 0)
    ns = None
    if getattr(p, "walsh", 0):
        ns = np.ascontiguousarray(np.zeros(p.NN) if p.ns is None else p.ns, dtype=f.dtype)
        lib.refk_set_ns(ns.ctypes.data_as(C.c_void_p))
    else:
        lib.refk_set_ns(None)
    rc = lib.refk_run(C.byref(st), f.ctypes.data_as(C.c_void_p),
                      sol.ctypes.data_as(C.c_void_p),
                      mv.ctypes.data_as(C.c_void_p), t0, nsteps, frame_rate)
    if rc != 0:
        raise ValueError("refk_run rejected the parameters")
    return f, mv


def variant_name(p: Params, dtype) -> str:
    base = "d2q9" if p.dims == 2 else "d3q19"
    if p.nsubs == 2:
        base += "s"
    elif not p.accurate:
        base += "p"
    elif p.compressible:
        base += "c"
    if getattr(p, "kahan", 0):
        base += "k"
    if getattr(p, "walsh", 0):
        base += "w"
    return base + "_" + _sfx(dtype)


def _ref_any():
    """Any built harness variant (the readers are the same in every variant)."""
    for v in ("d2q9_f64", "d3q19_f64"):
        if reference_available(v):
            if v not in _refs:
                lib = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % v))
                lib.refk_run.restype = C.c_int
                lib.refk_real_size.restype = C.c_int
                _refs[v] = lib
            return _refs[v]
    return None


def reference_read_params(path: str):
    """The reference's read_params (src/params.h:40-660) on `path`: selected
    fields as a dict, or None without the harness."""
    lib = _ref_any()
    if lib is None:
        return None
    iout = (C.c_int * 10)()
    dout = (C.c_double * 8)()
    lib.refk_read_params(path.encode(), iout, dout)
    keys_i = ["LX", "LY", "LZ", "NumFrames", "FrameRate", "initial_condition",
              "bc_ramp_start", "bc_ramp_stop", "pressure_n_in[0]", "pressure_s_in[0]"]
    keys_d = ["tau[0]", "rho_A[0]", "rho_B[0]", "rho_in", "rho_out", "sink",
              "gforce[0][0]", "pfmul"]
    out = dict(zip(keys_i, list(iout)))
    out.update(zip(keys_d, list(dout)))
    return out


def reference_read_bmp(path: str, LX: int, LY: int):
    """The reference's spy_bmp (src/lbio.c:3073-3363) decode, or None."""
    lib = _ref_any()
    if lib is None:
        return None
    out = np.zeros(LX * LY, np.uint8)
    lib.refk_read_bmp(path.encode(), LX, LY, out.ctypes.data_as(C.c_void_p))
    return out


def reference_read_raw(path: str, LX: int, LY: int, LZ: int):
    """The reference's read_solids (src/lbio.c:507-629), or None."""
    lib = _ref_any()
    if lib is None:
        return None
    out = np.zeros(LX * LY * LZ, np.uint8)
    lib.refk_read_raw(path.encode(), LX, LY, LZ, out.ctypes.data_as(C.c_void_p))
    return out


def frame_stats(mv_s: np.ndarray, mask: np.ndarray, dims: int) -> dict:
    """The frame statistics of compute_{max,min,ave}_{u,rho}
    (src/compute.c:1159-1416) for one substance's macro variables mv_s
    ([1+D][N]) over the nodes whose mask byte is 0 (is_not_solid,
    src/lattice.c:163-194): max and min of |rho| and |u_c| (a NaN never
    replaces a running max or min), and the means of rho and u_c; u_z = 0 in
    2D.  The sums are FP64."""
    keep = np.asarray(mask).reshape(-1) == 0
    nn = int(np.count_nonzero(keep))

    def one(v):
        v = np.asarray(v, dtype=np.float64)[keep]
        a = np.abs(v)
        ok = a[~np.isnan(a)]
        mx = max(0.0, float(ok.max())) if ok.size else 0.0
        mn = min(mx, float(ok.min())) if ok.size else mx
        return mx, mn, (float(np.sum(v)) / nn if nn else 0.0)

    r = one(mv_s[0])
    us = [one(mv_s[1 + c]) if c < dims else (0.0, 0.0, 0.0) for c in range(3)]
    return dict(nodes=nn, max_rho=r[0], min_rho=r[1], ave_rho=r[2],
                max_u=[u[0] for u in us], min_u=[u[1] for u in us],
                ave_u=[u[2] for u in us])


def reference_output_frame(variant: str, LX: int, LY: int, LZ: int, mv: np.ndarray,
                           sol: np.ndarray, time: int, frame: int, frame_rate: int,
                           workdir: str) -> bool:
    """The reference's output_frame (src/lbio.c:37-131) on macro variables
    mv ([nsubs][1+D][N] in the variant's precision) and mask bytes sol,
    writing into workdir/out.  False without the harness."""
    if not reference_available(variant):
        return False
    if variant not in _refs:
        _refs[variant] = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % variant))
    lib = _refs[variant]
    mv = np.ascontiguousarray(mv)
    sol = np.ascontiguousarray(sol, dtype=np.uint8)
    os.makedirs(os.path.join(workdir, "out"), exist_ok=True)
    here = os.getcwd()
    try:
        os.chdir(workdir)
        lib.refk_output_frame(LX, LY, LZ, mv.ctypes.data_as(C.c_void_p),
                              sol.ctypes.data_as(C.c_void_p), time, frame, frame_rate)
    finally:
        os.chdir(here)
    return True


def reference_cpu_loops(variant: str, p: Params, f: np.ndarray, solids: np.ndarray,
                        t0: int, nsteps: int) -> np.ndarray:
    """The reference's own host time loop (src/stream_collide_stream.c,
    src/collide.c: its CPU model, not the device arithmetic) on f in place,
    one thread; a cost baseline.  Periodic lattice with body force, one
    substance; `variant` names the flags it is built with."""
    if variant not in _refs:
        _refs[variant] = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % variant))
    lib = _refs[variant]
    lib.refk_real_size.restype = C.c_int
    assert f.dtype.itemsize == lib.refk_real_size(), "variant precision mismatch"
    assert f.flags.c_contiguous and f.size == p.nsubs * p.Q * p.NN
    sol = np.ascontiguousarray(solids, dtype=np.uint8).reshape(-1)
    g = (C.c_double * 3)(*[float(x) for x in p.gaccel[:3]])
    rc = lib.refk_cpu_loops(p.LX, p.LY, p.LZ, C.c_double(p.tau[0]), g,
                            sol.ctypes.data_as(C.c_void_p), f.ctypes.data_as(C.c_void_p),
                            int(t0), int(nsteps))
    if rc != 0:
        raise RuntimeError("refk_cpu_loops failed")
    return f


def reference_pest(variant: str, p: Params, f: np.ndarray, solids: np.ndarray, t0: int,
                   nsteps: int, workdir: str, frame_rate: int = 0,
                   mv: Optional[np.ndarray] = None):
    """The reference's PEST point sampling (src/latman.c:899-1232) around its
    own kernels: reads workdir/in/{timestep,x_coord,y_coord}_file.in, runs
    the steps, writes workdir/out/{conc_data,vel_data,conc_order}_proc0000.dat.
    Returns (f, mv, kept samples), or None without the harness variant."""
    if not reference_available(variant):
        return None
    if variant not in _refs:
        run_reference(variant, p, f.copy(), solids, t0, 0)     # loads the library
    lib = _refs[variant]
    os.makedirs(os.path.join(workdir, "out"), exist_ok=True)
    here = os.getcwd()
    try:
        os.chdir(workdir)
        kept = lib.refk_pest_begin(p.LX, p.LY, p.LZ)
        if kept < 0:
            raise ValueError("PEST input files missing in " + workdir)
        f, mv = run_reference(variant, p, f, solids, t0, nsteps, frame_rate, mv)
        lib.refk_pest_end()
    finally:
        os.chdir(here)
    return f, mv, kept


def pest_samples(p: Params, f: np.ndarray, solids: np.ndarray, t0: int, nsteps: int,
                 times, nodes, mv: Optional[np.ndarray] = None):
    """PEST point sampling restated (src/latman.c:1048-1176): samples in
    order; at each step t, while the next sample's time is t, take the
    solute's C and the flow's u_x, u_y at its node (written by that step).
    A sample whose time never comes blocks the ones after it, as in the
    reference.  Returns (f, mv, C, ux, uy, taken) with NaN for samples not
    taken."""
    times = list(times)
    nodes = list(nodes)
    n = len(times)
    c = np.full(n, np.nan)
    ux = np.full(n, np.nan)
    uy = np.full(n, np.nan)
    k = 0
    for t in range(t0 + 1, t0 + nsteps + 1):
        f, mv = run_oracle(p, f, solids, t - 1, 1, 1, mv=mv)
        while k < n and times[k] == t:
            c[k] = mv[1, 0, nodes[k]]
            ux[k] = mv[0, 1, nodes[k]]
            uy[k] = mv[0, 2, nodes[k]]
            k += 1
    return f, mv, c, ux, uy, k


def reference_pest_inputs(variant: str, LX: int, LY: int, LZ: int, workdir: str):
    """The reference's read_PEST_in_files on workdir/in: (order, time, x, y)
    of the kept samples, or None without the harness variant."""
    if not reference_available(variant):
        return None
    if variant not in _refs:
        _refs[variant] = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % variant))
    lib = _refs[variant]
    here = os.getcwd()
    try:
        os.chdir(workdir)
        kept = lib.refk_pest_begin(LX, LY, LZ)
        if kept < 0:
            return None
        arrs = [np.zeros(max(kept, 1), np.int32) for _ in range(4)]
        lib.refk_pest_samples(*[a.ctypes.data_as(C.c_void_p) for a in arrs])
        os.makedirs("out", exist_ok=True)
        lib.refk_pest_end()
    finally:
        os.chdir(here)
    return tuple(a[:kept] for a in arrs)


class _RefInit(C.Structure):
    _fields_ = [("initial_condition", C.c_int), ("rho_A", C.c_double * 2),
                ("rho_B", C.c_double * 2), ("rho_sigma", C.c_double),
                ("x1", C.c_int), ("x2", C.c_int), ("y1", C.c_int), ("y2", C.c_int),
                ("z1", C.c_int), ("z2", C.c_int)]


def reference_init_problem(variant: str, LX: int, LY: int, LZ: int, initial_condition: int,
                           rho_A=(1.0, 0.0), rho_B=(1.0, 0.0), rho_sigma: float = 0.0,
                           box=(0, -1, 0, -1, 0, -1)):
    """The reference's init_problem (src/latman.c:1270-2063) through the
    harness: (f [subs][Q][N], mv [subs][1+D][N]) in the variant's precision,
    or None without the harness.  Only initial_condition 0 and 2 exist in the
    reference (it exits on any other value); others raise ValueError here."""
    if not reference_available(variant):
        return None
    if variant not in _refs:
        _refs[variant] = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % variant))
    lib = _refs[variant]
    lib.refk_real_size.restype = C.c_int
    dims, nsubs = lib.refk_num_dims(), lib.refk_num_subs()
    Q = 9 if dims == 2 else 19
    dt = np.float64 if lib.refk_real_size() == 8 else np.float32
    NN = LX * LY * LZ
    f = np.zeros((nsubs, Q, NN), dt)
    mv = np.zeros((nsubs, 1 + dims, NN), dt)
    ip = _RefInit(initial_condition, (C.c_double * 2)(*rho_A), (C.c_double * 2)(*rho_B),
                  rho_sigma, *box)
    lib.refk_init_problem.restype = C.c_int
    rc = lib.refk_init_problem(LX, LY, LZ, C.byref(ip), f.ctypes.data_as(C.c_void_p),
                               mv.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError("initial_condition %d: the reference exits" % initial_condition)
    return f, mv


def reference_init_from_params(variant: str, path: str):
    """The reference's start-up path on a params.in: read_params
    (src/params.h:40-660) then init_problem (src/latman.c:1270-2063), through
    the harness.  (f [subs][Q][N], mv [subs][1+D][N]) in the variant's
    precision, or None without the harness; ValueError for an
    initial_condition the reference exits on."""
    if not reference_available(variant):
        return None
    if variant not in _refs:
        _refs[variant] = C.CDLL(os.path.join(REF_DIR, "librefk_%s.so" % variant))
    lib = _refs[variant]
    lib.refk_real_size.restype = C.c_int
    # the extents as this variant's read_params leaves them (a 2D build sets LZ = 1)
    iout = (C.c_int * 10)()
    dout = (C.c_double * 8)()
    lib.refk_read_params(path.encode(), iout, dout)
    rp = {"LX": iout[0], "LY": iout[1], "LZ": iout[2], "initial_condition": iout[5]}
    dims, nsubs = lib.refk_num_dims(), lib.refk_num_subs()
    Q = 9 if dims == 2 else 19
    dt = np.float64 if lib.refk_real_size() == 8 else np.float32
    NN = rp["LX"] * rp["LY"] * rp["LZ"]
    f = np.zeros((nsubs, Q, NN), dt)
    mv = np.zeros((nsubs, 1 + dims, NN), dt)
    lib.refk_init_from_params.restype = C.c_int
    rc = lib.refk_init_from_params(path.encode(), NN, f.ctypes.data_as(C.c_void_p),
                                   mv.ctypes.data_as(C.c_void_p))
    if rc == -1:
        raise ValueError("initial_condition %d: the reference exits" % rp["initial_condition"])
    if rc != 0:
        raise ValueError("refk_init_from_params failed (%d)" % rc)
    return f, mv


def run_oracle_btc_cs(p: Params, f: np.ndarray, solids: np.ndarray, t0: int, nsteps: int,
                      plane: int, threads: int = 0):
    """run_oracle_btc in complex arithmetic (the complex-step build): f is
    complex128 and advanced in place; p.d_tau, p.d_gaccel and
    p.d_profile_b/t give tau, gaccel and the inlet profiles imaginary parts.
    Returns (f, btc, btc_ux) with complex plane records."""
    assert f.dtype == np.complex128 and f.flags.c_contiguous
    assert f.size == p.nsubs * p.Q * p.NN
    sol = np.ascontiguousarray(solids, dtype=np.uint8).reshape(-1)
    mv = np.zeros((p.nsubs, 1 + p.dims, p.NN), np.complex128)
    btc = np.zeros(2 * nsteps)
    bux = np.zeros(2 * nsteps)
    keep = []
    st = _OrcParams()
    _fill(st, p, keep)
    nt = threads or min(os.cpu_count() or 1, 64)
    rc = _lib().orc_run_btc_cs(C.byref(st), f.ctypes.data, sol.ctypes.data, mv.ctypes.data,
                               t0, nsteps, 0, nt, plane,
                               btc.ctypes.data_as(C.POINTER(C.c_double)),
                               bux.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise ValueError("orc_run_btc_cs rejected the parameters")
    return f, btc[0::2] + 1j * btc[1::2], bux[0::2] + 1j * bux[1::2]


def tangent_objective(p: Params, f0: np.ndarray, solids: np.ndarray, nsteps: int,
                      plane: int, t_first: int, t_last: int, w_c: float, w_ux: float,
                      d_tau=(0.0, 0.0), d_gaccel=(0.0,) * 6, d_profile_b=None,
                      h: float = 1e-30):
    """The plane objective J = w_c mean_t <C>_plane + w_ux mean_t <u_x>_plane
    over the steps t_first..t_last of a run of `nsteps` steps from f0 (even
    time 0), and its forward-mode derivative dJ/dp . v along the direction
    v = (d_tau, d_gaccel, d_profile_b), by complex step with step h.
    Returns (J, dJ)."""
    import dataclasses
    q = dataclasses.replace(p)
    q.d_tau = tuple(h * x for x in d_tau)
    q.d_gaccel = tuple(h * x for x in d_gaccel)
    q.d_profile_b = None if d_profile_b is None else h * np.asarray(d_profile_b, np.float64)
    f = np.ascontiguousarray(f0, dtype=np.complex128).copy()
    _, btc, bux = run_oracle_btc_cs(q, f, solids, 0, nsteps, plane)
    win = slice(t_first - 1, t_last)
    J = 0j
    if w_c:
        J += w_c * np.mean(btc[win])
    if w_ux:
        J += w_ux * np.mean(bux[win])
    return float(J.real), float(J.imag / h)
