"""The benchmark configurations of the LBM path, runnable end to end.

    python -m lbx.configs cfg1 [--steps 2000]
    python -m lbx.configs cfg2 [--steps 10000]
    python -m lbx.configs cfg3 [--steps 20000] [--edge 192] [--quick]
    python -m lbx.configs cfg5 [--steps 4000]
    python -m lbx.configs cfg4 [--samples 512] [--steps 200] [--modes fused,...] [--quick]

cfg1: D2Q9 BGK 256x256, FP64, tau = 1.0, non-overlapping discs r = 8 to
      porosity 0.6 (the inlet/outlet rows kept fluid), Zou-He pressure
      rho_in = 1.001 / rho_out = 1.0, periodic across, start at rho = 1,
      u = 0.  The reference has pressure faces on its y faces only (north /
      south rows), so the flow runs along j; the lattice is the transpose of
      an x-directed channel.  Reports MLUPS and the Darcy permeability
      k = nu <u_flow> L / dp with nu = (tau - 1/2)/3, dp = (rho_in - rho_out)/3,
      L = 255 and <.> over all nodes (superficial).
cfg2: D3Q19 BGK 256^3, tau = 0.8, overlapping spheres r = 6 to porosity 0.4,
      gx = 1e-6, periodic.  Runs FP32 shifted, FP64 shifted and FP64 plain
      (unshifted, compressible) populations; reports MLUPS of each and the
      permeability k = nu <u_x> / gx of each with the relative error of the
      FP32 run against the FP64 run.

cfg3: D3Q19 flow + D3Q19 solute, 192x192x384, FP32, tau = 0.9, tau_s = 0.7,
      overlapping spheres r = 5 to porosity 0.35 with the two z face planes
      kept fluid (reservoir layers), Zou-He density rho_in = 1.0005 on the
      bottom plane (k = 0) and rho_out = 1.0 on the top plane, solute C = 1
      held on the bottom plane, zero gradient on the top, C = 0 elsewhere at
      t = 0.  Reports MLUPS, the outlet breakthrough curve (mean C over the
      fluid nodes of the top plane, every step, FP64 sums), the solute mass
      (FP64) every 1000 steps, the same run in FP64 for the precision
      comparison, and the solute mass drift of a closed periodic box (no
      faces, no sink) holding a blob of solute, where mass must be conserved.
cfg5: discrete adjoint, D3Q19 flow + solute, 128^3, FP32 (FP64 gradient
      sums), spheres r = 4 to porosity 0.45 (face planes kept fluid),
      tau = 0.8, tau_s = 0.75, body force gx = 1e-5 (periodic flow along x),
      solute held at the bottom plane by a 128x128 profile ~ U[0, 1] (seeded),
      zero gradient at the top, 4000 steps, checkpoints every 100.
      Objectives over the last 500 steps on the top plane: mean C, and mean
      u_x (the outlet x-flux).  Gradients w.r.t. gx, tau, tau_s and the
      profile, checked against FP64 central differences (h = 1e-6, relative
      for the scalars, along random unit directions for the profile);
      reports the adjoint's cost relative to one forward solve.
cfg4: 512 independent D3Q19 samples, FP32 shifted, cubic edges drawn from
      U{32..96}, tau ~ U[0.6, 1.2], porosity ~ U[0.3, 0.7], sphere radius
      ~ U{3..6} (seed base + i), gx = 1e-6, periodic.  One batch; reports the
      aggregate MLUPS of FUSED, PERSISTENT and SEQUENTIAL runs, the mode the
      autotuner picks, and the per-sample permeabilities.

frames: the cfg2 lattice (FP32) with the reference's per-frame output every
      --frame-rate steps (summary line, 3D byte images and .dat files; the
      text dumps with --frame-files all) written to a scratch directory.
      Reports the MLUPS without frames, with the reference's pattern (wait
      for the frame step, copy the macro variables to pageable host memory,
      statistics, files; the GPU idles meanwhile) and with the asynchronous
      pipeline (lbx_frame_enqueue / lbx_frame_wait: the files of frame k are
      written while the steps after it run).

Each run prints one JSON line.  Times come from CUDA events on the stream
the kernels run on.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from . import Domain, Params, LBX_LAYOUT_AUTO
from . import geometry


def _timed_run(dom: Domain, t0: int, steps: int, frame_at_end: bool = True):
    import torch
    s = torch.cuda.Stream()
    dom.set_stream(s.cuda_stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    if frame_at_end:
        dom.run(t0, steps - 1, 0)
        dom.step(t0 + steps, write_mv=True)
    else:
        dom.run(t0, steps, 0)
    e1.record(s)
    s.synchronize()
    return e0.elapsed_time(e1) / 1e3


def cfg1_params(precision: int = 8, layout: int = LBX_LAYOUT_AUTO) -> tuple:
    LX = LY = 256
    # discs placed along the flow direction x' (= j here) with the first and
    # last x' columns kept fluid, then transposed so x' runs along j
    mask = geometry.transpose_2d(geometry.disc_pack(LY, LX, radius=8, porosity=0.6, seed=2026),
                                 LY, LX)
    p = Params(dims=2, LX=LX, LY=LY, LZ=1, precision=precision, tau=(1.0, 1.0),
               pressure_s_in=(1, 0), pressure_n_out=(1, 0), rho_in=1.001, rho_out=1.0,
               layout=layout)
    return p, mask


def run_cfg1(steps: int = 2000) -> dict:
    p, mask = cfg1_params()
    with Domain(p, mask) as dom:
        dom.init_equilibrium(0, 1.0, 0.0, 0.0)
        dom.run(0, 20, 0)                         # warm-up
        dom.init_equilibrium(0, 1.0, 0.0, 0.0)
        secs = _timed_run(dom, 0, steps)
        mv = dom.download_mv()
        info = dom.info()
    fluid = mask != 1
    nu = (1.0 - 0.5) / 3.0
    dp = (1.001 - 1.0) / 3.0
    u_flow = np.where(fluid, mv[0, 2], 0.0).mean()     # superficial, along j
    k = nu * u_flow * 255.0 / dp
    return {"config": "cfg1", "lattice": [256, 256], "dtype": "f64", "steps": steps,
            "porosity": float(fluid.mean()), "mlups": 256 * 256 * steps / secs / 1e6,
            "seconds": secs, "permeability": k, "mean_u_flow": float(u_flow),
            "layout": info["layout"], "faces_fused": info["faces_fused"]}


def cfg2_params(precision: int, accurate: int = 1, compressible: int = 0,
                layout: int = LBX_LAYOUT_AUTO, n: int = 256):
    mask = geometry.sphere_pack(n, n, n, radius=6, porosity=0.4, seed=1234)
    p = Params(dims=3, LX=n, LY=n, LZ=n, precision=precision, accurate=accurate,
               compressible=compressible, tau=(0.8, 1.0), gaccel=(1e-6, 0, 0, 0, 0, 0),
               layout=layout)
    return p, mask


def run_cfg2(steps: int = 10000, n: int = 256) -> list:
    out = []
    nu = (0.8 - 0.5) / 3.0
    ks = {}
    for name, prec, acc, comp in (("fp32_shifted", 4, 1, 0), ("fp64_shifted", 8, 1, 0),
                                  ("fp64_plain", 8, 0, 1)):
        p, mask = cfg2_params(prec, acc, comp, n=n)
        fluid = mask != 1
        with Domain(p, mask) as dom:
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            dom.run(0, 8, 0)
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            secs = _timed_run(dom, 0, steps)
            r = dom.reduce()
            info = dom.info()
        ux_mean = r["u_sum"][0] / mask.size        # superficial: solids hold u = 0
        k = nu * ux_mean / 1e-6
        ks[name] = k
        out.append({"config": "cfg2", "run": name, "lattice": [n] * 3, "steps": steps,
                    "mlups": n ** 3 * steps / secs / 1e6,
                    "mflups": int(fluid.sum()) * steps / secs / 1e6, "seconds": secs,
                    "permeability": k, "mass": r["mass"], "layout": info["layout"]})
    for o in out:
        o["perm_rel_err_vs_fp64_shifted"] = abs(o["permeability"] - ks["fp64_shifted"]) / abs(
            ks["fp64_shifted"])
    f32 = next(o for o in out if o["run"] == "fp32_shifted")
    plain = next(o for o in out if o["run"] == "fp64_plain")
    f32["speedup_vs_fp64_plain"] = f32["mlups"] / plain["mlups"]
    return out


def cfg3_params(precision: int = 4, shape=(192, 192, 384), faces: bool = True,
                seed: int = 3003):
    LX, LY, LZ = shape
    mask = geometry.sphere_pack(LX, LY, LZ, radius=5, porosity=0.35, seed=seed)
    if faces:
        m3 = mask.reshape(LZ, LY, LX)
        m3[0] = 0
        m3[-1] = 0
        kw = dict(pressure_b_in=(1, 0), pressure_t_out=(1, 0), rho_in=1.0005, rho_out=1.0,
                  constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0)
    else:
        kw = {}
    p = Params(dims=3, LX=LX, LY=LY, LZ=LZ, nsubs=2, precision=precision, tau=(0.9, 0.7),
               sigma_t_on=0, sigma_t_off=1 << 30, **kw)
    return p, mask


def _cfg3_run(p, mask, steps: int, chunk: int, blob: bool = False):
    import torch
    LX, LY, LZ = p.LX, p.LY, p.LZ
    with Domain(p, mask) as dom:
        dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        if blob:
            k, j, i = np.meshgrid(np.arange(LZ), np.arange(LY), np.arange(LX), indexing="ij")
            r2 = (i - LX / 2) ** 2 + (j - LY / 2) ** 2 + (k - LZ / 2) ** 2
            c0 = np.where(r2 < (min(LX, LY, LZ) / 4) ** 2, 1.0, 0.0).reshape(-1)
        else:
            c0 = np.zeros(p.NN)
        dom.init_equilibrium(1, c0, 0.0, 0.0, 0.0)
        s = torch.cuda.Stream()
        dom.set_stream(s.cuda_stream)
        dom.step(1, write_mv=False)
        dom.step(2, write_mv=True)
        m0 = dom.reduce()["solute_mass"]
        dom.btc_start(LZ - 1, steps)
        masses = []
        secs = 0.0
        t = 2
        while t < steps + 2:
            n = min(chunk, steps + 2 - t)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            dom.run(t, n, n)
            e1.record(s)
            s.synchronize()
            secs += e0.elapsed_time(e1) / 1e3
            t += n
            masses.append((t, dom.reduce()["solute_mass"]))
        btc = dom.btc_read()
        r = dom.reduce()
    return dict(seconds=secs, m0=m0, masses=masses, btc=btc, reduce=r)


def run_cfg3(steps: int = 20000, shape=(192, 192, 384), chunk: int = 1000,
             quick: bool = False) -> list:
    """quick: the FP32 run between the faces only (no FP64 comparison, no
    closed box), e.g. under a profiler."""
    out = []
    res = {}
    for name, prec in (("fp32", 4),) + ((("fp64", 8),) if not quick else ()):
        p, mask = cfg3_params(prec, shape)
        r = _cfg3_run(p, mask, steps, chunk)
        res[name] = r
        btc = r["btc"]
        first = lambda x: int(np.argmax(btc > x)) + 3 if (btc > x).any() else None
        out.append({"config": "cfg3", "run": name, "lattice": list(shape), "steps": steps,
                    "mlups": p.NN * steps / r["seconds"] / 1e6, "seconds": r["seconds"],
                    "fluid_nodes": int((mask != 1).sum()),
                    "btc_every_1000": [float(btc[i]) for i in range(999, len(btc), 1000)],
                    "btc_first_above_0.01": first(0.01), "btc_first_above_0.5": first(0.5),
                    "solute_mass_every_chunk": [[t, m] for t, m in r["masses"]],
                    "flow_mass": r["reduce"]["mass"]})
    if quick:
        return out
    b32, b64 = res["fp32"]["btc"], res["fp64"]["btc"]
    m32, m64 = res["fp32"]["masses"][-1][1], res["fp64"]["masses"][-1][1]
    out.append({"config": "cfg3", "compare": "fp32_vs_fp64",
                "btc_max_abs_diff": float(np.abs(b32 - b64).max()),
                "btc_max": float(np.abs(b64).max()),
                "solute_mass_rel_diff": abs(m32 - m64) / abs(m64)})
    for name, prec in (("fp32", 4), ("fp64", 8)):
        p, mask = cfg3_params(prec, shape, faces=False)
        r = _cfg3_run(p, mask, steps, chunk * 5, blob=True)
        out.append({"config": "cfg3", "run": "closed_box_" + name, "steps": steps,
                    "solute_mass_start": r["m0"], "solute_mass_end": r["masses"][-1][1],
                    "solute_mass_rel_drift": (r["masses"][-1][1] - r["m0"]) / r["m0"],
                    "mlups": p.NN * steps / r["seconds"] / 1e6})
    return out


def cfg5_params(precision: int = 4, n: int = 128, gx: float = 1e-5, tau: float = 0.8,
                tau_s: float = 0.75, seed: int = 5005):
    mask = geometry.sphere_pack(n, n, n, radius=4, porosity=0.45, seed=seed)
    m3 = mask.reshape(n, n, n)
    m3[0] = 0
    m3[-1] = 0
    p = Params(dims=3, LX=n, LY=n, LZ=n, nsubs=2, precision=precision, tau=(tau, tau_s),
               gaccel=(gx, 0, 0, 0, 0, 0), sigma_t_on=0, sigma_t_off=1 << 30,
               constcon_b_in=1, zeroconcgrad_t=1, rho_sigma_in=1.0)
    profile = np.random.default_rng(seed + 1).uniform(0.0, 1.0, n * n)
    return p, mask, profile


def _cfg5_objective(p, mask, profile, steps, K, obj, grads, stream=None):
    """J (and its gradients) of one run; with gradients the run is done twice
    on the same domain and the second is timed (the steady state of an
    optimisation loop: checkpoints and workspace already allocated)."""
    import torch
    with Domain(p, mask) as dom:
        if stream is not None:
            dom.set_stream(stream.cuda_stream)
        dom.set_face_profile(False, profile)
        s = stream or torch.cuda.current_stream()
        for rep in range(2 if grads else 1):
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            dom.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(s)
            J = dom.adjoint_forward(0, steps, K, *obj)
            e1.record(s)
            g = dom.adjoint_backward(profile_b=True) if grads else None
            e2.record(s)
            s.synchronize()
        return J, g, e0.elapsed_time(e1) / 1e3, (e1.elapsed_time(e2) / 1e3 if grads else 0.0)


def run_cfg5(steps: int = 4000, n: int = 128, K: int = 100, window: int = 500,
             fd_dirs: int = 2) -> list:
    import torch
    s = torch.cuda.Stream()
    out = []
    plane = n - 1
    window = min(window, steps)
    objs = {"outlet_C": (plane, steps - window + 1, steps, 1.0, 0.0),
            "outlet_ux": (plane, steps - window + 1, steps, 0.0, 1.0)}
    p32, mask, prof = cfg5_params(4, n)
    # plain forward solve (the cost unit): lbx_run, no checkpoints
    with Domain(p32, mask) as dom:
        dom.set_stream(s.cuda_stream)
        dom.set_face_profile(False, prof)
        dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        dom.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
        dom.run(0, 20, 0)
        dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        dom.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        dom.run(0, steps, 0)
        e1.record(s)
        s.synchronize()
        t_plain = e0.elapsed_time(e1) / 1e3
    rng = np.random.default_rng(77)
    dirs = [v / np.linalg.norm(v) for v in rng.standard_normal((fd_dirs, n * n))]
    base = dict(gx=1e-5, tau=0.8, tau_s=0.75)
    for name, obj in objs.items():
        J32, g, t_fwd, t_bwd = _cfg5_objective(p32, mask, prof, steps, K, obj, True, s)
        p64, _, _ = cfg5_params(8, n)
        # the FP64 adjoint: the exact discrete gradient of the FP64 forward
        J64, g64, _, _ = _cfg5_objective(p64, mask, prof, steps, K, obj, True, s)

        def J_at(**kw):
            q = dict(base, **{k: v for k, v in kw.items() if k != "dprof"})
            pp, _, _ = cfg5_params(8, n, **q)
            return _cfg5_objective(pp, mask, prof + kw.get("dprof", 0.0), steps, steps, obj,
                                   False, s)[0]

        checks = {}
        for key, adj in (("gx", g["d_gaccel"][0]), ("tau", g["d_tau"]), ("tau_s", g["d_tau_s"])):
            h = 1e-6 * base[key]
            fd = (J_at(**{key: base[key] + h}) - J_at(**{key: base[key] - h})) / (2 * h)
            a64 = g64["d_gaccel"][0] if key == "gx" else g64["d_" + key]
            checks[key] = {"adjoint_fp32": adj, "adjoint_fp64": a64, "fd_fp64": fd,
                           "rel_err": abs(adj - fd) / max(abs(fd), 1e-300) if fd != 0 else abs(adj),
                           "fp64_adjoint_vs_fd": abs(a64 - fd) / max(abs(fd), 1e-300) if fd != 0 else abs(a64),
                           "fp32_vs_fp64_adjoint": abs(adj - a64) / max(abs(a64), 1e-300) if a64 != 0 else abs(adj)}
        for q, v in enumerate(dirs):
            h = 1e-6
            fd = (J_at(dprof=h * v) - J_at(dprof=-h * v)) / (2 * h)
            adj = float(g["d_profile_b"] @ v)
            a64 = float(g64["d_profile_b"] @ v)
            checks["profile_dir%d" % q] = {"adjoint_fp32": adj, "adjoint_fp64": a64, "fd_fp64": fd,
                                           "rel_err": abs(adj - fd) / max(abs(fd), 1e-300) if fd != 0 else abs(adj),
                                           "fp64_adjoint_vs_fd": abs(a64 - fd) / max(abs(fd), 1e-300) if fd != 0 else abs(a64),
                                           "fp32_vs_fp64_adjoint": abs(adj - a64) / max(abs(a64), 1e-300) if a64 != 0 else abs(adj)}
        out.append({"config": "cfg5", "objective": name, "lattice": [n] * 3, "steps": steps,
                    "checkpoint_every": K, "J_fp32": J32, "J_fp64": J64,
                    "J_rel_err": abs(J32 - J64) / abs(J64) if J64 else None,
                    "gradients": checks,
                    "profile_grad_norm": float(np.linalg.norm(g["d_profile_b"])),
                    "profile_grad_rel_err_vs_fp64_adjoint": float(
                        np.linalg.norm(g["d_profile_b"] - g64["d_profile_b"]) /
                        max(np.linalg.norm(g64["d_profile_b"]), 1e-300)),
                    "seconds_plain_forward": t_plain, "seconds_adjoint_forward": t_fwd,
                    "seconds_adjoint_backward": t_bwd,
                    "cost_vs_forward": (t_fwd + t_bwd) / t_plain})
    return out


def cfg4_samples(nsamples: int = 512, seed: int = 4000):
    rng = np.random.default_rng(seed)
    params, masks = [], []
    for i in range(nsamples):
        n = int(rng.integers(32, 97))
        tau = float(rng.uniform(0.6, 1.2))
        por = float(rng.uniform(0.3, 0.7))
        r = int(rng.integers(3, 7))
        masks.append(geometry.sphere_pack(n, n, n, r, por, seed + 1 + i))
        params.append(Params(dims=3, LX=n, LY=n, LZ=n, precision=4, tau=(tau, 1.0),
                             gaccel=(1e-6, 0, 0, 0, 0, 0)))
    return params, masks


def run_cfg4(nsamples: int = 512, steps: int = 200, perm_steps: int = 0,
             modes=("fused", "persistent", "sequential"), independent: bool = True,
             autotune: bool = True) -> list:
    import torch
    from .batch import Batch
    params, masks = cfg4_samples(nsamples)
    nodes = sum(m.size for m in masks)
    fluid = sum(int((m != 1).sum()) for m in masks)
    out = []
    with Batch(params, masks) as b:
        s = torch.cuda.Stream()
        b.set_stream(s.cuda_stream)
        times = {}
        for mode in modes:
            for i in range(nsamples):
                b.init_equilibrium(i, 1.0)
            b.run(0, 4, 0, mode=mode)                    # warm-up (graph capture)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.run(4, steps, 0, mode=mode)
            e1.record(s)
            s.synchronize()
            times[mode] = e0.elapsed_time(e1) / 1e3
        for mode, secs in times.items():
            line = {"config": "cfg4", "mode": mode, "samples": nsamples, "steps": steps,
                    "nodes": nodes, "fluid_nodes": fluid,
                    "mlups": nodes * steps / secs / 1e6,
                    "mflups": fluid * steps / secs / 1e6, "seconds": secs}
            if "sequential" in times:
                line["speedup_vs_sequential"] = times["sequential"] / secs
            out.append(line)
        if autotune:
            for i in range(nsamples):
                b.init_equilibrium(i, 1.0)
            tuned = b.autotune(6)
            out.append({"config": "cfg4", "autotuned": {"mode": tuned[0], "block": tuned[1]}})
        if perm_steps:
            for i in range(nsamples):
                b.init_equilibrium(i, 1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.run(0, perm_steps, perm_steps)
            e1.record(s)
            s.synchronize()
            secs = e0.elapsed_time(e1) / 1e3
            ks = []
            for i, p in enumerate(params):
                r = b.reduce(i)
                nu = (p.tau[0] - 0.5) / 3.0
                ks.append(nu * (r["u_sum"][0] / p.NN) / 1e-6)
            ks = np.array(ks)
            out.append({"config": "cfg4", "run": "permeability", "steps": perm_steps,
                        "mlups": nodes * perm_steps / secs / 1e6, "seconds": secs,
                        "k_min": float(ks.min()), "k_median": float(np.median(ks)),
                        "k_max": float(ks.max()), "k_first8": [float(x) for x in ks[:8]]})
    if not independent:
        return out
    # the same samples as independent lattices, one after another (what a
    # caller without the batch API runs): only the stepping is timed
    secs_ind = 0.0
    for p, m in zip(params, masks):
        with Domain(p, m) as dom:
            dom.set_stream(s.cuda_stream)
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            dom.run(0, 4, 0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            dom.run(4, steps, 0)
            e1.record(s)
            s.synchronize()
            secs_ind += e0.elapsed_time(e1) / 1e3
    out.append({"config": "cfg4", "mode": "independent_domains", "samples": nsamples,
                "steps": steps, "nodes": nodes, "fluid_nodes": fluid,
                "mlups": nodes * steps / secs_ind / 1e6, "mflups": fluid * steps / secs_ind / 1e6,
                "seconds": secs_ind,
                "fused_speedup": secs_ind / times["fused"]})
    return out


def run_frames(steps: int = 2000, frame_rate: int = 200, n: int = 256,
               files: str = "summary,raw,dat") -> list:
    import os
    import shutil
    import tempfile
    import time

    from . import host

    kinds = {"summary": host.FRAME_SUMMARY, "raw": host.FRAME_RAW, "dat": host.FRAME_DAT,
             "txt": host.FRAME_TXT, "all": host.FRAME_ALL}
    flags = 0
    for k in files.split(","):
        flags |= kinds[k]
    p, mask = cfg2_params(4, n=n)
    out = []
    nframes = steps // frame_rate
    work = tempfile.mkdtemp(prefix="lbx_frames_")
    try:
        for mode in ("none", "sync", "async"):
            with Domain(p, mask) as dom:
                dom.init_equilibrium(0, np.ones(p.NN), np.zeros(p.NN), np.zeros(p.NN),
                                     np.zeros(p.NN))
                dom.run(0, 2 * frame_rate, frame_rate)      # warm-up (graphs, allocations)
                dom.frame_enqueue(0)
                dom.frame_wait()
                dom.sync()
                t0 = 2 * frame_rate
                outdir = os.path.join(work, mode)
                os.makedirs(outdir)
                w0 = time.perf_counter()
                if mode == "none":
                    dom.run(t0, nframes * frame_rate, 0)
                    dom.sync()
                elif mode == "sync":
                    for k in range(1, nframes + 1):
                        dom.run(t0 + (k - 1) * frame_rate, frame_rate, frame_rate)
                        dom.sync()
                        mv = dom.download_mv()
                        st = [dom.frame_stats(s) for s in range(p.nsubs)]
                        host.write_frame(outdir, 3, p.LX, p.LY, p.LZ, t0 + k * frame_rate, k,
                                         mv, st, mask, flags)
                else:
                    for k in range(1, nframes + 1):
                        dom.run(t0 + (k - 1) * frame_rate, frame_rate, frame_rate)
                        dom.frame_enqueue(t0 + k * frame_rate)
                        if k > 1:
                            fr = dom.frame_wait(copy=False)
                            host.write_frame(outdir, 3, p.LX, p.LY, p.LZ, fr["time"], k - 1,
                                             fr["mv"], fr["stats"], mask, flags)
                    fr = dom.frame_wait(copy=False)
                    host.write_frame(outdir, 3, p.LX, p.LY, p.LZ, fr["time"], nframes,
                                     fr["mv"], fr["stats"], mask, flags)
                    dom.sync()
                wall = time.perf_counter() - w0
                nbytes = sum(os.path.getsize(os.path.join(outdir, f)) for f in os.listdir(outdir))
                shutil.rmtree(outdir)
            out.append(dict(run="frames", mode=mode, edge=n, steps=nframes * frame_rate,
                            frame_rate=frame_rate, frames=0 if mode == "none" else nframes,
                            files=files, wall_s=round(wall, 4),
                            mlups=round(p.NN * nframes * frame_rate / wall / 1e6, 1),
                            bytes_per_frame=0 if mode == "none" else nbytes // nframes))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    base = out[0]["wall_s"]
    for o in out[1:]:
        o["overhead_ms_per_frame"] = round((o["wall_s"] - base) / o["frames"] * 1e3, 2)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5", "frames"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--edge", type=int, default=256)
    ap.add_argument("--samples", type=int, default=512)
    ap.add_argument("--perm-steps", type=int, default=0)
    ap.add_argument("--checkpoint-every", type=int, default=100)
    ap.add_argument("--fd-dirs", type=int, default=2)
    ap.add_argument("--frame-rate", type=int, default=200)
    ap.add_argument("--frame-files", default="summary,raw,dat")
    ap.add_argument("--modes", default="fused,persistent,sequential",
                    help="cfg4: batch modes to time, comma-separated")
    ap.add_argument("--quick", action="store_true",
                    help="cfg4: skip the autotuner and the independent-lattice comparison; "
                         "cfg3: the FP32 run between the faces only (short runs, e.g. under "
                         "a profiler)")
    a = ap.parse_args(argv)
    if a.config == "cfg1":
        print(json.dumps(run_cfg1(a.steps or 2000)))
    elif a.config == "cfg5":
        for line in run_cfg5(a.steps or 4000, n=a.edge if a.edge != 256 else 128,
                             K=a.checkpoint_every, fd_dirs=a.fd_dirs):
            print(json.dumps(line))
    elif a.config == "cfg3":
        # --edge E: an E x E x 2E lattice instead of 192 x 192 x 384
        shape = (a.edge, a.edge, 2 * a.edge) if a.edge != 256 else (192, 192, 384)
        for line in run_cfg3(a.steps or 20000, shape, quick=a.quick):
            print(json.dumps(line))
    elif a.config == "frames":
        for line in run_frames(a.steps or 2000, a.frame_rate, a.edge, a.frame_files):
            print(json.dumps(line))
    elif a.config == "cfg4":
        for line in run_cfg4(a.samples, a.steps or 200, a.perm_steps,
                             modes=tuple(m for m in a.modes.split(",") if m),
                             independent=not a.quick, autotune=not a.quick):
            print(json.dumps(line))
    else:
        for line in run_cfg2(a.steps or 10000, a.edge):
            print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
