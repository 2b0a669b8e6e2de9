"""Benchmark: D3Q19 MLUPS of the AA-pattern LBM step on B200.

Workload (one replica per GPU; "replicas only" -- the path does not shard
here): D3Q19 BGK flow on a 256^3 lattice, FP32 shifted populations
(f_i - w_i rho_A), tau = 0.8, body force gx = 1e-6, periodic on every face,
solid mask = overlapping spheres of radius 6 from a fixed seed, added until
the porosity is 0.4.  Synthetic, seeded: no dataset is involved.

One bench step = one lattice time step (one odd or one even AA kernel; the
run alternates them as the reference does).  `value` = lattice node updates
per second over all ranks (MLUPS, all nodes); MFLUPS counts fluid nodes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--impl reference` times the reference's own implementation of this path on
the host cores: its kernel sources compiled for the CPU (oracle/_ref), on
the same lattice and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lbgpu-prime-dev_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N_EDGE = 256
TAU = 0.8
GX = 1e-6
RADIUS = 6
POROSITY = 0.4
SEED = 1234
Q = 19
REAL = 4
BYTES_PER_FLUID_UPDATE = 2 * Q * REAL          # 152 B: read + write 19 floats
FLAG_BYTES_PER_NODE = 1.0 / 8.0                 # bit-packed solid flag
METRIC = "D3Q19 MLUPS (FP32 shifted populations, 256^3 sphere pack)"


def workload_config(world: int) -> dict:
    return {
        "workload": "D3Q19 BGK %d^3, FP32 shifted populations, tau=0.8, gx=1e-6, "
                    "periodic, overlapping spheres r=6 to porosity 0.4 (seed 1234)" % N_EDGE,
        "lattice": [N_EDGE] * 3, "velocity_set": "D3Q19", "tau": TAU, "gx": GX,
        "sphere_radius": RADIUS, "porosity_target": POROSITY, "seed": SEED,
        "parallelism": "replicas x%d (one independent lattice per GPU)" % world,
        "l2": "inputs larger than L2 (%.2f GB populations per lattice)"
              % (Q * REAL * N_EDGE ** 3 / 1e9),
    }


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_traffic() -> dict:
    """DRAM bytes per launch of the step kernels (mean of the pair, odd,
    even) from the committed ncu summary of a 256^3 capture."""
    path = os.path.join(ROOT, "profiles", "aa_step_d3q19_f32_256cube.md")
    out = {"pair": None, "odd": None, "even": None}
    if not os.path.exists(path):
        return out
    text = open(path).read()
    for key, label in (("pair", "traffic"), ("odd", "traffic_odd"), ("even", "traffic_even")):
        m = re.search(r"^%s_bytes_per_launch:\s*([0-9.eE+]+)" % label, text, re.M)
        out[key] = float(m.group(1)) if m else None
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_mask():
    from lbx import geometry
    return geometry.sphere_pack(N_EDGE, N_EDGE, N_EDGE, RADIUS, POROSITY, SEED)


def cpu_baseline(mask, seconds: float = 10.0, max_steps: int = 64) -> dict:
    """The reference's kernels on the host cores, else the oracle port: AA
    step pairs of the full lattice until `seconds` have passed (bounded by
    `max_steps`)."""
    import pyoracle as po
    p = po.Params(dims=3, LX=N_EDGE, LY=N_EDGE, LZ=N_EDGE, tau=(TAU, 1.0),
                  gaccel=(GX, 0, 0, 0, 0, 0))
    f = np.zeros((1, Q, p.NN), np.float32)
    cores = os.cpu_count() or 1
    if po.reference_available("d3q19_f32"):
        kind = "reference"
        po.run_reference("d3q19_f32", p, f, mask, 0, 0)   # load the library
        po._refs["d3q19_f32"].refk_set_threads(cores)
        pair = lambda t: po.run_reference("d3q19_f32", p, f, mask, t, 2)
    else:
        kind = "port"
        pair = lambda t: po.run_oracle(p, f, mask, t, 2, threads=cores)
    steps = 0
    t0 = time.perf_counter()
    while True:
        pair(steps)
        steps += 2
        dt = time.perf_counter() - t0
        if dt >= seconds or steps >= max_steps:
            break
    return {"value": round(p.NN * steps / dt / 1e6, 3), "unit": "MLUPS", "cores": cores,
            "kind": kind,
            "sample": "%d lattice steps (%.1f s) of the full %d^3 workload, FP32, %s threads"
                      % (steps, dt, N_EDGE, cores)}


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return 0
    import pyoracle as po
    variant = "d3q19_f32"
    if not po.reference_available(variant):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (reference tree absent at build)"}))
        return 0
    mask = make_mask()
    p = po.Params(dims=3, LX=N_EDGE, LY=N_EDGE, LZ=N_EDGE, tau=(TAU, 1.0),
                  gaccel=(GX, 0, 0, 0, 0, 0))
    f = np.zeros((1, Q, p.NN), np.float32)
    cores = os.cpu_count() or 1
    po.run_reference(variant, p, f, mask, 0, 0)
    po._refs[variant].refk_set_threads(cores)
    # warm-up: an even number of steps, so the timed run starts at an even
    # time as every AA run must
    warm = args.warmup + (args.warmup % 2)
    po.run_reference(variant, p, f, mask, 0, warm)
    t0 = time.perf_counter()
    po.run_reference(variant, p, f, mask, warm, args.steps)
    dt = time.perf_counter() - t0
    value = p.NN * args.steps / dt / 1e6
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(1), "impl": "reference",
        "cpu_baseline": {"value": round(value, 3), "unit": "MLUPS", "cores": cores,
                         "kind": "reference",
                         "sample": "the full %d^3 lattice each step; the reference's "
                                   "kernel sources compiled for the host, %d threads"
                                   % (N_EDGE, cores)},
        "e2e": {"value": round(value, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def precision_leg(mask, local: int, steps: int) -> dict:
    """The rest of the headline metric on the same lattice: FP32 shifted
    populations against the plain FP64 model (ACCURATE 0, COMPRESSIBLE 1 in
    the reference, src/lattice.c:2880-2919) at the permeability error FP32
    costs.  Three runs of `steps` steps from rest (equilibrium at rho = 1):
    FP32 shifted and FP64 plain timed with CUDA events (seconds long, so the
    GPU sits at its sustained, power-capped clock; the FP32 run's clocks are
    sampled), and FP64 shifted as the reference result for the permeability
    k = nu <u_x> / g_x (superficial mean, FP64 device sums)."""
    import torch
    import lbx
    nu = (TAU - 0.5) / 3.0
    out = {}
    for name, prec, acc, comp in (("fp32_shifted", 4, 1, 0), ("fp64_plain", 8, 0, 1),
                                  ("fp64_shifted", 8, 1, 0)):
        p = lbx.Params(dims=3, LX=N_EDGE, LY=N_EDGE, LZ=N_EDGE, precision=prec, accurate=acc,
                       compressible=comp, tau=(TAU, 1.0), gaccel=(GX, 0, 0, 0, 0, 0),
                       device=local)
        stream = torch.cuda.Stream()
        with lbx.Domain(p, mask) as dom:
            dom.set_stream(stream.cuda_stream)
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            dom.run(0, 8, 0)                           # warm-up (graph capture)
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            torch.cuda.synchronize()
            sampler = ClockSampler(local) if name == "fp32_shifted" else None
            if sampler:
                sampler.start()
                time.sleep(0.3)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dom.run(0, steps - 1, 0)
            dom.step(steps, write_mv=True)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            clocks = sampler.stop() if sampler else None
            r = dom.reduce()
        k = nu * (r["u_sum"][0] / mask.size) / GX      # solid nodes hold u = 0
        out[name] = {"mlups": round(mask.size * steps / (ms / 1e3) / 1e6, 3),
                     "ms_per_step": round(ms / steps, 5), "permeability": k}
        if clocks:
            out[name]["clocks"] = clocks
    k64 = out["fp64_shifted"]["permeability"]
    for v in out.values():
        v["perm_rel_err_vs_fp64_shifted"] = abs(v["permeability"] - k64) / abs(k64)
    return out


def small_2d_leg(local: int, steps: int) -> dict:
    """The 2D case (256^2 D2Q9 FP64 between Zou-He pressure faces, discs of
    porosity 0.6, from rest): `steps` steps in one CUDA-event window, run
    as the library runs it (LBX_RUN_AUTO: the tiled path, rounds of steps on
    tiles in shared memory) and one launch per step (LBX_RUN_STEPS, graph
    replay), and the speed-up between them."""
    import torch
    import lbx
    from lbx import configs
    out = {}
    for mode in ("auto", "steps"):
        lp, mask = configs.cfg1_params(8)
        lp.device = local
        stream = torch.cuda.Stream()
        with lbx.Domain(lp, mask) as dom:
            dom.set_run_mode(mode)
            dom.set_stream(stream.cuda_stream)
            dom.init_equilibrium(0, 1.0, 0.0, 0.0)
            dom.run(0, 40, 0)                          # warm-up (plans, graphs)
            dom.init_equilibrium(0, 1.0, 0.0, 0.0)
            torch.cuda.synchronize()
            n0 = dom.launch_count()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dom.run(0, steps, 0)
            e1.record(stream)
            dom.sync()
            ms = e0.elapsed_time(e1)
            out[mode] = {"mlups": round(mask.size * steps / (ms / 1e3) / 1e6, 3),
                         "us_per_step": round(1e3 * ms / steps, 4),
                         "launches": dom.launch_count() - n0}
    out["tiled_over_steps"] = round(out["auto"]["mlups"] / out["steps"]["mlups"], 4)
    out["workload"] = "256^2 D2Q9 FP64, pressure_s_in / pressure_n_out, %d steps" % steps
    return out


def flow_solute_leg(local: int, steps: int) -> dict:
    """The coupled flow + solute lattice of the breakthrough case: 192 x 192
    x 384 D3Q19 FP32, spheres r = 5 to porosity 0.35 with the two z-face
    planes kept fluid, Zou-He density on the bottom (rho_in = 1.0005) and
    top (rho_out = 1.0) planes, solute C = 1 held at the bottom, zero
    gradient at the top, the outlet-plane record on: `steps` steps from rest
    in one CUDA-event window (one frame at the end).  The roofline counts
    2 x 152 B per fluid node update (both substances)."""
    import torch
    import lbx
    from lbx import configs
    p, mask = configs.cfg3_params(4)
    p.device = local
    fluid = int(np.count_nonzero(mask != 1))
    stream = torch.cuda.Stream()
    with lbx.Domain(p, mask) as dom:
        dom.set_stream(stream.cuda_stream)
        # the record is started once: starting it drops the captured graphs
        dom.btc_start(p.LZ - 1, 40 + steps)
        dom.init_equilibrium(0, 1.0)
        dom.init_equilibrium(1, 0.0)
        dom.run(0, 40, 40)                             # warm-up (graphs)
        dom.init_equilibrium(0, 1.0)                   # back to rest
        dom.init_equilibrium(1, 0.0)
        torch.cuda.synchronize()
        n0 = dom.launch_count()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dom.run(0, steps, steps)
        e1.record(stream)
        dom.sync()
        ms = e0.elapsed_time(e1)
        launches = dom.launch_count() - n0
        outlet_c = float(dom.btc_read()[-1])
    peaks = load_peaks()
    gbs = 2 * Q * REAL * 2 * fluid * steps / (ms / 1e3) / 1e9
    return {"mlups": round(mask.size * steps / (ms / 1e3) / 1e6, 3),
            "ms_per_step": round(ms / steps, 5), "steps": steps, "launches": launches,
            "fluid_nodes": fluid, "roofline_frac": round(gbs / peaks["hbm_gbs"], 4),
            "outlet_c_last": outlet_c,
            "workload": "192x192x384 D3Q19 flow + solute FP32, Zou-He z faces, C = 1 inlet, "
                        "outlet record, %d steps from rest" % steps}


def batch_leg(local: int, nsamples: int, steps: int) -> dict:
    """Many small lattices at once: 512 D3Q19 FP32 sphere packs with edges
    32..96 (172.8M nodes, 87.0M fluid) stepped as one batch (one launch per
    step, graph-replayed), timed over `steps` steps with CUDA events
    (`fused`, about half a second: the power-capped clock) and over the
    headline's 40-step window (`fused_40`); the roofline counts 152 B per
    fluid node update plus the rank-table bit per node, as the headline
    does.  Also the per-kind launch times and the per-sample launches of
    SEQUENTIAL mode."""
    import torch
    from lbx.batch import Batch
    from lbx.configs import cfg4_samples
    params, masks = cfg4_samples(nsamples)
    for p in params:
        p.device = local
    nodes = sum(m.size for m in masks)
    fluid = sum(int(np.count_nonzero(m != 1)) for m in masks)
    peaks = load_peaks()
    out = {"samples": nsamples, "nodes": nodes, "fluid_nodes": fluid, "steps": steps}
    with Batch(params, masks) as b:
        s = torch.cuda.Stream()
        b.set_stream(s.cuda_stream)
        for mode in ("fused", "sequential"):
            for i in range(nsamples):
                b.init_equilibrium(i, 1.0)
            b.run(0, 4, 0, mode=mode)                  # warm-up (graph capture)
            s.synchronize()
            sampler = ClockSampler(local) if mode == "fused" else None
            if sampler:
                sampler.start()
                time.sleep(0.3)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.run(4, steps, 0, mode=mode)
            e1.record(s)
            s.synchronize()
            if sampler:
                out["clocks"] = sampler.stop()
            secs = e0.elapsed_time(e1) / 1e3
            alg = fluid * BYTES_PER_FLUID_UPDATE + nodes * FLAG_BYTES_PER_NODE
            out[mode] = {"mlups": round(nodes * steps / secs / 1e6, 3),
                         "mflups": round(fluid * steps / secs / 1e6, 3),
                         "ms_per_step": round(1e3 * secs / steps, 4),
                         "frac": round(alg * steps / secs / 1e9 / peaks["hbm_gbs"], 4)}
        # the headline's 40-step window (a burst at the full clock), same run
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t = 4 + steps                                   # even: the next step is odd
        b.run(t, 4, 0, mode="fused")
        t += 4
        s.synchronize()
        e0.record(s)
        b.run(t, 40, 0, mode="fused")
        e1.record(s)
        s.synchronize()
        t += 40
        secs = e0.elapsed_time(e1) / 1e3
        alg = fluid * BYTES_PER_FLUID_UPDATE + nodes * FLAG_BYTES_PER_NODE
        out["fused_40"] = {"mlups": round(nodes * 40 / secs / 1e6, 3),
                           "ms_per_step": round(1e3 * secs / 40, 4),
                           "frac": round(alg * 40 / secs / 1e9 / peaks["hbm_gbs"], 4)}
        per_kind = {"odd": [], "even": []}
        for rep in range(8):
            for kind in ("odd", "even"):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(s)
                b.run(t, 1, 0, mode="fused")
                e1.record(s)
                s.synchronize()
                if rep >= 2:
                    per_kind[kind].append(e0.elapsed_time(e1))
                t += 1
        alg = fluid * BYTES_PER_FLUID_UPDATE + nodes * FLAG_BYTES_PER_NODE
        out["by_kind_ms"] = {k: round(float(np.median(v)), 4) for k, v in per_kind.items()}
        out["by_kind_frac"] = {k: round(alg / (float(np.median(v)) / 1e3) / 1e9 / peaks["hbm_gbs"], 4)
                               for k, v in per_kind.items()}
    out["fused_over_sequential"] = round(out["fused"]["mlups"] / out["sequential"]["mlups"], 4)
    out["workload"] = ("cfg 4: %d D3Q19 FP32 sphere packs, edges 32-96, porosity 0.3-0.7"
                       % nsamples)
    return out


def adjoint_leg(local: int, steps: int, K: int = 100, window: int = 500) -> dict:
    """The discrete adjoint's cost against a plain forward solve on the
    128^3 flow + solute configuration (sphere pack r = 4 to porosity 0.45,
    tau 0.8 / tau_s 0.75, gx 1e-5, C from a 128 x 128 inlet profile on the
    bottom plane): `steps` steps, checkpoints every K, objective = mean
    outlet C over the last `window` steps, gradients w.r.t. g, tau, tau_s
    and the profile.  CUDA-event times; the gradient run is the second on
    its domain (checkpoints and workspace allocated), as in an optimisation
    loop."""
    import torch
    from lbx import Domain, configs
    torch.cuda.set_device(local)
    s = torch.cuda.Stream()
    p, mask, prof = configs.cfg5_params(4, 128)
    with Domain(p, mask) as dom:
        dom.set_stream(s.cuda_stream)
        dom.set_face_profile(False, prof)
        for rep in range(2):
            dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
            dom.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            dom.run(0, steps if rep else 20, 0)
            e1.record(s)
            s.synchronize()
        t_plain = e0.elapsed_time(e1) / 1e3
    w = min(window, steps)
    obj = (p.LZ - 1, steps - w + 1, steps, 1.0, 0.0)
    J, g, t_fwd, t_bwd = configs._cfg5_objective(p, mask, prof, steps, K, obj, True, s)
    return {"value": round((t_fwd + t_bwd) / t_plain, 4), "unit": "x plain forward",
            "J": J, "d_gx": g["d_gaccel"][0], "d_tau": g["d_tau"], "d_tau_s": g["d_tau_s"],
            "profile_grad_norm": float(np.linalg.norm(g["d_profile_b"])),
            "seconds_plain_forward": round(t_plain, 5),
            "seconds_forward_with_checkpoints": round(t_fwd, 5),
            "seconds_backward": round(t_bwd, 5),
            "workload": "D3Q19 flow + solute 128^3, FP32 (FP64 gradient sums), %d steps, "
                        "checkpoints every %d, objective mean outlet C over the last %d "
                        "steps" % (steps, K, w)}


def max_over_ranks(dist, value: float, device) -> float:
    """The maximum of `value` over the ranks of the process group (the
    slowest replica sets the whole job's time); `value` itself without one."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(world: int, nodes: int, steps: int, seconds: float) -> float:
    """Whole-job MLUPS of `world` replicas that each advanced `nodes` nodes
    by `steps` steps in `seconds` (the slowest replica's time)."""
    return world * nodes * steps / seconds / 1e6


def cpu_table() -> int:
    """The CPU side on the host cores, beside the GPU numbers: the oracle
    port (C restatement, all cores) and the reference's own kernels
    (oracle/_ref, all cores and one core) on the 256^2 D2Q9 pressure-driven
    case and a 128^3 crop of the benchmark lattice (FP64 and FP32).  One
    JSON line per case and implementation; bounded samples (a few seconds
    each)."""
    import pyoracle as po
    from lbx import geometry
    cores = os.cpu_count() or 1
    cases = []
    m2 = geometry.transpose_2d(geometry.disc_pack(256, 256, radius=8, porosity=0.6, seed=1),
                               256, 256)
    p2 = po.Params(dims=2, LX=256, LY=256, LZ=1, tau=(1.0, 1.0), pressure_s_in=(1, 0),
                   pressure_n_out=(1, 0), rho_in=1.001, rho_out=1.0)
    cases.append(("D2Q9 256^2 FP64, Zou-He pressure", p2, m2, np.float64, "d2q9_f64", 40))
    m3 = geometry.sphere_pack(128, 128, 128, radius=6, porosity=0.4, seed=1234)
    for dt, v in ((np.float64, "d3q19_f64"), (np.float32, "d3q19_f32")):
        p3 = po.Params(dims=3, LX=128, LY=128, LZ=128, tau=(TAU, 1.0),
                       gaccel=(GX, 0, 0, 0, 0, 0))
        cases.append(("D3Q19 128^3 %s, benchmark lattice crop" % ("FP64" if dt == np.float64
                                                                   else "FP32"),
                      p3, m3, dt, v, 6))
    for name, p, mask, dt, variant, steps in cases:
        runs = [("port", cores)]
        if po.reference_available(variant):
            runs += [("reference", cores), ("reference", 1)]
        for kind, nt in runs:
            f = np.zeros((p.nsubs, p.Q, p.NN), dt)
            if kind == "port":
                po.run_oracle(p, f, mask, 0, 2, threads=nt)
                t0 = time.perf_counter()
                po.run_oracle(p, f, mask, 2, steps, threads=nt)
            else:
                po.run_reference(variant, p, f, mask, 0, 0)
                po._refs[variant].refk_set_threads(nt)
                po.run_reference(variant, p, f, mask, 0, 2)
                t0 = time.perf_counter()
                po.run_reference(variant, p, f, mask, 2, steps)
            dt_s = time.perf_counter() - t0
            print(json.dumps({"cpu_table": name, "kind": kind, "threads": nt,
                              "mlups": round(p.NN * steps / dt_s / 1e6, 3), "steps": steps,
                              "cpu": platform.processor() or platform.machine()}))
    # the reference's own host loops (stream_collide_stream.c + collide.c):
    # a different model (unshifted, no face rows), single-threaded as
    # shipped, built with ACCURATE 0 / COMPRESSIBLE 1; a cost baseline only
    for name, p, mask, dt, variant, steps in (
            (cases[0][0], cases[0][1], cases[0][2], np.float64, "d2q9p_f64", 20),
            (cases[1][0], cases[1][1], cases[1][2], np.float64, "d3q19p_f64", 4),
            (cases[2][0], cases[2][1], cases[2][2], np.float32, "d3q19p_f32", 4)):
        if not po.reference_available(variant):
            continue
        w = po.init_feq(po.Params(dims=p.dims, LX=p.LX, LY=p.LY, LZ=p.LZ, accurate=0,
                                  compressible=1),
                        np.ones((1, p.NN)), np.zeros((1, p.NN)), np.zeros((1, p.NN)),
                        np.zeros((1, p.NN))).astype(dt)
        f = np.ascontiguousarray(w)
        po.reference_cpu_loops(variant, p, f, mask, 0, 2)
        t0 = time.perf_counter()
        po.reference_cpu_loops(variant, p, f, mask, 2, steps)
        dt_s = time.perf_counter() - t0
        print(json.dumps({"cpu_table": name, "kind": "reference host loops", "threads": 1,
                          "mlups": round(p.NN * steps / dt_s / 1e6, 3), "steps": steps,
                          "finite": bool(np.isfinite(f).all()),
                          "cpu": platform.processor() or platform.machine()}))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="lbx", choices=["lbx", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision-steps", type=int, default=6000,
                    help="steps of each run of the FP32-vs-FP64 leg (0: skip it)")
    ap.add_argument("--adjoint-steps", type=int, default=4000,
                    help="steps of the adjoint cost leg (0: skip it)")
    ap.add_argument("--flow-solute-steps", type=int, default=2000,
                    help="steps of the flow + solute key (192x192x384 with z faces); 0: skip")
    ap.add_argument("--small-steps", type=int, default=2000,
                    help="steps of the 256^2 D2Q9 FP64 leg (0: skip it)")
    ap.add_argument("--batch-samples", type=int, default=512,
                    help="samples of the batched-lattice leg (0: skip it)")
    ap.add_argument("--batch-steps", type=int, default=200,
                    help="timed steps of the batched-lattice leg")
    ap.add_argument("--cpu-table", action="store_true",
                    help="print the host-core timings of the oracle port and of the "
                         "reference's kernels on the 2D case and a 128^3 crop, then exit")
    ap.add_argument("--edge", type=int, default=256,
                    help="lattice edge; 256 is the benchmark workload, smaller "
                         "edges are for profiling captures only")
    args = ap.parse_args(argv)
    global N_EDGE
    N_EDGE = args.edge
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.cpu_table:
        return cpu_table()
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    import lbx
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    mask = make_mask()
    fluid = int(np.count_nonzero(mask != 1))
    NN = mask.size
    params = lbx.Params(dims=3, LX=N_EDGE, LY=N_EDGE, LZ=N_EDGE, precision=REAL,
                        tau=(TAU, 1.0), gaccel=(GX, 0, 0, 0, 0, 0), device=local)
    # a dedicated stream: its handle is non-zero, and the events below are
    # recorded on the stream the step kernels run on
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dom = lbx.Domain(params, mask)
    dom.set_stream(stream.cuda_stream)
    dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
    layout = dom.info()["layout"]

    # warm-up (W >= 3 steps), then K timed steps between barriers
    t = 0
    dom.run(t, args.warmup, 0)
    t += args.warmup
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    launches0 = dom.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    dom.run(t, args.steps, 0)
    ev1.record(stream)
    torch.cuda.synchronize()
    t += args.steps
    ms = ev0.elapsed_time(ev1)
    launches = dom.launch_count() - launches0
    clocks = sampler.stop()
    ms = max_over_ranks(dist, ms, "cuda")
    if dist:
        dist.barrier()
    ms_step = ms / args.steps
    value = job_mlups(world, NN, args.steps, ms / 1e3)
    mflups = job_mlups(world, fluid, args.steps, ms / 1e3)

    # per-kind launch durations (odd = stream-collide-stream, even = collide)
    per_kind = {}
    for kind in ("odd", "even"):
        if (t % 2 == 0) != (kind == "odd"):
            dom.step(t + 1)
            t += 1
        reps = 6
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(reps)]
        durs = []
        for a, b in evs:
            a.record(stream)
            dom.step(t + 1)
            b.record(stream)
            t += 1
            dom.step(t + 1)   # keep the AA order; not timed
            t += 1
        torch.cuda.synchronize()
        durs = [a.elapsed_time(b) for a, b in evs]
        per_kind[kind] = float(np.median(durs))

    peaks = load_peaks()
    traffic = load_traffic()
    alg_bytes = fluid * BYTES_PER_FLUID_UPDATE + NN * FLAG_BYTES_PER_NODE
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    roofline = {
        "bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
        "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
        "traffic": traffic["pair"],
        "traffic_by_kind": {"odd": traffic["odd"], "even": traffic["even"]},
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at 256^3, "
                          "steady state (profiles/aa_step_d3q19_f32_256cube.md)",
        "peak_source": peaks["source"],
        "kernel": "%s<float,19,1,SHIFTED_INC> (odd and even alternate)"
                  % ("aa_step_compact" if layout == "compact" else "aa_step"),
        "alg_bytes_per_launch": alg_bytes,
        "by_kind_ms": {k: round(v, 4) for k, v in per_kind.items()},
        "by_kind_frac": {k: round(alg_bytes / (v / 1e3) / 1e9 / peaks["hbm_gbs"], 4)
                         for k, v in per_kind.items()},
    }

    # end to end through the C ABI with host buffers, K steps and the macro
    # variables of the last step back, started two ways: from the density
    # (the reference's init_problem: rho per node, u = 0, f = feq, here
    # formed on the device) and from an upload of all populations (a restart
    # from saved populations)
    f_host = torch.zeros((Q, NN), dtype=torch.float32, pin_memory=True)
    rho_host = torch.ones(NN, dtype=torch.float32, pin_memory=True)
    mv_host = torch.empty((4, NN), dtype=torch.float32, pin_memory=True)
    lib = lbx.load_library()
    h = dom._h

    def job(start):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        if start == "density":
            # rest at rho = 1: the same shifted populations (all zero) as the
            # upload; u given as NULL is zero (init_problem starts at rest)
            lbx._check(lib.lbx_init_equilibrium(h, 0, rho_host.data_ptr(), None, None, None))
        else:
            lbx._check(lib.lbx_upload_f(h, 0, f_host.data_ptr()))   # natural order at time 0
        lbx._check(lib.lbx_run(h, 0, args.steps - 1, 0))
        lbx._check(lib.lbx_step(h, args.steps, lbx.LBX_WRITE_MV))
        lbx._check(lib.lbx_download_mv(h, 0, mv_host[0].data_ptr(), mv_host[1].data_ptr(),
                                       mv_host[2].data_ptr(), mv_host[3].data_ptr()))
        return max_over_ranks(dist, time.perf_counter() - t0, "cuda")

    # one untimed job of each kind first, as the steps get warm-up steps: the
    # first copies into freshly pinned host buffers run ~3 ms slower
    job("density")
    job("populations")
    e2e_s = job("density")
    up_s = job("populations")
    e2e = {"value": round(job_mlups(world, NN, args.steps, e2e_s), 3), "unit": "MLUPS",
           "h2d_bytes_per_step": int(NN * REAL / args.steps),
           "d2h_bytes_per_step": int(4 * NN * REAL / args.steps),
           "note": "lbx_init_equilibrium from rho in pinned host memory, at rest (the "
                   "reference's init_problem start), K steps, download of rho,u of the last "
                   "step; wall clock, after one untimed job",
           "from_populations": {
               "value": round(job_mlups(world, NN, args.steps, up_s), 3), "unit": "MLUPS",
               "h2d_bytes_per_step": int(Q * NN * REAL / args.steps),
               "d2h_bytes_per_step": int(4 * NN * REAL / args.steps),
               "note": "lbx_upload_f of all populations instead (a restart), same steps "
                       "and download"}}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": workload_config(world),
        "mflups": round(mflups, 3), "fluid_nodes": fluid, "nodes": NN, "layout": layout,
        "roofline": roofline, "clocks": clocks, "e2e": e2e,
        "gpu_launches": launches,
    }
    if args.precision_steps > 0:
        prec = precision_leg(mask, local, args.precision_steps)
        f32, plain = prec["fp32_shifted"], prec["fp64_plain"]
        line["sustained"] = {
            "value": f32["mlups"], "unit": "MLUPS", "ms_per_step": f32["ms_per_step"],
            "steps": args.precision_steps, "clocks": f32.get("clocks"),
            "note": "FP32 shifted, one lattice, %d steps from rest in one CUDA-event "
                    "window (seconds long: the power-capped clock)" % args.precision_steps}
        line["fp64_plain"] = {
            "value": plain["mlups"], "unit": "MLUPS", "ms_per_step": plain["ms_per_step"],
            "steps": args.precision_steps,
            "model": "ACCURATE 0, COMPRESSIBLE 1 (plain compressible BGK), FP64"}
        line["fp32_over_fp64_plain"] = round(f32["mlups"] / plain["mlups"], 4)
        line["perm_rel_err"] = f32["perm_rel_err_vs_fp64_shifted"]
        line["precision"] = {
            k: {kk: vv for kk, vv in v.items() if kk != "clocks"} for k, v in prec.items()}
        line["precision"]["note"] = (
            "permeability k = nu <u_x> / g_x after %d steps from rest; perm_rel_err = "
            "|k(FP32 shifted) - k(FP64 shifted)| / k(FP64 shifted), the same kernels"
            % args.precision_steps)
    if args.adjoint_steps > 0:
        line["adjoint"] = adjoint_leg(local, args.adjoint_steps)
    if args.small_steps > 0:
        line["small_2d"] = small_2d_leg(local, args.small_steps)
    if args.flow_solute_steps > 0:
        line["flow_solute"] = flow_solute_leg(local, args.flow_solute_steps)
    if args.batch_samples > 0:
        line["batch"] = batch_leg(local, args.batch_samples, args.batch_steps)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(mask)
    dom.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
