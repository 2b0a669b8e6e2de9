"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own kernel sources (compiled for the CPU by
oracle/ref_build.py through oracle/refk_harness.c) on small seeded cases and
stores inputs and outputs as .npz.  Needs oracle/_ref (built where the
reference tree is available); the fixtures are committed so the tests need
neither the reference nor the harness.

    python tests/golden/make_golden.py [name ...]
    python tests/golden/make_golden.py init [name ...]   (the start-up path)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
W19 = np.array([1 / 3] + [1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] * 2 + [1 / 36] * 8)


def cases():
    out = []
    g3 = (2e-4, -3e-5, 5e-5, 0, 0, 0)
    for name, kw, dt in [
        ("d3q19_f64", dict(), np.float64),
        ("d3q19_f32", dict(), np.float32),
        ("d3q19p_f64", dict(accurate=0, compressible=1), np.float64),
        ("d3q19c_f64", dict(compressible=1), np.float64),
        ("d3q19s_f64", dict(nsubs=2, sink=2e-3, sigma_t_on=3, sigma_t_off=40), np.float64),
        ("d3q19s_f32", dict(nsubs=2, sink=2e-3, sigma_t_on=3, sigma_t_off=40), np.float32),
    ]:
        p = po.Params(dims=3, LX=10, LY=9, LZ=8, tau=(0.8, 0.7), gaccel=g3, **kw)
        out.append((name, p, dt, 16, 4))
    g2 = (2e-4, 3e-5, 0, 0, 0, 0)
    bc = dict(pressure_s_in=(1, 0), pressure_n_out=(1, 0), rho_in=1.004, rho_out=1.0,
              bc_ramp_start=2, bc_ramp_stop=9)
    for name, kw, dt in [
        ("d2q9_f64", dict(), np.float64),
        ("d2q9_f32", dict(), np.float32),
        ("d2q9p_f64", dict(accurate=0, compressible=1), np.float64),
        ("d2q9_bc_f64", bc, np.float64),
        ("d2q9_bc_f32", bc, np.float32),
        ("d2q9p_bc_f64", dict(bc, accurate=0, compressible=1), np.float64),
        ("d2q9_table_f64", dict(pressure_n_in=(2, 0), pressure_s_out=(1, 0), pfadd=1.0,
                                pfmul=0.01, rho_out=0.999,
                                pressure_n_table=np.array([0.1, 0.3, 0.2, 0.5, 0.4])),
         np.float64),
        ("d2q9s_bc_f64", dict(bc, nsubs=2, sink=1e-3, zeroconcgrad_n=1, zeroconcgrad_s=1),
         np.float64),
    ]:
        p = po.Params(dims=2, LX=12, LY=10, LZ=1, tau=(0.9, 0.75), gaccel=g2, **kw)
        out.append((name, p, dt, 18, 6))
    # compensated density sums (KAHAN_SUMMATION); last, so that the inputs of
    # the fixtures above keep their seeded draws
    for name, kw, dt in [
        ("d3q19k_f32", dict(kahan=1), np.float32),
        ("d3q19k_f64", dict(kahan=1), np.float64),
        ("d3q19sk_f32", dict(nsubs=2, kahan=1, sink=2e-3, sigma_t_on=3, sigma_t_off=40),
         np.float32),
    ]:
        p = po.Params(dims=3, LX=10, LY=9, LZ=8, tau=(0.8, 0.7), gaccel=g3, **kw)
        out.append((name, p, dt, 16, 4))
    p = po.Params(dims=2, LX=12, LY=10, LZ=1, tau=(0.9, 0.75), gaccel=g2, kahan=1)
    out.append(("d2q9k_f32", p, np.float32, 18, 6))
    # Walsh partial bounce-back (WALSH_NS_ON with COMPUTE_ON_SOLIDS); the
    # per-node fraction ns is drawn with the inputs
    for name, kw, dt in [
        ("d3q19w_f64", dict(walsh=1), np.float64),
        ("d3q19w_f32", dict(walsh=1), np.float32),
        ("d3q19sw_f64", dict(nsubs=2, walsh=1, sink=2e-3, sigma_t_on=3, sigma_t_off=40),
         np.float64),
    ]:
        p = po.Params(dims=3, LX=10, LY=9, LZ=8, tau=(0.8, 0.7), gaccel=g3, **kw)
        out.append((name, p, dt, 16, 4))
    p = po.Params(dims=2, LX=12, LY=10, LZ=1, tau=(0.9, 0.75), gaccel=g2, walsh=1)
    out.append(("d2q9w_f64", p, np.float64, 18, 6))
    # the solute switched on at t = 7 and off after t = 14 with zero-gradient
    # faces: the reference runs its face kernels on the idle solute too
    p = po.Params(dims=2, LX=12, LY=10, LZ=1, tau=(0.9, 0.75), gaccel=g2,
                  **dict(bc, nsubs=2, sink=1e-3, zeroconcgrad_n=1, zeroconcgrad_s=1,
                         sigma_t_on=7, sigma_t_off=14))
    out.append(("d2q9s_bc_gate_f64", p, np.float64, 18, 6))
    return out


def make_inputs(name, p, dtype, rng, fluid_faces):
    sol = rng.choice([0, 1, 255], size=p.NN, p=[0.72, 0.2, 0.08]).astype(np.uint8)
    if fluid_faces and p.dims == 2:
        m = sol.reshape(p.LY, p.LX)
        m[0, :] = np.where(m[0, :] == 1, 0, m[0, :])
        m[-1, :] = np.where(m[-1, :] == 1, 0, m[-1, :])
    f = rng.standard_normal((p.nsubs, p.Q, p.NN)) * 1e-3
    W = W9 if p.dims == 2 else W19
    if not p.accurate:
        f[0] += W[:, None]
    if p.nsubs == 2:
        f[1] = np.abs(f[1]) + 0.5 * W[:, None]
    if p.walsh:
        # fractions in [0, 1] with exact 0 (open) and 1 (full bounce-back)
        ns = rng.uniform(0.0, 1.0, size=p.NN)
        pick = rng.choice([0, 1, 2], size=p.NN, p=[0.5, 0.3, 0.2])
        ns = np.where(pick == 1, 0.0, np.where(pick == 2, 1.0, ns))
        p.ns = ns.astype(dtype).astype(np.float64)
    return sol, f.astype(dtype)


def main(only=None):
    """Writes every fixture, or only those named in `only` (the inputs of the
    others are still drawn, so each fixture's seeded inputs never change)."""
    rng = np.random.default_rng(20261203)
    for name, p, dtype, steps, fr in cases():
        variant = po.variant_name(p, dtype)
        for tag, fluid_faces in (("", True),) if "bc" not in name and "table" not in name \
                else (("", True), ("_wrapsolid", False)):
            sol, f0 = make_inputs(name, p, dtype, rng, fluid_faces)
            if only and name + tag not in only:
                continue
            f = f0.copy()
            f, mv = po.run_reference(variant, p, f, sol, 0, steps, frame_rate=fr)
            pd = {k: (np.asarray(v) if v is not None else np.array([]))
                  for k, v in p.__dict__.items()}
            np.savez_compressed(os.path.join(HERE, name + tag + ".npz"),
                                solids=sol, f0=f0, f=f, mv=mv, steps=steps,
                                frame_rate=fr, variant=variant,
                                **{"p_" + k: v for k, v in pd.items()})
            print(name + tag, variant, f.dtype, steps, "steps")


# ---- the start-up path ---------------------------------------------------------
# The reference's read_params + init_problem on params.in files that differ in
# initial_condition (0 uniform, 2 cube), dimensions, substances and model, with
# explicit and defaulted cube bounds.  Written to tests/golden/init/.
INIT_DIR = os.path.join(HERE, "init")


def init_cases():
    base2 = {"LX": 12, "LY": 10, "LZ": 1}
    base3 = {"LX": 10, "LY": 9, "LZ": 8}
    box2 = {"x1": 3, "x2": 8, "y1": 2, "y2": 5}
    box3 = {"x1": 2, "x2": 6, "y1": 1, "y2": 4, "z1": 1, "z2": 5}
    dflt = {"x1": -1, "x2": -1, "y1": -1, "y2": -1, "z1": -1, "z2": -1,
            "rel_x1": 0.25, "rel_x2": -1.0, "rel_y1": -1.0, "rel_y2": 0.6,
            "rel_z1": -1.0, "rel_z2": -1.0}
    ic0 = {"initial_condition": 0}
    ic2 = {"initial_condition": 2}
    rho = {"rho_A[0]": 1.003, "rho_B[0]": 1.05}
    return [
        ("d2q9_ic0_f64", "d2q9_f64", dict(base2, **ic0, **rho)),
        ("d2q9_ic2_f64", "d2q9_f64", dict(base2, **ic2, **rho, **box2)),
        ("d2q9p_ic2_f64", "d2q9p_f64", dict(base2, **ic2, **rho, **dflt)),
        ("d2q9s_ic0_f64", "d2q9s_f64", dict(base2, **ic0, **rho)),
        ("d2q9s_ic2_f64", "d2q9s_f64", dict(base2, **ic2, **rho, **box2, rho_sigma=0.8)),
        ("d3q19_ic2_f64", "d3q19_f64", dict(base3, **ic2, **rho, **box3)),
        ("d3q19p_ic2_f64", "d3q19p_f64", dict(base3, **ic2, **rho, **dflt)),
        ("d3q19c_ic2_f64", "d3q19c_f64", dict(base3, **ic2, **rho, **box3)),
        ("d3q19s_ic0_f64", "d3q19s_f64", dict(base3, **ic0, **rho)),
        ("d3q19s_ic2_f64", "d3q19s_f64", dict(base3, **ic2, **rho, **box3, rho_sigma=0.6)),
        ("d3q19_ic2_f32", "d3q19_f32", dict(base3, **ic2, **rho, **box3)),
        ("d3q19s_ic2_f32", "d3q19s_f32", dict(base3, **ic2, **rho, **box3, rho_sigma=0.6)),
    ]


def make_init(only=None):
    sys.path.insert(0, os.path.join(ROOT, "lbgpu-prime-dev_b200"))
    sys.path.insert(0, os.path.dirname(HERE))
    import tempfile
    from _host_files import write_params
    os.makedirs(INIT_DIR, exist_ok=True)
    for name, variant, values in init_cases():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "params.in")
            write_params(path, values)
            text = open(path).read()
            f, mv = po.reference_init_from_params(variant, path)
        np.savez_compressed(os.path.join(INIT_DIR, name + ".npz"), params_in=np.array(text),
                            variant=variant, f=f, mv=mv)
        print(name, variant, f.shape, f.dtype)


if __name__ == "__main__":
    args = sys.argv[1:]
    if args and args[0] == "init":
        make_init(args[1:] or None)
    else:
        main(args or None)
