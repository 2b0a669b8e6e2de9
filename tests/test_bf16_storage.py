"""The BF16-storage variant of the FP32 shifted-population path, measured on
the CPU oracle: populations are rounded to bfloat16 (round to nearest even)
every time the state is stored, and the mean u_x (the permeability, up to a
constant) after a few hundred steps is compared with the FP64 run of the same
inputs.  BF16 keeps 8 significand bits, so the shifted deviations lose ~4e-3
relative per store; the measured error (~8e-4 here, while rounding only every
second store) is far above the 1e-5 tolerance of the FP32 path, which is why
the library has no BF16 storage mode.  The FP32 run of the same case stays
below 1e-6."""
import numpy as np

import pyoracle as po
from lbx import geometry


def _bf16(x):
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _mean_ux(p, mask, dtype, round_bf16, steps):
    f = np.zeros((1, 19, p.NN), dtype=dtype)
    mv = None
    for t in range(0, steps, 2):     # the oracle steps in AA pairs
        f, mv = po.run_oracle(p, f, mask, t, 2, 2)
        if round_bf16:
            f[...] = _bf16(f)
    return mv[0, 1][mask != 1].mean()


def test_bf16_storage_misses_the_fp32_tolerance():
    n = 32
    mask = geometry.sphere_pack(n, n, n, 3, 0.45, 7)
    p = po.Params(dims=3, LX=n, LY=n, LZ=n, tau=(0.8, 1.0), gaccel=(1e-5, 0, 0, 0, 0, 0))
    u64 = _mean_ux(p, mask, np.float64, False, 600)
    e32 = abs(_mean_ux(p, mask, np.float32, False, 600) - u64) / abs(u64)
    ebf = abs(_mean_ux(p, mask, np.float32, True, 600) - u64) / abs(u64)
    assert e32 < 1e-6
    assert ebf > 1e-4          # measured 8.4e-4: 84x the 1e-5 tolerance
