"""Loading helpers for the committed golden fixtures (tests/golden/*.npz)."""
import glob
import os

import numpy as np

import pyoracle as po

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _is_walsh(name):
    # variant letters follow the lattice name: d3q19sw_f64 = solute + Walsh
    return "w" in name.split("_")[0].replace("d3q19", "").replace("d2q9", "")


def golden_names(walsh=None):
    """All fixtures, or only the Walsh (walsh=True) or non-Walsh ones."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    return [n for n in names if walsh is None or _is_walsh(n) == walsh]


def load(name):
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"), allow_pickle=False)
    p = po.Params()
    for key in z.files:
        if not key.startswith("p_"):
            continue
        k = key[2:]
        v = z[key]
        if k.endswith("_table") or k.startswith("constcon_profile") or k == "ns":
            setattr(p, k, None if v.size == 0 else v.astype(np.float64))
        elif v.ndim == 0:
            setattr(p, k, v.item())
        else:
            setattr(p, k, tuple(v.tolist()))
    return p, z


def rel_err(a, b, mask=None):
    """Norm-wise relative error ||a-b|| / ||b|| (over `mask` if given)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is not None:
        a = a[..., mask]
        b = b[..., mask]
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
