"""The C-ABI library loads and exports every declared symbol (CPU only)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import lbx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "lbx.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbx_[a-z_]+)\s*\(", text)))


def test_library_built():
    assert os.path.exists(lbx.LIB_PATH), "run make -C lbgpu-prime-dev_b200"


def test_exports_every_declared_symbol():
    lib = C.CDLL(lbx.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(lbx.exported_symbols()) == syms


def test_library_is_sm100a_only():
    blob = open(lbx.LIB_PATH, "rb").read()
    assert b"sm_100a" in blob


def test_params_default_matches_reference_defaults():
    lib = lbx.load_library()
    cp = lbx._CParams()
    lib.lbx_params_default(C.byref(cp))
    assert cp.precision == 8 and cp.accurate == 1 and cp.compressible == 0
    assert cp.tau[0] == 1.0 and cp.rho_A[0] == 1.0
    assert cp.bc_ramp_start == -1 and cp.sigma_t_off == -1


@pytest.mark.parametrize("bad", [
    dict(dims=4), dict(LX=0), dict(dims=2, LZ=3), dict(nsubs=3),
    dict(precision=2), dict(accurate=0, compressible=0), dict(tau=(0.5, 1.0)),
    dict(dims=3, pressure_s_in=(1, 0)),
    dict(dims=2, LZ=1, LY=2, pressure_s_in=(1, 0)),
    dict(dims=2, LZ=1, pressure_n_in=(2, 0)),
    dict(walsh=1, pressure_t_in=(1, 0)),
    dict(dims=2, LZ=1, walsh=1, pressure_s_in=(1, 0)),
    dict(walsh=1, layout=lbx.LBX_LAYOUT_COMPACT),
])
def test_create_validates_before_touching_the_device(bad):
    kw = dict(dims=3, LX=4, LY=4, LZ=4)
    kw.update(bad)
    p = lbx.Params(**kw)
    with pytest.raises(lbx.LbxError) as ei:
        lbx.Domain(p, np.zeros(max(p.NN, 1), np.uint8)[:p.NN] if p.NN > 0 else np.zeros(0, np.uint8))
    assert ei.value.code == lbx.LBX_ERR_INVALID
    assert lbx._lib.lbx_last_error()
