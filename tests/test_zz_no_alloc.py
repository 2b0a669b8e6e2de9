"""lbx_reduce_mv_static: the reductions for callers that cannot allocate (GPU).

Some host programs cannot let a library call cudaMalloc: their device memory
is handed in full to their own pool allocator, or an allocation (which can
synchronize the whole device, or fail) is not allowed in their time-critical
loop.  lbx_reduce_mv_static takes the macro variables and the mask as device
pointers the caller owns and keeps its scratch in a fixed array inside the
library.  This file checks it against lbx_reduce, the entry point that
allocates its scratch, on two calls in a row.  It is collected last on
purpose, and runs alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import lbx

pytestmark = pytest.mark.gpu

MAX_NODES = 4096 * 16384


def _static_fn():
    lib = lbx.load_library()
    fn = lib.lbx_reduce_mv_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_int,
                   C.c_void_p, C.POINTER(lbx._CReductions)]
    return fn


def _as_dict(r):
    return dict(mass=r.mass, solute_mass=r.solute_mass, momentum=tuple(r.momentum),
                u_sum=tuple(r.u_sum), rho_min=r.rho_min, rho_max=r.rho_max,
                fluid_nodes=r.fluid_nodes, nonfinite=r.nonfinite)


def _close(a, b, rtol=1e-12):
    for k in ("mass", "solute_mass", "rho_min", "rho_max"):
        assert a[k] == pytest.approx(b[k], rel=rtol, abs=1e-300), k
    for k in ("momentum", "u_sum"):
        for x, y in zip(a[k], b[k]):
            assert x == pytest.approx(y, rel=rtol, abs=1e-9), k
    assert a["fluid_nodes"] == b["fluid_nodes"] and a["nonfinite"] == b["nonfinite"]


@pytest.mark.parametrize("dims,nsubs,precision,shape", [
    (3, 1, 4, (40, 36, 32)),
    (3, 2, 8, (33, 20, 24)),
    (2, 1, 8, (256, 256, 1)),
    (3, 1, 4, (96, 96, 96)),
])
def test_static_reduce_matches_allocating_reduce(dims, nsubs, precision, shape):
    torch = pytest.importorskip("torch")
    fn = _static_fn()
    LX, LY, LZ = shape
    N = LX * LY * LZ
    dt = np.float64 if precision == 8 else np.float32
    rng = np.random.default_rng(N)
    sol = rng.choice([0, 1, 255], size=N, p=[0.55, 0.4, 0.05]).astype(np.uint8)
    p = lbx.Params(dims=dims, LX=LX, LY=LY, LZ=LZ, nsubs=nsubs, precision=precision)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):                   # two calls in a row share the scratch
        mv = (rng.random((nsubs, 1 + dims, N)) + 0.5).astype(dt)
        with lbx.Domain(p, sol) as d:
            d.upload_mv(mv)
            want = d.reduce()
        mv_dev = torch.from_numpy(mv).cuda()
        sol_dev = torch.from_numpy(sol).cuda()
        torch.cuda.synchronize()
        r = lbx._CReductions()
        free0 = torch.cuda.mem_get_info()[0]
        rc = fn(mv_dev.data_ptr(), sol_dev.data_ptr(), N, dims, nsubs, precision,
                stream, C.byref(r))
        assert rc == lbx.LBX_OK, lbx._lib.lbx_last_error()
        if call == 1:
            # the first call may load the library's module onto the device;
            # after that a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free0
        _close(_as_dict(r), want)


def test_static_reduce_rejects_oversize_and_bad_args():
    fn = _static_fn()
    r = lbx._CReductions()
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    rc = fn(dummy, dummy, MAX_NODES + 1, 3, 1, 4, None, C.byref(r))
    assert rc == lbx.LBX_ERR_INVALID
    assert b"exceeds" in lbx._lib.lbx_last_error()
    assert fn(None, dummy, 10, 3, 1, 4, None, C.byref(r)) == lbx.LBX_ERR_INVALID
    assert fn(dummy, dummy, 10, 4, 1, 4, None, C.byref(r)) == lbx.LBX_ERR_INVALID
