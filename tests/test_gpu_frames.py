"""Frame statistics and the asynchronous frame pipeline on the GPU.

lbx_frame_stats_compute against the oracle's restatement of the reference's
compute_* functions (max/min exact, means within 1e-13 relative), and
lbx_frame_enqueue / lbx_frame_wait: every frame returned equals the state at
its own time even though the steps after it (which overwrite the macro
variables) were queued before the wait.
"""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from _golden import rel_err

pytestmark = pytest.mark.gpu


def check_stats(got, want):
    assert got["nodes"] == want["nodes"]
    for k in ("max_rho", "min_rho", "max_u", "min_u"):
        assert np.array_equal(np.atleast_1d(got[k]), np.atleast_1d(want[k])), k
    # means: FP64 sums in different orders, so within 1e-13 of the largest
    # magnitude summed
    for k, m in (("ave_rho", "max_rho"), ("ave_u", "max_u")):
        g, w = np.atleast_1d(got[k]), np.atleast_1d(want[k])
        assert np.all(np.abs(g - w) <= 1e-13 * (np.abs(w) + np.atleast_1d(want[m]))), k


@pytest.mark.parametrize("dims,prec,nsubs", [(3, 4, 1), (3, 8, 2), (2, 8, 1)])
def test_gpu_frame_stats_match_oracle(dims, prec, nsubs):
    LX, LY, LZ = (40, 36, 30) if dims == 3 else (96, 80, 1)
    p = lbx.Params(dims=dims, LX=LX, LY=LY, LZ=LZ, nsubs=nsubs, precision=prec)
    rng = np.random.default_rng(61)
    mask = rng.choice([0, 1, 255], size=p.NN, p=[0.7, 0.2, 0.1]).astype(np.uint8)
    mv = (rng.standard_normal((nsubs, 1 + dims, p.NN)) * 1e-3).astype(p.dtype)
    mv[:, 0] += 1
    with lbx.Domain(p, mask) as d:
        d.upload_mv(mv)
        for s in range(nsubs):
            check_stats(d.frame_stats(s), po.frame_stats(mv[s], mask, dims))


def test_gpu_frame_pipeline_returns_each_frame_state():
    n = 48
    p = po.Params(dims=3, LX=n, LY=n, LZ=n, tau=(0.8, 1.0), gaccel=(1e-5, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(n, n, n, radius=5, porosity=0.5, seed=3)
    f0 = (np.random.default_rng(4).standard_normal((1, 19, p.NN)) * 1e-4).astype(np.float32)
    lp = lbx.Params(dims=3, LX=n, LY=n, LZ=n, precision=4, tau=(0.8, 1.0),
                    gaccel=(1e-5, 0, 0, 0, 0, 0))
    fr = 8
    got = []
    with lbx.Domain(lp, sol) as d:
        d.upload_f(f0)
        d.run(0, fr, fr)
        d.frame_enqueue(fr)
        for k in range(2, 6):
            d.run((k - 1) * fr, fr, fr)          # queued before the wait
            d.frame_enqueue(k * fr)
            got.append(d.frame_wait())
        got.append(d.frame_wait())
        with pytest.raises(lbx.LbxError) as ei:
            d.frame_wait()
        assert ei.value.code == lbx.LBX_ERR_STATE
        d.frame_enqueue(99)
        d.frame_enqueue(99)
        with pytest.raises(lbx.LbxError) as ei:
            d.frame_enqueue(99)
        assert ei.value.code == lbx.LBX_ERR_STATE
    f = f0.copy()
    mv = None
    for k in range(1, 6):
        f, mv = po.run_oracle(p, f, sol, (k - 1) * fr, fr, fr, mv=mv)
        g = got[k - 1]
        assert g["time"] == k * fr
        fluid = sol != 1
        for c in range(4):
            assert rel_err(g["mv"][0, c][fluid], mv[0, c][fluid]) <= 1e-5, (k, c)
        check_stats(g["stats"][0], po.frame_stats(g["mv"][0], sol, 3))


def test_gpu_frame_view_survives_the_next_enqueue():
    """A frame returned with copy=False while a second frame is outstanding
    keeps its values through the next enqueue (the header promises them
    until the second enqueue after the wait)."""
    n = 32
    lp = lbx.Params(dims=3, LX=n, LY=n, LZ=n, precision=4, tau=(0.8, 1.0),
                    gaccel=(1e-5, 0, 0, 0, 0, 0))
    sol = geometry.sphere_pack(n, n, n, radius=4, porosity=0.5, seed=9)
    f0 = (np.random.default_rng(5).standard_normal((1, 19, lp.NN)) * 1e-4).astype(np.float32)
    fr = 4
    with lbx.Domain(lp, sol) as d:
        d.upload_f(f0)
        d.run(0, fr, fr)
        d.frame_enqueue(fr)                       # A
        d.run(fr, fr, fr)
        d.frame_enqueue(2 * fr)                   # B: two outstanding
        a = d.frame_wait(copy=False)
        a_copy = a["mv"].copy()
        d.run(2 * fr, fr, fr)
        d.frame_enqueue(3 * fr)                   # C: the first enqueue after A's wait
        b = d.frame_wait(copy=True)
        c = d.frame_wait(copy=False)              # C's host copy has landed
        assert (a["time"], b["time"], c["time"]) == (fr, 2 * fr, 3 * fr)
        assert np.array_equal(a["mv"], a_copy)
        assert not np.array_equal(b["mv"], a_copy)
        assert not np.array_equal(c["mv"], a_copy)
