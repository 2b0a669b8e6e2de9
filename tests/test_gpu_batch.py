"""Batched lattices (GPU): every sample of a batch must evolve exactly as the
same lattice run alone, in every batch mode."""
import numpy as np
import pytest

import lbx
import pyoracle as po
from lbx import geometry
from lbx.batch import Batch
from _golden import rel_err

pytestmark = pytest.mark.gpu


def make_samples(n, seed, prec=4, sizes=(12, 30)):
    rng = np.random.default_rng(seed)
    params, masks = [], []
    for i in range(n):
        L = [int(x) for x in rng.integers(sizes[0], sizes[1], size=3)]
        tau = float(rng.uniform(0.6, 1.2))
        por = float(rng.uniform(0.3, 0.7))
        r = int(rng.integers(2, 5))
        masks.append(geometry.sphere_pack(L[0], L[1], L[2], r, por, seed * 1000 + i))
        params.append(lbx.Params(dims=3, LX=L[0], LY=L[1], LZ=L[2], precision=prec,
                                 tau=(tau, 1.0), gaccel=(1e-5, 0, 0, 0, 0, 0)))
    return params, masks


@pytest.mark.parametrize("mode", ["fused", "persistent", "sequential"])
@pytest.mark.parametrize("prec", [8, 4])
def test_batch_matches_oracle_per_sample(mode, prec):
    params, masks = make_samples(7, seed=3, prec=prec)
    rng = np.random.default_rng(1)
    f0 = [(rng.standard_normal((19, p.NN)) * 1e-4).astype(p.dtype) for p in params]
    with Batch(params, masks) as b:
        for i in range(len(params)):
            b.upload_f(i, f0[i])
        b.run(0, 23, 23, mode=mode)
        b.sync()
        out = [(b.download_f(i), b.download_mv(i)) for i in range(len(params))]
    tol = 1e-12 if prec == 8 else 1e-5
    for i, p in enumerate(params):
        q = po.Params(dims=3, LX=p.LX, LY=p.LY, LZ=p.LZ, tau=tuple(p.tau),
                      gaccel=tuple(p.gaccel))
        fo, mvo = po.run_oracle(q, f0[i].reshape(1, 19, -1).copy(), masks[i], 0, 23, 23)
        fl = masks[i] != 1
        assert rel_err(out[i][0], fo[0]) <= tol, (i, rel_err(out[i][0], fo[0]))
        for c in range(4):
            e = rel_err(out[i][1][c], mvo[0, c], fl)
            assert e <= (tol if prec == 8 else 2e-5), (i, c, e)


def test_batch_autotune_keeps_state_and_picks_a_mode():
    params, masks = make_samples(5, seed=9, prec=4)
    with Batch(params, masks) as b:
        for i in range(5):
            b.init_equilibrium(i, 1.0)
        before = [b.download_f(i) for i in range(5)]
        mode, bs = b.autotune(4)
        assert mode in ("fused", "persistent") and bs in (128, 256)
        after = [b.download_f(i) for i in range(5)]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
        b.run(0, 10, 10)
        r = b.reduce(0)
        assert r["fluid_nodes"] == int((masks[0] != 1).sum())


def _check_against_oracle(params, masks, f0, out, steps, tol=1e-12):
    for i, p in enumerate(params):
        q = po.Params(dims=3, LX=p.LX, LY=p.LY, LZ=p.LZ, tau=tuple(p.tau),
                      gaccel=tuple(p.gaccel))
        fo, mvo = po.run_oracle(q, f0[i].reshape(1, 19, -1).copy(), masks[i], 0, steps, steps,
                                threads=1)
        assert rel_err(out[i][0], fo[0]) <= tol, (i, rel_err(out[i][0], fo[0]))
        fl = masks[i] != 1
        if fl.any():
            assert rel_err(out[i][1][0], mvo[0, 0], fl) <= tol, i


def _run_batch(b, params, f0, steps, mode="fused"):
    for i in range(len(params)):
        b.upload_f(i, f0[i])
    b.run(0, steps, steps, mode=mode)
    b.sync()
    return [(b.download_f(i), b.download_mv(i)) for i in range(len(params))]


@pytest.mark.parametrize("mode", ["fused", "sequential"])
def test_batch_beyond_the_descriptor_pool(mode):
    """600 FP64 samples: their descriptors (112 bytes each) do not fit the
    constant-memory pool (63 KB), so the batch reads them from its per-block
    table in global memory.  Every sample still evolves as the oracle's run
    of it alone, empty and all-fluid samples included."""
    params, masks = make_samples(600, seed=21, prec=8, sizes=(3, 8))
    masks[5][:] = 1                       # a sample without fluid nodes
    masks[9][:] = 0                       # an all-fluid sample
    rng = np.random.default_rng(4)
    f0 = [rng.standard_normal((19, p.NN)) * 1e-4 for p in params]
    with Batch(params, masks) as b:
        out = _run_batch(b, params, f0, 11, mode)
    _check_against_oracle(params, masks, f0, out, 11)


def test_batches_alive_together_keep_their_own_descriptors():
    """Batches alive at the same time hold disjoint ranges of the descriptor
    pool; a destroyed batch's range goes to the next batch that fits it, and
    the batch created in between keeps its own."""
    pa, ma = make_samples(5, seed=31, prec=8)
    pb, mb = make_samples(4, seed=32, prec=8)
    pc, mc = make_samples(3, seed=33, prec=8)
    rng = np.random.default_rng(5)
    fa, fb, fc = ([rng.standard_normal((19, p.NN)) * 1e-4 for p in ps] for ps in (pa, pb, pc))
    ba = Batch(pa, ma)
    with Batch(pb, mb) as bb:
        out_a = _run_batch(ba, pa, fa, 13)
        ba.close()
        with Batch(pc, mc) as bc:
            out_b = _run_batch(bb, pb, fb, 13)
            out_c = _run_batch(bc, pc, fc, 13)
    _check_against_oracle(pa, ma, fa, out_a, 13)
    _check_against_oracle(pb, mb, fb, out_b, 13)
    _check_against_oracle(pc, mc, fc, out_c, 13)


@pytest.mark.parametrize("prec", [8, 4])
def test_batch_layouts_give_the_same_results(prec):
    """The three sample orders of the compact array (largest first,
    interleaved, as given) give the same populations, and switching the
    order mid-run keeps the state; FP64 matches the oracle."""
    params, masks = make_samples(9, seed=41, prec=prec)
    rng = np.random.default_rng(6)
    f0 = [(rng.standard_normal((19, p.NN)) * 1e-4).astype(p.dtype) for p in params]
    out = {}
    for layout in ("largest_first", "interleaved", "given"):
        with Batch(params, masks) as b:
            b.set_layout(layout)
            assert b.layout() == layout
            for i in range(len(params)):
                b.upload_f(i, f0[i])
            b.run(0, 10, 0, mode="fused")
            b.set_layout("given" if layout != "given" else "interleaved")
            b.run(10, 12, 0, mode="fused")
            b.sync()
            out[layout] = [b.download_f(i) for i in range(len(params))]
    for layout in ("interleaved", "given"):
        for i in range(len(params)):
            if prec == 8:
                assert np.array_equal(out[layout][i], out["largest_first"][i]), (layout, i)
            else:
                assert rel_err(out[layout][i], out["largest_first"][i]) <= 1e-6, (layout, i)
    if prec == 8:
        for i, p in enumerate(params):
            q = po.Params(dims=3, LX=p.LX, LY=p.LY, LZ=p.LZ, tau=tuple(p.tau),
                          gaccel=tuple(p.gaccel))
            fo, _ = po.run_oracle(q, f0[i].reshape(1, 19, -1).copy(), masks[i], 0, 22, 0,
                                  threads=1)
            assert rel_err(out["given"][i], fo[0]) <= 1e-12, i


def test_batch_autotune_over_layouts_keeps_state():
    params, masks = make_samples(6, seed=43, prec=4)
    with Batch(params, masks) as b:
        for i in range(6):
            b.init_equilibrium(i, 1.0)
        b.run(0, 6, 0)
        before = [b.download_f(i) for i in range(6)]
        mode, bs = b.autotune(4)
        assert b.layout() in ("largest_first", "interleaved", "given")
        after = [b.download_f(i) for i in range(6)]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)


def _samples_2d(n, seed):
    rng = np.random.default_rng(seed)
    params, masks = [], []
    for i in range(n):
        LX, LY = (int(x) for x in rng.integers(16, 80, size=2))
        tau = float(rng.uniform(0.6, 1.2))
        masks.append(geometry.transpose_2d(
            geometry.disc_pack(LY, LX, radius=3, porosity=float(rng.uniform(0.4, 0.8)),
                               seed=seed * 100 + i), LY, LX))
        params.append(lbx.Params(dims=2, LX=LX, LY=LY, LZ=1, precision=8, tau=(tau, 1.0),
                                 gaccel=(1e-5, -2e-6, 0, 0, 0, 0)))
    return params, masks


@pytest.mark.parametrize("mode", ["fused", "persistent", "sequential"])
def test_batch_d2q9_matches_oracle(mode):
    """A batch of D2Q9 FP64 samples (uneven extents, discs): every sample
    evolves as the oracle's run of it alone."""
    params, masks = _samples_2d(7, seed=51)
    rng = np.random.default_rng(2)
    f0 = [rng.standard_normal((9, p.NN)) * 1e-4 for p in params]
    with Batch(params, masks) as b:
        for i in range(len(params)):
            b.upload_f(i, f0[i])
        b.run(0, 21, 21, mode=mode)
        b.sync()
        out = [(b.download_f(i), b.download_mv(i)) for i in range(len(params))]
    for i, p in enumerate(params):
        q = po.Params(dims=2, LX=p.LX, LY=p.LY, LZ=1, tau=tuple(p.tau), gaccel=tuple(p.gaccel))
        fo, mvo = po.run_oracle(q, f0[i].reshape(1, 9, -1).copy(), masks[i], 0, 21, 21,
                                threads=1)
        assert rel_err(out[i][0], fo[0]) <= 1e-12, i
        fl = masks[i] != 1
        for c in range(3):
            assert rel_err(out[i][1][c], mvo[0, c], fl) <= 1e-12, (i, c)


@pytest.mark.parametrize("model,kahan", [((0, 1), 0), ((1, 1), 0), ((1, 0), 1)])
def test_batch_models_match_oracle(model, kahan):
    """Plain compressible, shifted compressible and Kahan-summed batches
    (FP64) against the oracle."""
    acc, comp = model
    params, masks = make_samples(5, seed=61, prec=8)
    for p in params:
        p.accurate, p.compressible, p.kahan = acc, comp, kahan
    rng = np.random.default_rng(3)
    w = np.array([1 / 3] + [1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] * 2 + [1 / 36] * 8)
    f0 = []
    for p in params:
        noise = rng.standard_normal((19, p.NN)) * 1e-4
        f0.append(w[:, None] * (1.0 + noise) if not acc else noise)
    with Batch(params, masks) as b:
        for i in range(len(params)):
            b.upload_f(i, f0[i])
        b.run(0, 17, 17, mode="fused")
        b.sync()
        out = [b.download_f(i) for i in range(len(params))]
    for i, p in enumerate(params):
        q = po.Params(dims=3, LX=p.LX, LY=p.LY, LZ=p.LZ, tau=tuple(p.tau),
                      gaccel=tuple(p.gaccel), accurate=acc, compressible=comp, kahan=kahan)
        fo, _ = po.run_oracle(q, f0[i].reshape(1, 19, -1).copy(), masks[i], 0, 17, 17,
                              threads=1)
        assert np.isfinite(out[i]).all()
        assert rel_err(out[i], fo[0]) <= 1e-12, i
