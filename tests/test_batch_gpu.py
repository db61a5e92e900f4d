"""Batched counts (tpcf_batch_*): DD and DR of several mocks of uneven size
against one shared random catalogue, in one persistent launch replayed as a
CUDA graph, against one tpcf_count per pair.  Unit weights: bit-identical;
weights: 1e-12 (the batch picks one fixed-point scale for all pairs)."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.gpu

BOX = 300.0
AX1, AX2 = (0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 10)


def subcube_jk(xyz, box=BOX, k=3):
    c = np.clip((xyz / (box / k)).astype(int), 0, k - 1)
    return (c[:, 0] * k + c[:, 1]) * k + c[:, 2]


def mocks(seed, sizes, weighted):
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        sigma = rng.uniform(3, 8)
        x = synthetic.neyman_scott_box(rng, n, BOX, max(1, n // 40), 40.0, sigma)
        w = rng.lognormal(0, 0.2, n).astype(np.float32) if weighted else None
        out.append((x, w))
    return out


def catalog(ctx, x, w):
    return tp.Catalog(ctx, x, weight=w, jk_region=subcube_jk(x).astype(np.int32), n_jk_regions=27)


@pytest.mark.parametrize("weighted", [False, True])
def test_batch_matches_single_counts(ctx, weighted):
    sizes = [2000, 7000, 3500, 5200]
    ms = mocks(1, sizes, weighted)
    rng = np.random.default_rng(2)
    xr = rng.uniform(0, BOX, (15000, 3))
    R = catalog(ctx, xr, None)
    M = [catalog(ctx, x, w) for x, w in ms]
    b = tp.Binning(ctx, tp.S_MU, AX1, AX2, 27)
    batch = tp.Batch(ctx, M, R, b, what=tp.BATCH_DD | tp.BATCH_DR)
    assert batch.n_outputs == 2 * len(M)
    for rep in range(2):  # graph replays give the same result
        full, reg, st = batch.run()
        for i, m in enumerate(M):
            for k, other in ((0, None), (1, R)):
                f1, r1, _ = tp.count(ctx, m, other, b)
                if weighted:
                    np.testing.assert_allclose(full[2 * i + k], f1, rtol=1e-12, atol=1e-9)
                    np.testing.assert_allclose(reg[2 * i + k], r1, rtol=1e-12, atol=1e-9)
                else:
                    assert np.array_equal(full[2 * i + k], f1)
                    assert np.array_equal(reg[2 * i + k], r1)
        assert st["in_range"] > 0


def test_batch_autotune_and_dd_only(ctx):
    ms = mocks(3, [3000, 6000], False)
    M = [catalog(ctx, x, w) for x, w in ms]
    b = tp.Binning(ctx, tp.S_MU, AX1, AX2, 27)
    batch = tp.Batch(ctx, M, None, b, what=tp.BATCH_DD, refinement=tp.BATCH_AUTOTUNE)
    assert batch.refinement in (1, 2, 3)
    assert batch.n_outputs == 2
    full, _, _ = batch.run(with_regions=False)
    for i, m in enumerate(M):
        f1, _, _ = tp.count(ctx, m, None, b)
        assert np.array_equal(full[i], f1)


def test_batch_fp64_path(ctx):
    ms = mocks(4, [2500, 4000], False)
    rng = np.random.default_rng(5)
    R = catalog(ctx, rng.uniform(0, BOX, (8000, 3)), None)
    M = [catalog(ctx, x, w) for x, w in ms]
    b = tp.Binning(ctx, tp.SIGMA_PI, (0.0, 40.0, 1.0, 20), (0.0, 40.0, 1.0, 20), 27)
    batch = tp.Batch(ctx, M, R, b, precision=tp.FP64, refinement=2)
    full, reg, _ = batch.run()
    for i, m in enumerate(M):
        for k, other in ((0, None), (1, R)):
            f1, r1, _ = tp.count(ctx, m, other, b, tp.FP32_GUARD)
            assert np.array_equal(full[2 * i + k], f1)
            assert np.array_equal(reg[2 * i + k], r1)


@pytest.mark.parametrize("weighted", [False, True])
def test_batch_matches_oracle(ctx, weighted):
    """The batch's job table straight against the oracle: mocks of uneven
    size, 27 sub-cube regions, every mock's DD and DR in one launch.  The
    oracle returns the reference's convention (delete-one slices, auto counts
    doubled); the batch returns raw sums and the sums touching each region,
    so the oracle's slices are turned back: touching = full - slice."""
    from oracle import port
    ms = mocks(7, [1800, 5200, 3100], weighted)
    rng = np.random.default_rng(8)
    xr = rng.uniform(0, BOX, (9000, 3))
    R = catalog(ctx, xr, None)
    M = [catalog(ctx, x, w) for x, w in ms]
    b = tp.Binning(ctx, tp.S_MU, AX1, AX2, 27)
    full, reg, _ = tp.Batch(ctx, M, R, b, what=tp.BATCH_DD | tp.BATCH_DR).run()
    pr = port.Cat(xr, jk=subcube_jk(xr).astype(np.int32))
    for i, (x, w) in enumerate(ms):
        pm = port.Cat(x, w=w, jk=subcube_jk(x).astype(np.int32))
        for k, other in ((0, None), (1, pr)):
            auto = other is None
            of, osub, _ = port.count_3d(port.S_MU, pm, other, is_auto=auto, n_jk=27, axes=AX1 + AX2)
            scale = 0.5 if auto else 1.0
            want_full = of * scale
            want_reg = (of[None, :] - osub) * scale
            if weighted:
                np.testing.assert_allclose(full[2 * i + k], want_full, rtol=1e-12, atol=1e-9)
                np.testing.assert_allclose(reg[2 * i + k], want_reg, rtol=1e-12, atol=1e-9)
            else:
                assert np.array_equal(full[2 * i + k], want_full)
                assert np.array_equal(reg[2 * i + k], want_reg)
            assert want_full.sum() > 0


def test_batch_autotune_with_dr_orders(ctx):
    """The batch autotuner probes refinements 1-3 and both orders of the DR
    jobs on sampled work items and builds the fastest in full; whatever it
    picks, every output equals one tp.count."""
    ms = mocks(9, [2600, 4800], True)
    rng = np.random.default_rng(10)
    R = catalog(ctx, rng.uniform(0, BOX, (12000, 3)), None)
    M = [catalog(ctx, x, w) for x, w in ms]
    b = tp.Binning(ctx, tp.S_MU, AX1, AX2, 27)
    batch = tp.Batch(ctx, M, R, b, what=tp.BATCH_DD | tp.BATCH_DR, refinement=tp.BATCH_AUTOTUNE)
    assert batch.refinement in (1, 2, 3) and batch.order in (0, 1)
    full, reg, _ = batch.run()
    for i, m in enumerate(M):
        for k, other in ((0, None), (1, R)):
            f1, r1, _ = tp.count(ctx, m, other, b)
            np.testing.assert_allclose(full[2 * i + k], f1, rtol=1e-12, atol=1e-9)
            np.testing.assert_allclose(reg[2 * i + k], r1, rtol=1e-12, atol=1e-9)
