"""Parity of the CUDA 3-D pair counts with the oracle (CPU restatement of
the reference, itself pinned to the reference build and the golden
fixtures).  Unit-weight counts must match bit for bit; weighted sums match to
1e-12 relative (the engine sums the reference's float pair weights exactly in
fixed point; the oracle, like the reference, accumulates them in double)."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from oracle import port

pytestmark = pytest.mark.gpu

WEIGHT_RTOL = 1e-12

AXES = {
    "monopole_log": (tp.MONOPOLE, (0.0, 100.0, 1.3, 30), None),
    "monopole_lin_min": (tp.MONOPOLE, (5.0, 80.0, 1.0, 15), None),
    "s_mu_log": (tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50)),
    "s_mu_lin_min": (tp.S_MU, (3.0, 60.0, 1.0, 19), (0.0, 1.0, 0.0, 7)),
    "sigma_pi_lin": (tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50)),
    "sigma_pi_log": (tp.SIGMA_PI, (0.5, 40.0, 1.4, 12), (0.0, 30.0, 1.0, 10)),
    # second axes the kernel cannot bin directly (a mu axis from above 0, a log pi axis): table 2 and its
    # edge-coded buckets
    "s_mu_mu_min": (tp.S_MU, (0.0, 80.0, 1.3, 20), (0.1, 1.0, 0.0, 9)),
    "sigma_pi_log_pi": (tp.SIGMA_PI, (0.0, 40.0, 1.0, 20), (0.5, 30.0, 1.4, 10)),
}


def oracle_axes(mode, ax1, ax2):
    if mode == tp.MONOPOLE:
        return (ax1[0], ax1[1], ax1[2], ax1[3], 0.0, 0.0, 0.0, 0)
    return (ax1[0], ax1[1], ax1[2], ax1[3], ax2[0], ax2[1], ax2[2], ax2[3])


def make_points(seed, n, box=260.0, offset=300.0, dup=20, faces=20):
    """Clustered points with duplicates and points exactly on lattice faces."""
    rng = np.random.default_rng(seed)
    nc = n // 40
    centres = rng.uniform(0, box, (nc, 3))
    pts = np.repeat(centres, 40, axis=0)[:n] + rng.normal(0, 6.0, (n, 3))
    pts = np.mod(pts, box) + offset
    pts[:dup] = pts[dup:2 * dup]                      # exact duplicates: s^2 = 0, never counted
    pts[2 * dup:2 * dup + faces, 0] = offset + 100.0  # on a face of a side-100 lattice
    rng.shuffle(pts[2 * dup:])
    return pts


def make_cat(seed, n, n_jk, weighted):
    rng = np.random.default_rng(seed + 1000)
    xyz = make_points(seed, n)
    w = rng.lognormal(0, 0.2, n).astype(np.float32) if weighted else None
    jk = rng.integers(0, n_jk, n).astype(np.int32) if n_jk > 1 else None
    return xyz, w, jk


def run_case(ctx, name, n_jk, weighted, is_auto, precision, refinement=0):
    mode, ax1, ax2 = AXES[name]
    x1, w1, j1 = make_cat(11, 3000, n_jk, weighted)
    x2, w2, j2 = make_cat(23, 4000, n_jk, weighted)
    c1 = tp.Catalog(ctx, x1, weight=w1, jk_region=j1, n_jk_regions=n_jk)
    c2 = tp.Catalog(ctx, x2, weight=w2, jk_region=j2, n_jk_regions=n_jk)
    b = tp.Binning(ctx, mode, ax1, ax2, n_jk)
    ctx.set_refinement(refinement)
    if is_auto:
        full, sub, st = tp.auto_pair_count(ctx, c1, b, precision)
    else:
        full, sub, st = tp.cross_pair_count(ctx, c1, c2, b, precision)
    ctx.set_refinement(0)
    o1 = port.Cat(x1, w=w1, jk=j1)
    o2 = port.Cat(x2, w=w2, jk=j2)
    ofull, osub, _ = port.count_3d(mode, o1, None if is_auto else o2, is_auto=is_auto, n_jk=n_jk,
                                   axes=oracle_axes(mode, ax1, ax2))
    return full, sub, ofull, osub, st


def assert_match(full, sub, ofull, osub, weighted):
    if weighted:
        np.testing.assert_allclose(full, ofull, rtol=WEIGHT_RTOL, atol=0)
        np.testing.assert_allclose(sub, osub, rtol=WEIGHT_RTOL, atol=1e-9 * max(1.0, np.abs(ofull).max()))
    else:
        assert np.array_equal(full, ofull), np.flatnonzero(full != ofull)[:10]
        assert np.array_equal(sub, osub)


@pytest.mark.parametrize("name", list(AXES))
@pytest.mark.parametrize("is_auto", [True, False])
@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_unit_weights_no_jk(ctx, name, is_auto, precision):
    full, sub, ofull, osub, st = run_case(ctx, name, 1, False, is_auto, precision)
    assert ofull.sum() > 0
    assert_match(full, sub, ofull, osub, False)


@pytest.mark.parametrize("name", ["monopole_log", "s_mu_log", "sigma_pi_lin"])
@pytest.mark.parametrize("is_auto", [True, False])
@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_weights_and_jackknife(ctx, name, is_auto, precision):
    full, sub, ofull, osub, st = run_case(ctx, name, 7, True, is_auto, precision)
    assert_match(full, sub, ofull, osub, True)


@pytest.mark.parametrize("name", ["s_mu_log", "sigma_pi_lin"])
def test_unit_weights_jackknife_exact(ctx, name):
    for is_auto in (True, False):
        full, sub, ofull, osub, st = run_case(ctx, name, 7, False, is_auto, tp.FP32_GUARD)
        assert_match(full, sub, ofull, osub, False)


@pytest.mark.parametrize("m", [1, 2, 3])
def test_refinement_independent(ctx, m):
    """Any complete cell decomposition gives the same counts."""
    full, sub, ofull, osub, st = run_case(ctx, "s_mu_log", 1, False, True, tp.FP32_GUARD, refinement=m)
    assert_match(full, sub, ofull, osub, False)


def test_stats_consistent(ctx):
    full, sub, ofull, osub, st = run_case(ctx, "monopole_log", 1, False, True, tp.FP32_GUARD)
    # every binned pair is in range; auto counts are reported once, histogram twice
    assert st["in_range"] >= full.sum() / 2
    assert st["candidates"] >= st["in_range"]
    assert st["guard_evals"] < 0.05 * st["in_range"] + 100


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_wide_range_and_negative_weights(ctx, precision):
    """Weights over six decades, some negative (the reference accepts any
    float weight).  Pair weights are summed in fixed point, 64-bit in shared
    memory and 128-bit in global memory, with resolution 2^-(S+1) per pair,
    S = floor(62 - log2(w_max1 w_max2 P)) and P at most the product of the
    catalogue sizes: the sums agree with the oracle's double sums within
    that quantisation (here far above the doubles' own rounding) plus 1e-12
    of the bin's absolute weight."""
    rng = np.random.default_rng(8)
    n_jk = 5
    n1, n2 = 3000, 3600
    x1 = make_points(31, n1)
    x2 = make_points(37, n2)
    w1 = (10.0 ** rng.uniform(-3, 3, n1) * rng.choice([-1.0, 1.0], n1, p=[0.2, 0.8])).astype(np.float32)
    w2 = (10.0 ** rng.uniform(-3, 3, n2)).astype(np.float32)
    j1 = rng.integers(0, n_jk, n1).astype(np.int32)
    j2 = rng.integers(0, n_jk, n2).astype(np.int32)
    mode, ax1, ax2 = AXES["s_mu_log"]
    b = tp.Binning(ctx, mode, ax1, ax2, n_jk)
    c1 = tp.Catalog(ctx, x1, weight=w1, jk_region=j1, n_jk_regions=n_jk)
    c2 = tp.Catalog(ctx, x2, weight=w2, jk_region=j2, n_jk_regions=n_jk)
    a1 = port.Cat(x1, w=np.abs(w1), jk=j1)
    a2 = port.Cat(x2, w=w2, jk=j2)
    for is_auto in (True, False):
        other = w1 if is_auto else w2
        wmax = float(np.abs(w1).max()) * float(np.abs(other).max())
        s_min = int(np.floor(62 - np.log2(wmax * (1 + 1e-6)) - np.log2(n1 * (n1 if is_auto else n2))))
        full, sub, st = tp.count(ctx, c1, None if is_auto else c2, b, precision)
        quant = st["in_range"] * 2.0 ** -(s_min + 1)
        of, os_, _ = port.count_3d(mode, port.Cat(x1, w=w1, jk=j1), None if is_auto else port.Cat(x2, w=w2, jk=j2),
                                   is_auto=is_auto, n_jk=n_jk, axes=oracle_axes(mode, ax1, ax2))
        af, asub, _ = port.count_3d(mode, a1, None if is_auto else a2, is_auto=is_auto, n_jk=n_jk,
                                    axes=oracle_axes(mode, ax1, ax2))
        k = 2.0 if is_auto else 1.0  # the oracle returns the reference's doubled, inverted form
        ref_full = of / k
        ref_sub = (of[None, :] - os_) / k
        scale_full = af / k
        scale_sub = (af[None, :] + np.abs(af[None, :] - asub)) / k
        assert np.all(np.abs(full - ref_full) <= 1e-12 * scale_full + quant)
        assert np.all(np.abs(sub - ref_sub) <= 1e-12 * scale_sub + quant)
        assert np.abs(ref_full).max() > 0
        # quantisation is the only loss: far below the bins' absolute weight
        assert quant < 1e-6 * scale_full.max()
