"""Sharded counts, host side: partial sums (four 32-bit limbs of a 128-bit
fixed-point sum plus non-finite counters per slot) added over shards and
turned into doubles by tpcf_shard_combine, against exact Python integer
arithmetic; and the same reduction across two gloo ranks on CPU."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import two_pcf_b200 as tp
from two_pcf_b200 import _capi

W = _capi.PARTIAL_WORDS
M128 = (1 << 128) - 1


def limbs(v):
    u = v & M128
    return [(u >> (32 * k)) & 0xffffffff for k in range(4)]


def synthetic(seed, n_slots, n_shards, scale_exp):
    """Shard partials whose sums are known totals (signed, |t| < 2^124)."""
    rng = np.random.default_rng(seed)
    totals = [int(rng.integers(-2**62, 2**62)) << int(rng.integers(0, 63)) for _ in range(n_slots)]
    parts = np.zeros((n_shards, n_slots, W), np.int64)
    for s, t in enumerate(totals):
        vals = [int(rng.integers(0, 2**63)) << int(rng.integers(0, 64)) for _ in range(n_shards - 1)]
        vals.append(t - sum(vals))
        for k, v in enumerate(vals):
            parts[k, s, :4] = limbs(v)
    expected = np.array([float(t) * 2.0 ** -scale_exp for t in totals])
    return parts, expected


@pytest.mark.parametrize("n_shards", [1, 2, 5, 64])
def test_combine_exact(n_shards):
    b = tp.Binning(None, tp.S_MU, (0.0, 100.0, 1.3, 8), (0.0, 1.0, 0.0, 5), 3)
    n_slots = 4 * b.nb
    se = 37
    parts, expected = synthetic(n_shards, n_slots, n_shards, se)
    full, reg = tp.shard_combine(b, parts.sum(0), se)
    assert np.array_equal(full, expected[:b.nb])
    assert np.array_equal(reg.ravel(), expected[b.nb:])


def test_combine_nonfinite_markers():
    b = tp.Binning(None, tp.MONOPOLE, (0.0, 10.0, 1.0, 4), None, 1)
    p = np.zeros((2 * b.nb, W), np.int64)
    p[0, 4] = 1            # NaN met
    p[1, 5] = 2            # +inf only
    p[2, 6] = 1            # -inf only
    p[3, 5] = p[3, 6] = 1  # both infinities: NaN
    p[4, 0] = 5            # finite region slot
    full, reg = tp.shard_combine(b, p, 0)
    assert np.isnan(full[0]) and np.signbit(full[0])
    assert full[1] == np.inf and full[2] == -np.inf and np.isnan(full[3])
    assert reg[0, 0] == 5.0


def _rank(rank, world, port, n_slots, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = tp.Binning(None, tp.SIGMA_PI, (0.0, 40.0, 1.0, 6), (0.0, 40.0, 1.0, 6), 2)
        parts, expected = synthetic(7, 3 * b.nb, world, 20)
        t = torch.from_numpy(parts[rank].copy())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        full, reg = tp.shard_combine(b, t.numpy(), 20)
        ok = np.array_equal(np.concatenate([full, reg.ravel()]), expected)
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_partials():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, 0, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: True, 1: True}
