"""Sharded counts on the GPU: the partial sums of every shard of a count,
added word by word and combined, give exactly the histograms of one
tpcf_count — weighted sums included (the shards add in the same fixed
point).  The shards run one after another on this GPU; each is an
independent launch."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def survey(ctx):
    w = synthetic.survey_catalogue(seed=12, n_data=15_000, n_rand=45_000)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    U = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"])
    return {"D": D, "R": R, "U": U, "n_jk": w["n_jk"]}


def run_shards(ctx, a, b, binning, n, precision=tp.FP32_GUARD):
    tot = None
    se0 = None
    items = 0
    for k in range(n):
        p, se, st = tp.count_shard(ctx, a, b, binning, k, n, precision)
        items += st["work_items"]
        se0 = se if se0 is None else se0
        assert se == se0
        tot = p if tot is None else tot + p
    return tp.shard_combine(binning, tot, se0), items


@pytest.mark.parametrize("n_shards", [1, 2, 3, 7])
@pytest.mark.parametrize("mode,ax1,ax2", [
    (tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50)),
    (tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50)),
])
def test_shards_sum_to_the_count(ctx, survey, mode, ax1, ax2, n_shards):
    b = tp.Binning(ctx, mode, ax1, ax2, survey["n_jk"])
    D, R = survey["D"], survey["R"]
    for a, bb in ((D, None), (D, R)):
        full, reg, st = tp.count(ctx, a, bb, b)
        (f2, r2), items = run_shards(ctx, a, bb, b, n_shards)
        assert items == st["work_items"]
        assert np.array_equal(f2, full)
        assert np.array_equal(r2, reg)


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_shards_unit_weights_no_regions(ctx, survey, precision):
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 100.0, 1.3, 30))
    U = survey["U"]
    full, reg, _ = tp.count(ctx, U, None, b, precision)
    (f2, r2), _ = run_shards(ctx, U, None, b, 4, precision)
    assert np.array_equal(f2, full)
    assert np.array_equal(r2[0], reg[0])


def test_count_sharded_single_process(ctx, survey):
    b = tp.Binning(ctx, tp.S_MU, (0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 10), survey["n_jk"])
    full, reg, _ = tp.count(ctx, survey["D"], survey["R"], b)
    f2, r2, _ = tp.count_sharded(ctx, survey["D"], survey["R"], b)
    assert np.array_equal(f2, full) and np.array_equal(r2, reg)


def test_bad_shard_index(ctx, survey):
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 50.0, 1.0, 10))
    with pytest.raises(tp.TpcfError):
        tp.count_shard(ctx, survey["U"], None, b, 3, 3)


def _sharded_rank(rank, world, port, q):
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        ctx = tp.Context(0)
        w = synthetic.survey_catalogue(seed=12, n_data=15_000, n_rand=45_000)
        d, r = w["data"], w["rand"]
        D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
        R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
        b = tp.Binning(ctx, tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), w["n_jk"])
        full, reg, st = tp.count_sharded(ctx, D, R, b)
        ref, rreg, st1 = tp.count(ctx, D, R, b)
        q.put((rank, bool(np.array_equal(full, ref) and np.array_equal(reg, rreg)), st["work_items"],
               st1["work_items"]))
    finally:
        dist.destroy_process_group()


def test_count_sharded_two_processes(tmp_path):
    """Two processes (a gloo group on the host), each running its shard on
    this GPU as an independent launch; the all-reduced partials give both
    ranks the whole count."""
    import os
    import torch.multiprocessing as mp
    c = mp.get_context("spawn")
    q = c.Queue()
    port = 29700 + os.getpid() % 200
    procs = [c.Process(target=_sharded_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert all(ok for _, ok, _, _ in res)
    assert res[0][2] + res[1][2] == res[0][3]  # the two shards split the work list
