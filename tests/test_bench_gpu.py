"""bench.py --gpus 2 on one GPU: two ranks, each counting its shard of every
count of the survey step, the int64 partial sums exchanged over gloo (the
ranks share the device, which NCCL refuses); no kernel of one rank waits on
the other.  The JSON line reports two ranks and the histograms rank 0 writes
equal one unsplit tp.count of the same workload bit for bit."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import two_pcf_b200 as tp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_two_ranks_match_unsplit_counts(ctx, tmp_path):
    sys.path.insert(0, ROOT)
    import bench
    out = tmp_path / "hists.npz"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--scale", "0.01",
                        "--steps", "1", "--warmup", "3", "--no-fp64", "--no-cpu-baseline", "--no-e2e",
                        "--save-hists", str(out)], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["n_gpus"] == 2 and line["scaling"] == "strong"
    assert line["config"]["parallelism"] == "shards2" and line["config"]["exchange"] == "gloo"
    got = np.load(out)
    w = bench.make_workload(2, 0.01)
    d, rr = w["data"], w["rand"]
    n_jk = w["n_jk"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], n_jk)
    R = tp.Catalog(ctx, rr["xyz"], rr["x_norm"], rr["d_comov"], rr["weight"], None, rr["jk"], n_jk)
    for mode, axes, name in ((tp.SIGMA_PI, bench.SIGMA_PI_AXES, "sigma_pi"), (tp.S_MU, bench.S_MU_AXES, "s_mu")):
        b = tp.Binning(ctx, mode, *axes, n_jk)
        for lab, a, bb in (("dd", D, None), ("dr", D, R), ("rr", R, None)):
            full, reg, _ = tp.count(ctx, a, bb, b)
            assert np.array_equal(got[f"{name}_{lab}_full"], full)
            assert np.array_equal(got[f"{name}_{lab}_regions"], reg)
