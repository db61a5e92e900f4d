"""The reference arm of bench.py counts the in-range pairs of its sample by
KD-tree (no part of the engine on that path).  Its count must equal the
reference's range test (src/correlators.cpp:33-40: d = (float)(x1 - x2) per
axis, s^2 = (d0^2 + d1^2) + d2^2 in float, min^2 < s^2 < max^2, auto counts
over unordered pairs), restated here in float32 numpy on a small sample with
a duplicate point (s^2 = 0 is never in range)."""
import numpy as np

import bench
from two_pcf_b200 import synthetic


def float_range_pairs(a, b, max_sq, auto):
    tot = 0
    m = np.float32(max_sq)
    for i0 in range(0, a.shape[0], 500):
        A = a[i0:i0 + 500]
        d = [(A[:, None, q] - b[None, :, q]).astype(np.float32) for q in range(3)]
        s2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]
        ok = (s2 > np.float32(0)) & (s2 < m)
        if auto:
            ok &= np.arange(b.shape[0])[None, :] > np.arange(i0, i0 + A.shape[0])[:, None]
        tot += int(ok.sum())
    return tot


def test_kdtree_tally_matches_the_reference_range_test():
    w = synthetic.survey_catalogue(seed=9, n_data=3000, n_rand=8000)
    cd = {"xyz": w["data"]["xyz"].copy(), "dcom": w["data"]["d_comov"]}
    cr = {"xyz": w["rand"]["xyz"], "dcom": w["rand"]["d_comov"]}
    cd["xyz"][1] = cd["xyz"][0]
    got = bench.in_range_pairs_kdtree(cd, cr)
    xd, xr = cd["xyz"], cr["xyz"]
    sp, sm = bench.SIGMA_PI_AXES, bench.S_MU_AXES
    want = 0
    for max_sq in (sp[0][1] ** 2 + sp[1][1] ** 2, sm[0][1] ** 2):  # sigma-pi: sigma_max^2 + pi_max^2
        want += (float_range_pairs(xd, xd, max_sq, True) + float_range_pairs(xd, xr, max_sq, False)
                 + float_range_pairs(xr, xr, max_sq, True))
    assert got == want and got > 0


def test_gpus_2_launches_two_ranks_and_reduces_exactly():
    """bench.py --gpus 2 started plainly re-launches itself as two ranks
    (torch.distributed.run on 127.0.0.1); without a GPU the ranks exchange
    over gloo.  The exchange of the sharded count (reduce_partials, then
    tpcf_shard_combine) must give both ranks the known totals exactly."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--exchange-selftest"],
                       capture_output=True, text=True, timeout=300, cwd=root, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert line == {"exchange_selftest": True, "n_ranks": 2, "backend": "gloo"}


def test_reference_grid_candidates_brute_force():
    """The reference's candidate set (cells of side r_max on the joint bounding
    box, 27 neighbours; auto counts each unordered pair once) counted by the
    bench's histogram convolution equals a pair-by-pair enumeration."""
    rng = np.random.default_rng(1)
    a = rng.uniform(0, 30, (300, 3))
    b = rng.uniform(0, 30, (500, 3))
    lo, hi = np.minimum(a.min(0), b.min(0)), np.maximum(a.max(0), b.max(0))
    r = 7.0
    top = np.floor((hi - lo) / r).astype(int)

    def cells(x):
        return np.minimum(((x - lo) / r).astype(int), top)
    ca, cb = cells(a), cells(b)
    near_ab = np.all(np.abs(ca[:, None, :] - cb[None, :, :]) <= 1, axis=2)
    near_aa = np.all(np.abs(ca[:, None, :] - ca[None, :, :]) <= 1, axis=2)
    assert bench.reference_grid_candidates(a, b, r, False, lo, hi) == int(near_ab.sum())
    assert bench.reference_grid_candidates(a, None, r, True, lo, hi) == int(np.triu(near_aa, 1).sum())
