#!/usr/bin/env python
"""Benchmark of the grid-binned pair-counting hot path on B200.

Workload (one "step"): the equatorial survey-slab configuration — 1M
clustered data objects and 5M randoms (ra in [0, 60] deg, dec in
[-10, 10] deg, z ~ N(0.3, 0.08) on [0.1, 0.5], flat LCDM Omega_m = 0.25),
lognormal(0, 0.2) weights, 100 jackknife regions on a 10 x 10 ra/dec grid —
counted as the reference's driver does it (src/main.cpp:63-70): sigma-pi
(50 x 50 linear bins over 0-50 Mpc/h) DD, DR and RR, then s-mu (40 log bins,
base 1.3, 0-100 Mpc/h, x 50 mu bins) DD, DR and RR.  Each step rebuilds the
cell grids (the GalaxyBoxes stage) from the resident catalogues.

Metric: in-range pairs per second (pairs passing the reference's float range
test, auto pairs counted once) on the FP32+guard path, with the plain FP64
path run on the same step for comparison and bit-exactness of the two
paths' histograms checked.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--scale f]

With --gpus N > 1 (started plainly, bench.py re-launches itself under
torch.distributed.run with N ranks; under torchrun it uses the ranks it is
given) one workload is split over the ranks: every count runs its share of
the work items on each rank's GPU and one all-reduce of the exact int64
partial sums -- NCCL when every rank has its own GPU, gloo when ranks share
one -- gives every rank the histograms of the whole count (strong scaling).
--replicas runs one seeded copy of the workload per rank instead (weak
scaling, no exchange).  The step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "in-range pairs/sec, FP32+guard vs FP64 GPU path at bit-exact counts"
UNIT = "pairs/s"
SIGMA_PI_AXES = ((0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50))
S_MU_AXES = ((0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50))
F_MODE = {1: 16, 2: 13, 0: 0}   # FP32 flops per in-range pair beyond the 8 of s^2
TRAFFIC_SMU_RR = 21.254e9   # DRAM bytes (read + write) of one full-size s-mu RR launch (ncu, see profiles/)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--scale", type=float, default=1.0, help="fraction of the catalogue sizes (quick runs)")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--strong", action="store_true",
                   help="with --gpus N > 1: one workload, every count split over the ranks (the default)")
    p.add_argument("--replicas", action="store_true",
                   help="with --gpus N > 1: one seeded workload replica per rank, no exchange (weak scaling)")
    p.add_argument("--gloo", action="store_true", help="exchange over gloo on the host even with a GPU per rank")
    p.add_argument("--no-autotune", action="store_true",
                   help="the refinement rule and default kernel configuration instead of the count autotuner "
                        "(the warm-up steps absorb the autotuner's probes)")
    p.add_argument("--save-hists", default=None,
                   help="rank 0 writes the last FP32+guard step's histograms (full, regions per count) to this .npz")
    p.add_argument("--exchange-selftest", action="store_true",
                   help="launcher check without a GPU: the ranks reduce known partial sums through the sharded "
                        "count's exchange and rank 0 prints whether every rank combined them exactly")
    p.add_argument("--refinement", type=int, default=0,
                   help="--one-count: cells per maximum separation (1-3; 0 = the engine's rule)")
    p.add_argument("--one-count", choices=["s_mu", "sigma_pi"], default=None,
                   help="profiling case: one RR count of the workload's randoms at --scale, then exit")
    p.add_argument("--workload", choices=["survey", "mocks", "invp", "adjoint"], default="survey",
                   help="survey: the headline line (default); mocks / invp / adjoint: one JSON line for the "
                        "batched-mocks, inverse-p angular and weight-gradient workloads at --scale (1 GPU)")
    return p.parse_args()


def one_count(args):
    """A single FP32+guard RR count (weighted, jackknife) of the step's
    randoms: the case the committed ncu summaries profile."""
    import two_pcf_b200 as tp
    w = make_workload(2, args.scale)
    r = w["rand"]
    ctx = tp.Context(0)
    if args.refinement:
        ctx.set_refinement(args.refinement)
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    axes = S_MU_AXES if args.one_count == "s_mu" else SIGMA_PI_AXES
    b = tp.Binning(ctx, tp.S_MU if args.one_count == "s_mu" else tp.SIGMA_PI, *axes, w["n_jk"])
    full, _, st = tp.count(ctx, R, None, b, tp.FP32_GUARD)
    print(json.dumps({"one_count": args.one_count, "scale": args.scale, **st}))


def other_workload(args):
    """The other survey workloads on one GPU, each one JSON line (FP32+guard
    path, device time from CUDA events, median of --steps after --warmup):

    mocks   -- 64 Neyman-Scott mocks in a 1000 Mpc/h box (sizes uniform on
               [200k, 2M] x scale, cluster sigma uniform on [3, 8]), one shared
               uniform random catalogue of 10M x scale, 27 sub-cube regions,
               s-mu 40 log (1.3, 0-150) x 50: every mock's DD and DR in one
               batched launch (graph replay, autotuned refinement), RR once;
    invp    -- 500k x scale data on the survey footprint with 32 bitwise masks
               (2048 runs, p uniform on [0.3, 1]) and 2M x scale randoms:
               angular DD, DD-inverse-p, DR, DR-inverse-p (40 log bins, base
               1.6, theta < 0.175 rad), then the 3-D s-mu inverse-p DD and DR
               with the up-weights from those histograms;
    adjoint -- the weight-gradient workload on the survey slab at scale:
               weights w = exp(theta . f) with 8 standardised smooth random
               Fourier fields f over ra/dec and theta ~ N(0, 0.05); loss =
               sum over s-mu bins of (xi - xi_target)^2, xi_target from an
               independent clustered catalogue of the same footprint with unit
               weights.  Forward: s-mu DD, DR, RR; backward: dL/d(histogram)
               from the normalisation and Landy-Szalay chain, then the adjoint
               (per-point dL/dw) of the three counts and dL/dtheta.

    Every line carries the clock record of its timed region."""
    import two_pcf_b200 as tp
    from two_pcf_b200 import synthetic
    ctx = tp.Context(0)
    ctx.set_autotune(not args.no_autotune)   # the warm-up steps absorb the probes
    scale = args.scale
    rng = np.random.default_rng(11)

    def median_ms(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        ms, out = [], None
        for _ in range(max(1, args.steps)):
            out = fn()
            ms.append(out[0])
        return statistics.median(ms), out

    line = {"workload": args.workload, "scale": scale, "unit": UNIT, "dtype": "f32", "data": "synthetic"}
    clk = ClockSampler(0)
    clk.__enter__()
    if args.workload == "mocks":
        box, n_mocks = 1000.0, 64

        def cat(x):
            c = np.clip((x / (box / 3)).astype(int), 0, 2)
            return tp.Catalog(ctx, x, jk_region=((c[:, 0] * 3 + c[:, 1]) * 3 + c[:, 2]).astype(np.int32),
                              n_jk_regions=27)
        sizes = rng.integers(int(200_000 * scale), int(2_000_000 * scale) + 1, n_mocks)
        M = [cat(synthetic.neyman_scott_box(rng, int(n), box, max(1, int(n) // 50), 50.0, rng.uniform(3, 8)))
             for n in sizes]
        R = cat(rng.uniform(0.0, box, (int(10_000_000 * scale), 3)))
        b = tp.Binning(ctx, tp.S_MU, (0.0, 150.0, 1.3, 40), (0.0, 1.0, 0.0, 50), 27)
        batch = tp.Batch(ctx, M, R, b, what=tp.BATCH_DD | tp.BATCH_DR, refinement=tp.BATCH_AUTOTUNE)

        def run_batch():
            _, _, st = batch.run()
            return st["ms_kernel"], st
        ms_b, (_, st_b) = median_ms(run_batch)

        def run_rr():
            _, _, st = tp.count(ctx, R, None, b)
            return st["ms_kernel"], st
        ms_r, (_, st_r) = median_ms(run_rr)
        pairs = st_b["in_range"] + st_r["in_range"]
        line.update({"metric": "in-range pairs/sec, 64 mocks DD+DR in one batched launch + shared RR",
                     "value": pairs / ((ms_b + ms_r) * 1e-3), "ms": ms_b + ms_r, "batch_ms": ms_b, "rr_ms": ms_r,
                     "batch_pairs": st_b["in_range"], "rr_pairs": st_r["in_range"], "mock_points": int(sizes.sum()),
                     "random_points": int(10_000_000 * scale), "refinement": batch.refinement,
                     "dr_order": batch.order,
                     "batch_work_items": st_b["work_items"]})
    elif args.workload == "invp":
        w = synthetic.survey_catalogue(seed=4, n_data=int(500_000 * scale), n_rand=int(2_000_000 * scale))
        d, r = w["data"], w["rand"]
        n_runs = 2048
        md = synthetic.bitwise_masks(5, d["xyz"].shape[0], n_runs=n_runs)
        mr = synthetic.bitwise_masks(6, r["xyz"].shape[0], n_runs=n_runs, all_set=True)
        wd, iwd = tp.iip_weights(md, d["weight"], n_runs)
        wr, iwr = tp.iip_weights(mr, r["weight"], n_runs)
        D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], wd, iwd, d["jk"], w["n_jk"], md)
        R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], wr, iwr, r["jk"], w["n_jk"], mr)
        t_ax = (0.0, 1.0 - np.cos(0.175), 1.6, 40)
        ba = tp.Binning(ctx, tp.ANGULAR, t_ax, None, w["n_jk"])
        ang_jobs = [("DD", D, None, None), ("DD_invp", D, None, tp.Weights(tp.WEIGHTS_INVP_DD, n_runs)),
                    ("DR", D, R, None), ("DR_invp", D, R, tp.Weights(tp.WEIGHTS_INVP_DR))]

        def run_ang():
            out = [tp.pair_count_weighted(ctx, a, bb, ba, wt) for _, a, bb, wt in ang_jobs]
            return sum(o[2]["ms_kernel"] for o in out), out
        ms_a, (_, ang) = median_ms(run_ang)
        bs = tp.Binning(ctx, tp.S_MU, *S_MU_AXES, w["n_jk"])
        w_dd = tp.Weights(tp.WEIGHTS_INVP_DD, n_runs, t_ax, ang[0][0], ang[1][0])
        w_dr = tp.Weights(tp.WEIGHTS_INVP_DR, n_runs, t_ax, ang[2][0], ang[3][0])

        def run_3d():
            out = [tp.pair_count_weighted(ctx, D, None, bs, w_dd), tp.pair_count_weighted(ctx, D, R, bs, w_dr)]
            return sum(o[2]["ms_kernel"] for o in out), out
        ms_3, (_, td) = median_ms(run_3d)
        pa = sum(o[2]["in_range"] for o in ang)
        p3 = sum(o[2]["in_range"] for o in td)
        line.update({"metric": "in-range pairs/sec, inverse-p angular stage + 3-D s-mu inverse-p DD and DR",
                     "value": (pa + p3) / ((ms_a + ms_3) * 1e-3), "ms": ms_a + ms_3,
                     "angular_ms": ms_a, "angular_pairs": pa, "angular_value": pa / (ms_a * 1e-3),
                     "angular_ms_each": {n: o[2]["ms_kernel"] for (n, _, _, _), o in zip(ang_jobs, ang)},
                     "s_mu_ms": ms_3, "s_mu_pairs": p3, "n_data": int(d["xyz"].shape[0]),
                     "n_rand": int(r["xyz"].shape[0]), "mask_words": 32, "n_bitwise_runs": n_runs})
    else:
        w = make_workload(2, scale)
        d, r = w["data"], w["rand"]
        b = tp.Binning(ctx, tp.S_MU, *S_MU_AXES, 1)

        def feats(c, seed):
            rs = np.random.default_rng(seed)
            f = np.empty((c["ra"].size, 8))
            for j in range(8):
                a1, a2 = rs.normal(0, 0.3, 2)
                f[:, j] = np.cos(a1 * c["ra"] + a2 * c["dec"] + rs.uniform(0, 2 * np.pi))
            return (f - f.mean(0)) / f.std(0)
        fd, fr = feats(d, 21), feats(r, 22)
        theta = rng.normal(0, 0.05, 8)
        wd = np.exp(fd @ theta).astype(np.float32)
        wr = np.exp(fr @ theta).astype(np.float32)
        D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], wd)
        R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], wr)
        # target: an independent clustered catalogue, unit weights, same randoms
        wt = synthetic.survey_catalogue(seed=31, n_data=d["xyz"].shape[0], n_rand=1000)["data"]
        T = tp.Catalog(ctx, wt["xyz"], wt["x_norm"], wt["d_comov"])
        R1 = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"])
        nt, nr_ = wt["xyz"].shape[0], r["xyz"].shape[0]
        tdd, tdr, trr = (tp.count(ctx, a, bb, b, with_regions=False)[0] for a, bb in ((T, None), (T, R1), (R1, None)))
        tn_dd = 2 * tdd / (nt * nt * (1 - 1 / nt))
        tn_rr = 2 * trr / (nr_ * nr_ * (1 - 1 / nr_))
        with np.errstate(divide="ignore", invalid="ignore"):
            xi_t = np.where(tn_rr > 0, (tn_dd - 2 * tdr / (nt * nr_)) / np.where(tn_rr > 0, tn_rr, 1) + 1, 0.0)
        jobs = [(D, None), (D, R), (R, None)]
        sd, sr = float(wd.astype(np.float64).sum()), float(wr.astype(np.float64).sum())
        nd_ = d["xyz"].shape[0]
        kd, kr = sd * sd * (1 - 1 / nd_), sr * sr * (1 - 1 / nr_)

        def fwd():
            out = [tp.count(ctx, a, bb, b, with_regions=False) for a, bb in jobs]
            return sum(o[2]["ms_kernel"] for o in out), out
        ms_f, (_, fo) = median_ms(fwd)
        # dL/d(raw histograms) from the normalisation (JKHists::normalise of
        # the doubled auto counts) and the Landy-Szalay chain
        f_dd, f_dr, f_rr = (o[0] for o in fo)
        ndd, ndr, nrr = 2 * f_dd / kd, f_dr / (sd * sr), 2 * f_rr / kr
        ok = nrr > 0
        safe = np.where(ok, nrr, 1)
        xi = np.where(ok, (ndd - 2 * ndr) / safe + 1, 0.0)
        loss = float(((xi - xi_t) ** 2).sum())
        gx = np.where(ok, 2 * (xi - xi_t), 0.0)
        g_ndd, g_ndr, g_nrr = gx / safe, -2 * gx / safe, -gx * (ndd - 2 * ndr) / safe ** 2
        Gs = [2 * g_ndd / kd, g_ndr / (sd * sr), 2 * g_nrr / kr]

        def bwd():
            out = [tp.count_backward(ctx, a, bb, b, G) for (a, bb), G in zip(jobs, Gs)]
            return sum(o[2]["ms_kernel"] for o in out), out
        ms_b, (_, bo) = median_ms(bwd)
        # per-object dL/dw: adjoint of the pair sums plus the weight-sum terms
        # of the normalisation; dL/dtheta = sum_i dL/dw_i w_i f_i
        gd = bo[0][0] + bo[1][0] - 2 * (g_ndd * ndd).sum() / sd - (g_ndr * ndr).sum() / sd
        gr = bo[1][1] + bo[2][0] - 2 * (g_nrr * nrr).sum() / sr - (g_ndr * ndr).sum() / sr
        dtheta = (gd * wd) @ fd + (gr * wr) @ fr
        pairs = sum(o[2]["in_range"] for o in fo)
        line.update({"metric": "in-range pairs/sec of forward + backward (s-mu DD, DR, RR, loss on xi)",
                     "value": pairs / ((ms_f + ms_b) * 1e-3), "ms": ms_f + ms_b, "forward_ms": ms_f,
                     "backward_ms": ms_b, "forward_plus_backward_over_forward": (ms_f + ms_b) / ms_f,
                     "pairs": pairs, "n_data": int(nd_), "n_rand": int(nr_), "loss": loss,
                     "dL_dtheta": [float(x) for x in dtheta], "dL_dw_data_rms": float(np.sqrt((gd ** 2).mean())),
                     "dL_dw_rand_rms": float(np.sqrt((gr ** 2).mean()))})
    clk.__exit__()
    line["clocks"] = clk.summary()
    line["steps"], line["warmup"] = args.steps, args.warmup
    print(json.dumps(line))
    ctx.close()


def relaunch(args) -> int:
    """bench.py --gpus N started without torchrun: run it again as N ranks
    under torch.distributed.run (127.0.0.1, a free port) and return their
    exit status."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def dist_setup(args):
    """(world size, rank, local GPU index, backend).  NCCL when every rank
    has a GPU of its own, gloo when ranks share one (NCCL refuses two ranks
    on one device) or without a GPU.  NCCL_DEBUG=INFO unless set: its
    communicator lines record the ranks of the exchange."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    backend = None
    if ws > 1 and os.environ.get("OMP_NUM_THREADS") == "1":
        # torchrun's default of one thread per rank would serialise the host
        # planning of each count (work lists, tables): give every rank its
        # share of the host cores before the engine library loads
        per = max(1, (os.cpu_count() or 1) // int(os.environ.get("LOCAL_WORLD_SIZE", str(ws))))
        os.environ["OMP_NUM_THREADS"] = str(per)
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        n_dev = torch.cuda.device_count() if torch.cuda.is_available() else 0
        if n_dev:
            local = local % n_dev
        backend = "nccl" if (n_dev >= ws and not args.gloo and not args.exchange_selftest) else "gloo"
        if backend == "nccl":
            os.environ.setdefault("NCCL_DEBUG", "INFO")
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    return ws, rank, local, backend


def _dist_tensor(x: float):
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor([x], dtype=torch.float64, device=dev)


def dist_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist
    t = _dist_tensor(x)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist
    t = _dist_tensor(x)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dist_barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def exchange_selftest(ws: int, rank: int):
    """Every rank holds one shard's share of known 128-bit totals as int64
    limbs; the sharded count's exchange (two_pcf_b200.reduce_partials) adds
    them and tpcf_shard_combine converts; rank 0 prints whether every rank
    got the totals exactly."""
    import numpy as np
    import torch.distributed as dist
    import two_pcf_b200 as tp
    from two_pcf_b200 import _capi
    b = tp.Binning(None, tp.SIGMA_PI, (0.0, 40.0, 1.0, 6), (0.0, 40.0, 1.0, 6), 2)
    rng = np.random.default_rng(5)
    n_slots, se, words = 3 * b.nb, 20, _capi.PARTIAL_WORDS
    totals = [int(rng.integers(-2**62, 2**62)) << int(rng.integers(0, 60)) for _ in range(n_slots)]
    mine = np.zeros((n_slots, words), np.int64)
    for k, t in enumerate(totals):
        parts = [int(rng.integers(0, 2**63)) << int(rng.integers(0, 64)) for _ in range(ws - 1)]
        parts.append(t - sum(parts))
        u = parts[rank] & ((1 << 128) - 1)
        mine[k, :4] = [(u >> (32 * j)) & 0xffffffff for j in range(4)]
    full, reg = tp.shard_combine(b, tp.reduce_partials(mine, se), se)
    ok = np.array_equal(np.concatenate([full, reg.ravel()]), np.array([float(t) * 2.0 ** -se for t in totals]))
    flags = _dist_tensor(1.0 if ok else 0.0)
    dist.all_reduce(flags)
    if rank == 0:
        print(json.dumps({"exchange_selftest": bool(int(flags.item()) == ws), "n_ranks": ws,
                          "backend": dist.get_backend()}))


def make_workload(seed: int, scale: float):
    from two_pcf_b200 import synthetic
    w = synthetic.survey_catalogue(seed=seed, n_data=max(1000, int(1_000_000 * scale)),
                                   n_rand=max(5000, int(5_000_000 * scale)))
    return w


def reference_grid_candidates(xa, xb, rmax, auto, lo, hi):
    """Candidate pairs the reference's own cell scheme enumerates for one
    count: cells of side rmax on the joint bounding box of the driver's two
    catalogues (cell index (int)((x - min) / rmax), src/boxes.cpp:29-80), every
    cell against its 27 neighbours (src/correlators.cpp:11-125; an auto count
    pairs a cell with itself once, k < l, and with each other neighbour once).
    The FP32 flop model counted on this fixed set of pairs does not depend on
    this engine's refinement or order."""
    from scipy.ndimage import convolve
    dims = (np.floor((hi - lo) / rmax).astype(int) + 1)

    def hist(x):
        c = np.minimum(((x - lo) / rmax).astype(np.int64), dims - 1)
        return np.bincount((c[:, 0] * dims[1] + c[:, 1]) * dims[2] + c[:, 2],
                           minlength=int(np.prod(dims))).reshape(dims).astype(np.float64)
    na = hist(xa)
    nb = na if auto else hist(xb)
    nbr = convolve(nb, np.ones((3, 3, 3)), mode="constant", cval=0.0)
    if auto:
        return int(round((float((na * nbr).sum()) - float(na.sum())) / 2))
    return int(round(float((na * nbr).sum())))


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.dir = tempfile.mkdtemp(prefix="tpcf_clocks_")
        self.path = os.path.join(self.dir, "clocks.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        import shutil
        shutil.rmtree(self.dir, ignore_errors=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def count_step(tp, ctx, D, R, bins, precision, release=True, sharded=False):
    """One pass: grids rebuilt, then DD, DR, RR for each binning; sharded:
    each count split over the ranks (tp.count_sharded), this rank's shard.
    Returns (in_range, candidates, kernel_ms, flops, hists) of this rank."""
    if release:
        for c in (D, R):
            tp._capi.lib().tpcf_catalog_release_cache(c._h)
    in_range = cand = 0
    kms = 0.0
    flops = 0.0
    hists = []
    jobs = [(mode, a, bb, b) for mode, b in bins for a, bb in ((D, None), (D, R), (R, None))]
    if sharded:
        results = [tp.count_sharded(ctx, a, bb, b, precision) for _, a, bb, b in jobs]
    else:
        # one call: each count's host planning overlaps the previous kernel
        results = tp.count_many(ctx, [(a, bb, b) for _, a, bb, b in jobs], precision)
    for (mode, _, _, _), (full, reg, st) in zip(jobs, results):
        in_range += st["in_range"]
        cand += st["candidates"]
        kms += st["ms_kernel"]
        flops += 8.0 * st["candidates"] + F_MODE[mode] * st["in_range"]
        hists.append((full, reg))
    return in_range, cand, kms, flops, hists


def reference_sample(w, target_s: float, rng):
    """A random subsample of the workload sized so that one pass of the
    reference's own OpenMP code (oracle/_ref, built from the reference
    sources) over the step's six counts takes about target_s on this host:
    a 1 % sample calibrates the size.  Returns (data, randoms, fraction,
    seconds of the last pass)."""
    def draw(frac):
        d, r = w["data"], w["rand"]
        nd = max(200, int(d["xyz"].shape[0] * frac))
        nr = max(1000, int(r["xyz"].shape[0] * frac))
        di = np.sort(rng.choice(d["xyz"].shape[0], nd, replace=False))
        ri = np.sort(rng.choice(r["xyz"].shape[0], nr, replace=False))

        def cat(c, idx):
            return {"xyz": c["xyz"][idx], "unit": c["x_norm"][idx], "dcom": c["d_comov"][idx],
                    "w": c["weight"][idx], "jk": c["jk"][idx]}
        return cat(d, di), cat(r, ri)

    frac = 0.01
    cd, cr = draw(frac)
    dt = time_reference(cd, cr)
    if dt < target_s / 8:
        frac = min(1.0, frac * np.sqrt(target_s / max(dt, 1e-3)))
        cd, cr = draw(frac)
        dt = time_reference(cd, cr)
    return cd, cr, frac, dt


def time_reference(cd, cr):
    """Seconds of one pass of the reference's auto_/cross_pair_count_* over
    the step's six counts (sigma-pi and s-mu DD, DR, RR) on all host threads."""
    from oracle import refl
    n_threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    for ax, mode in ((SIGMA_PI_AXES, refl.SIGMA_PI), (S_MU_AXES, refl.S_MU)):
        axes = (*ax[0][:3], ax[0][3], *ax[1][:3], ax[1][3])
        refl.count_3d(mode, cd, cr, is_auto=True, n_jk=100, axes=axes, n_threads=n_threads)
        refl.count_3d(mode, cd, cr, is_auto=False, n_jk=100, axes=axes, n_threads=n_threads)
        refl.count_3d(mode, cr, cd, is_auto=True, n_jk=100, axes=axes, n_threads=n_threads)
    return time.perf_counter() - t0


def sample_text(cd, cr, frac):
    return (f"random {frac:.3f} subsample of the workload: {cd['xyz'].shape[0]} data, {cr['xyz'].shape[0]} "
            f"randoms; sigma-pi and s-mu DD+DR+RR through the reference's auto_/cross_pair_count_* built from its "
            f"sources (g++ -O3 -fopenmp), {os.cpu_count() or 1} OpenMP threads")


def cpu_reference_sample(w, target_s: float = 12.0, ctx=None):
    """The reference's own OpenMP code timed on a random subsample of the
    workload (this arm's cpu_baseline); the sample's in-range pairs come from
    the engine on the identical sample.  Returns a cpu_baseline dict."""
    import two_pcf_b200 as tp
    cd, cr, frac, dt = reference_sample(w, target_s, np.random.default_rng(7))
    D = tp.Catalog(ctx, cd["xyz"], cd["unit"], cd["dcom"], cd["w"], None, cd["jk"], 100)
    R = tp.Catalog(ctx, cr["xyz"], cr["unit"], cr["dcom"], cr["w"], None, cr["jk"], 100)
    bins = [(1, tp.Binning(ctx, tp.SIGMA_PI, *SIGMA_PI_AXES, 100)), (2, tp.Binning(ctx, tp.S_MU, *S_MU_AXES, 100))]
    pairs = count_step(tp, ctx, D, R, bins, tp.FP32_GUARD)[0]
    return {"value": pairs / dt, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference", "seconds": dt,
            "in_range_pairs": pairs, "sample": sample_text(cd, cr, frac)}


def _kdtree_count(job):
    """One count's in-range pairs (0 < s < r) by KD-tree pair counting."""
    from scipy.spatial import cKDTree
    a, b, r = job
    ta = cKDTree(a)
    if b is None:  # unordered pairs of distinct points
        return (int(ta.count_neighbors(ta, r)) - int(ta.count_neighbors(ta, 0.0))) // 2
    tb = cKDTree(b)
    return int(tb.count_neighbors(ta, r)) - int(tb.count_neighbors(ta, 0.0))


def in_range_pairs_kdtree(cd, cr):
    """In-range pairs of the step's six counts on a sample (the reference's
    range test 0 < s^2 < max^2 of sigma-pi and s-mu), counted with scipy's
    KD-tree in spawned worker processes, no part of this engine involved.
    Separations are compared in double; pairs within ~1e-7 relative of a
    range limit may fall on the other side of the reference's float test."""
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp
    xd = cd["xyz"][cd["dcom"] >= 0]
    xr = cr["xyz"][cr["dcom"] >= 0]
    radii = [float(np.sqrt(SIGMA_PI_AXES[0][1] ** 2 + SIGMA_PI_AXES[1][1] ** 2)), float(S_MU_AXES[0][1])]
    jobs = [(a, b, r * (1.0 - 1e-12)) for r in radii for a, b in ((xd, None), (xd, xr), (xr, None))]
    with ProcessPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1),
                             mp_context=mp.get_context("spawn")) as ex:
        return int(sum(ex.map(_kdtree_count, jobs)))


def run_reference_arm(args, ws, rank):
    """--impl reference: the reference's CPU implementation on the host cores.
    One sample of the workload is drawn (sized for ~8 s of reference work per
    step) and its in-range pairs are counted once by KD-tree; each of the
    --steps steps times one pass of the reference's code over it."""
    if rank != 0:
        return
    from oracle import refl
    if not refl.available("plain"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtwopcf_ref_plain.so not built "
                          "(oracle/build_ref.sh needs the reference sources)"}))
        return
    w = make_workload(2, args.scale)
    cd, cr, frac, _ = reference_sample(w, 8.0, np.random.default_rng(7))   # also the warm-up pass
    pairs = in_range_pairs_kdtree(cd, cr)
    secs = [time_reference(cd, cr) for _ in range(max(1, args.steps))]
    v = pairs / statistics.median(secs)
    sample = sample_text(cd, cr, frac) + "; in-range pairs of the sample by KD-tree pair counting"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": {"workload": "survey slab 1M data / 5M randoms, sigma-pi 50x50 + "
                                                        "s-mu 40x50, 100 jackknife regions, weighted",
                                            "sample": sample},
            "in_range_pairs_per_step": pairs,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.one_count:
        one_count(args)
        return
    if args.workload != "survey":
        other_workload(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args))
    ws, rank, local, backend = dist_setup(args)
    if args.exchange_selftest:
        exchange_selftest(ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    import two_pcf_b200 as tp
    torch.cuda.set_device(local)
    ctx = tp.Context(local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_autotune(not args.no_autotune)

    sharded = ws > 1 and not args.replicas
    w = make_workload(2 if sharded else 2 + rank, args.scale)
    n_jk = w["n_jk"]
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], n_jk)
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], n_jk)
    bins = [(1, tp.Binning(ctx, tp.SIGMA_PI, *SIGMA_PI_AXES, n_jk)),
            (2, tp.Binning(ctx, tp.S_MU, *S_MU_AXES, n_jk))]
    fp32_tflops, atom_rate = 0.0, 0.0
    import ctypes as C
    a1, a2 = C.c_double(), C.c_double()
    if tp._capi.lib().tpcf_measure_peaks(ctx._h, C.byref(a1), C.byref(a2)) == 0:
        fp32_tflops, atom_rate = a1.value, a2.value
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    for _ in range(max(3, args.warmup)):
        count_step(tp, ctx, D, R, bins, tp.FP32_GUARD, sharded=sharded)
    torch.cuda.synchronize()

    def timed_steps(precision, k):
        """k steps of `precision`, each after an L2 flush, bracketed by CUDA
        events on the engine's stream; returns per-step device ms and the
        step totals."""
        ms, n_in, n_c, kms, fl, last = [], 0, 0, 0.0, 0.0, None
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.random_(0, 255)   # evict the L2 between steps
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            a, c, km, f, last = count_step(tp, ctx, D, R, bins, precision, sharded=sharded)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            n_in += a
            n_c += c
            kms += km
            fl += f
        return ms, n_in, n_c, kms, fl, last

    launches0 = tp._capi.lib().tpcf_kernel_launches(ctx._h)
    with ClockSampler(local) as clk:
        dist_barrier(ws)
        torch.cuda.synchronize()
        step_ms, tot_in, tot_cand, tot_kms, tot_flops, hists = timed_steps(tp.FP32_GUARD, args.steps)
        torch.cuda.synchronize()
        dist_barrier(ws)
        launches = tp._capi.lib().tpcf_kernel_launches(ctx._h) - launches0
        # the plain FP64 path on the same steps, timed the same way (one
        # untimed step first builds its grids and warms its kernels)
        fp64_run = None
        if not args.no_fp64:
            count_step(tp, ctx, D, R, bins, tp.FP64, sharded=sharded)
            torch.cuda.synchronize()
            dist_barrier(ws)
            fp64_run = timed_steps(tp.FP64, args.steps)
            torch.cuda.synchronize()
            dist_barrier(ws)
    total_ms = dist_max(sum(step_ms), ws)
    # whole job: pairs counted by all ranks (replicas, or the shards of one workload)
    value = dist_sum(tot_in, ws) / (total_ms * 1e-3)
    clocks = clk.summary()

    fp64 = None
    if fp64_run is not None:
        ms64, n64, _, kms64, _, h64 = fp64_run
        t64 = dist_max(sum(ms64), ws)
        exact = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(hists, h64))
        fp64 = {"value": dist_sum(n64, ws) / (t64 * 1e-3), "steps": args.steps, "ms_per_step": t64 / args.steps,
                "kernel_ms_per_step": kms64 / args.steps,
                "speedup_fp32_guard": t64 / total_ms,
                "speedup_fp32_guard_kernels": kms64 / tot_kms if tot_kms > 0 else None,
                "bit_exact_histograms": bool(exact), "in_range_equal": int(n64) == int(tot_in)}

    # end to end through the C ABI: pinned host catalogues in, histograms out
    e2e = None
    if not args.no_e2e:
        pin = {}
        for name, c in (("d", d), ("r", r)):
            pin[name] = {k: torch.from_numpy(np.ascontiguousarray(c[k])).pin_memory().numpy()
                         for k in ("xyz", "x_norm", "d_comov", "weight", "jk")}
        h2d = sum(pin[n][k].nbytes for n in pin for k in ("xyz", "x_norm", "weight", "jk"))
        d2h = sum(b.nb * (1 + n_jk) * 8 * 3 for _, b in bins)
        e_ms = []
        e_in = 0
        for s in range(args.steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Dp = tp.Catalog(ctx, pin["d"]["xyz"], pin["d"]["x_norm"], pin["d"]["d_comov"], pin["d"]["weight"], None,
                            pin["d"]["jk"], n_jk)
            Rp = tp.Catalog(ctx, pin["r"]["xyz"], pin["r"]["x_norm"], pin["r"]["d_comov"], pin["r"]["weight"], None,
                            pin["r"]["jk"], n_jk)
            n_in = count_step(tp, ctx, Dp, Rp, bins, tp.FP32_GUARD, release=False, sharded=sharded)[0]
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            Dp.close()
            Rp.close()
            if s > 0:   # first pass warms the allocator
                e_ms.append(dt * 1e3)
                e_in += n_in
        e_total = dist_max(sum(e_ms), ws)
        e2e = {"value": dist_sum(e_in, ws) / (e_total * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": e_total / len(e_ms)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            from oracle import refl
            if refl.available("plain"):
                cpu = cpu_reference_sample(w, ctx=ctx)
        except Exception as ex:  # report, do not fail the bench
            cpu = {"value": None, "error": str(ex)}

    achieved = tot_flops / (tot_kms * 1e-3) / 1e12 if tot_kms > 0 else 0.0
    # the same flop model on the reference's own candidate set (cells of side
    # r_max, 27 neighbours): a fixed amount of work per step
    lo = np.minimum(d["xyz"].min(0), r["xyz"].min(0))
    hi = np.maximum(d["xyz"].max(0), r["xyz"].max(0))
    ref_cand, ref_flops = 0, 0.0
    in_per_step = tot_in / args.steps
    for mode, rmax in ((1, float(np.hypot(SIGMA_PI_AXES[0][1], SIGMA_PI_AXES[1][1]))), (2, S_MU_AXES[0][1])):
        for xa, xb, auto in ((d["xyz"], None, True), (d["xyz"], r["xyz"], False), (r["xyz"], None, True)):
            ref_cand += reference_grid_candidates(xa, xb, rmax, auto, lo, hi)
    ref_flops = 8.0 * ref_cand + (tot_flops - 8.0 * tot_cand) / args.steps  # in-range part as measured
    ref_achieved = ref_flops / (tot_kms / args.steps * 1e-3) / 1e12 if tot_kms > 0 else 0.0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong" if sharded else "weak",
        "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "survey slab: 1M clustered data + 5M randoms, weights lognormal(0,0.2), 100 jk "
                               "regions; sigma-pi 50x50 linear 0-50 + s-mu 40 log(1.3) 0-100 x 50 mu; "
                               "DD+DR+RR each; grids rebuilt every step",
                   "scale": args.scale, "n_data": int(d["xyz"].shape[0]), "n_rand": int(r["xyz"].shape[0]),
                   "l2": "inputs larger than L2 (sorted tiles 192 MB + catalogues) and a 256 MB L2 flush "
                         "between steps",
                   "parallelism": (f"shards{ws}" if sharded else f"replicas{ws}") if ws > 1 else "single",
                   "exchange": backend if sharded else None},
        "in_range_pairs_per_step": tot_in // args.steps, "candidates_per_step": tot_cand // args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_tflops, "unit": "TFLOP/s",
                     "frac": achieved / fp32_tflops if fp32_tflops else None,
                     "traffic": TRAFFIC_SMU_RR,
                     "traffic_note": "DRAM bytes (read + write) of one full-size s-mu RR launch (5M randoms, 3 cells "
                                     "per maximum separation; one-pass ncu capture, profiles/"
                                     "pair_count_smu_jk_weighted_ncu.md): 21.3 GB, about 1.1x the algorithmic tile "
                                     "loads (each work item streams the B points of its segments once per A chunk "
                                     "of at most 1024 points: at least 32 B x 6.09e11 candidates / 1024 = 19.0 GB; "
                                     "the catalogue itself is 0.16 GB); 12 GB/s over the launch, 0.2 % of HBM "
                                     "bandwidth",
                     "smem_atomics_per_s": 2.0 * tot_in / (tot_kms * 1e-3) if tot_kms > 0 else None,
                     "smem_atomic_frac": (2.0 * tot_in / (tot_kms * 1e-3) / atom_rate) if (tot_kms > 0 and atom_rate)
                     else None,
                     "peak_source": "FP32 FMA probe kernel run live on this GPU (tpcf_measure_peaks); "
                                    "MEASURED_PEAKS.json has no FP32 figure",
                     "flops_model": "8 per candidate pair + 16 (sigma-pi) / 13 (s-mu) per in-range pair",
                     "kernel_ms_per_step": tot_kms / args.steps,
                     "smem_atomic_peak_per_s": atom_rate,
                     "reference_grid": {
                         "candidates_per_step": ref_cand, "achieved": ref_achieved,
                         "frac": ref_achieved / fp32_tflops if fp32_tflops else None,
                         "note": "the same flop model with the candidates the reference's own cell scheme "
                                 "enumerates (cells of side r_max, 27 neighbours): a fixed workload; `achieved` "
                                 "above counts the candidates this engine enumerated, fewer when its refinement "
                                 "is finer"}},
        "fp64_path": fp64, "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clocks,
        "autotune": ctx.autotune_table() if not args.no_autotune else None,
    }
    if rank == 0:
        print(json.dumps(line))
        if args.save_hists:
            names = [f"{m}_{c}" for m in ("sigma_pi", "s_mu") for c in ("dd", "dr", "rr")]
            np.savez(args.save_hists, **{f"{n}_full": h[0] for n, h in zip(names, hists)},
                     **{f"{n}_regions": h[1] for n, h in zip(names, hists)})
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
