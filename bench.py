#!/usr/bin/env python
"""Pair-count throughput of the post-growth analysis path on one B200.

Workload (the exact-count configuration of the analysis path): mixed-type
cover-shaped synthetic data, n = 50,000 samples, p = 54 (10 continuous + one-hot
groups of 4 and 40), 7 imbalanced classes; a forest of 1,000 trees (mtry 7,
nodesize 1) grown by the library's restatement of the reference's grower.

One step = one full analysis pass through the C ABI with device-resident
inputs and outputs: leaf routing of every (tree, sample) with OOB votes, the
per-tree leaf member lists, the exact INT32 upper-triangle pair counts S, and
permutation importance over all 54 features (overall and local).
metric = pair updates per second (sum over trees and leaves of
#OOB x #in-bag members; counted exactly by the kernel) of that step.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--workload exact|lowrank|large|batch|rows]
Under torchrun (N > 1) every rank runs an independent replica on its own GPU
(the path needs no exchange between replicas); value is the sum over ranks,
timed as the max over ranks.  The other workloads print their own line: the
low-rank proximity + MDS in the mixed and the FP32 form (lowrank: n = 200,000;
large: n = 1,000,000 with outlier scores), 64 uneven forests in one CUDA graph
(batch), and the device time of finishprox, prediction and the full-matrix MDS
(rows).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SAMPLES = 50_000
N_TREES = 1000
MTRY = 7
WORKLOAD = ("exact pair counts + varimp: n={n} p=54 (10 continuous + one-hot 4 + one-hot 40) c=7, "
            "ntree={T} mtry=7 nodesize=1, INT32 upper-triangle S (n(n+1)/2) + all 54 feature permutations")
FALLBACK_HBM_GBS = 6650.0


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def replica_reduce(x: float, op: str, device=None) -> float:
    """Max or sum of a per-rank number over the replicas (identity without a
    process group).  Every rank calls it in the same order."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def forest_cache_path(n, T):
    """Where the bench forest of (n, T) is kept between the two arms' runs."""
    from rfx_b200 import synth

    return os.path.join(tempfile.gettempdir(),
                        f"rfx_bench_forest_n{n}_t{T}_mtry{MTRY}_seed{synth.SEED_BASE + 2}_v1.npz")


def grow_forest_file(n, T, path):
    """Grow the bench forest with the library's grower and save it (run in a
    child process by `cached_forest`)."""
    from rfx_b200 import abi, synth

    X, y = synth.mixed_cover(n)
    cat = synth.detect_categorical(X)
    f = abi.grow_forest(X, y, T, MTRY, 1, cat=cat, nclass=7)
    tmp = path + f".{os.getpid()}.tmp.npz"
    f.save(tmp)
    os.replace(tmp, path)


def cached_forest(n, T):
    """Data + forest of the exact workload, identical in both arms.

    The forest is grown once per (n, T) by a child process (the library's
    restatement of the reference grower) and read back here with the
    numpy-only loader, so this process maps no native library for it: the
    reference arm's timed process then runs only the reference's code and
    the oracle.  Returns (X, y, forest, seconds spent obtaining it)."""
    from rfx_b200 import synth
    from rfx_b200.forest import Forest

    X, y = synth.mixed_cover(n)
    path = forest_cache_path(n, T)
    t0 = time.time()
    f = None
    if os.path.exists(path):
        try:
            f = Forest.load(path)
            if f.n != n or f.ntree != T:
                f = None
        except Exception:
            f = None
    if f is None:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--grow-forest", path, "--n", str(n),
                        "--trees", str(T)], check=True)
        f = Forest.load(path)
    return X, y, f, time.time() - t0


def make_forest(n, T, rank, ws, barrier):
    """Data + forest; rank 0 obtains it (grown once, kept on disk), the other
    ranks read the same file after a barrier."""
    from rfx_b200 import synth
    from rfx_b200.forest import Forest

    t0 = time.time()
    if rank == 0:
        X, y, f, _ = cached_forest(n, T)
    barrier()
    if rank != 0:
        X, y = synth.mixed_cover(n)
        f = Forest.load(forest_cache_path(n, T))
    barrier()
    return X, y, f, time.time() - t0


def exact_config(n, p, T, U):
    """The `config` of the exact workload, printed identically by both arms."""
    return {"workload": WORKLOAD.format(n=n, T=T), "n": n, "p": p, "ntree": T, "pair_updates_per_step": int(U),
            "l2": "inputs larger than L2 (S 5.0 GB written per step; nodes and leaf keys > 126 MB)"}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.remove(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def tree_pair_updates(X, y, f):
    """Pair updates of every tree (the metric's unit count) on the CPU: per
    tree, the sum over terminal nodes of OOB members x in-bag members, from
    the oracle's leaf ids (OOB rows by testreebag, in-bag rows by
    find_terminal_node; rows that end on a non-terminal node count nowhere,
    as in cpu_proximity's dense branch, src/rf_proximity.cpp:108-231)."""
    from oracle import oracle as orc

    leaf = orc.analyse(X, y, f, do_imp=False, impn=False, do_prox=False, want_leaf=True)["leaf"]
    U = np.zeros(f.ntree, np.int64)
    for t in range(f.ntree):
        lf = leaf[t].astype(np.int64)
        term = f.nodestatus[f.offs[t]: f.offs[t + 1]][lf] == -1
        inb = f.nin[t] > 0
        no = np.bincount(lf[term & ~inb], minlength=int(f.nnode[t]))
        ni = np.bincount(lf[term & inb], minlength=int(f.nnode[t]))
        U[t] = int(no @ ni)
    return U


def forest_pair_updates(X, y, f):
    """Pair updates of the whole forest (see tree_pair_updates)."""
    return int(tree_pair_updates(X, y, f).sum())


class CpuTrees:
    """The reference's CPU path, one tree at a time, on the box's host cores.

    Per tree, as grow_tree_single does: cpu_testreebag, the vote loop,
    cpu_varimp (OpenMP over features) and find_terminal_node, all from
    oracle/_ref (the reference's own sources); the pair counts use the
    oracle's restatement of cpu_proximity's dense branch (the shipped
    cpu_proximity takes its sparse branch above n = 5000, and its n*n int32
    size overflows at n = 50,000), added into one upper-triangle array that is
    allocated and touched once, as the reference accumulates one proximity
    array over the forest.  Without oracle/_ref the oracle runs the whole
    sequence ("port").  Trees are taken in a seeded random order: per-tree
    pair counts are heavy-tailed (a tree with one large leaf has 100x the
    median), so the first trees are not a fair sample."""

    def __init__(self, X, y, f):
        from oracle import reference as ref

        self.X, self.y, self.f = X, y, f
        self.cores = os.cpu_count() or 1
        if ref.available():
            ref.set_threads(self.cores)
            self.kind = "reference"
        else:
            self.kind = "port"
        self.order = np.random.default_rng(0).permutation(f.ntree)
        self.S = np.empty(f.n * (f.n + 1) // 2, np.int32)
        self.S.fill(0)

    def tree_seconds(self, k):
        """Wall seconds of the k-th tree of the sample order."""
        from oracle import oracle as orc, reference as ref

        sub = self.f.subset([int(self.order[k % self.f.ntree])])
        t0 = time.perf_counter()
        if self.kind == "reference":
            ref.analyse_trees(self.X, self.y, sub, do_imp=True, impn=True, do_prox=False)
            orc.analyse(self.X, self.y, sub, do_imp=False, impn=False, do_prox=True, S=self.S)
        else:
            orc.analyse(self.X, self.y, sub, do_imp=True, impn=True, do_prox=True, S=self.S)
        return time.perf_counter() - t0


def cpu_baseline_run(X, y, f, budget_s=15.0, min_trees=2, pair_updates=None):
    """The reference's CPU path (CpuTrees) on a bounded sample of trees:
    the forest's rate = its total pair updates / (mean seconds per sampled
    tree x ntree).  Returns (pair updates/s, dict)."""
    U = forest_pair_updates(X, y, f) if pair_updates is None else int(pair_updates)
    run = CpuTrees(X, y, f)
    done, t_total = 0, 0.0
    while done < f.ntree and (done < min_trees or t_total < budget_s):
        t_total += run.tree_seconds(done)
        done += 1
    per_tree = t_total / done
    return U / (per_tree * f.ntree), {
        "cores": run.cores if run.kind == "reference" else 1, "kind": run.kind, "trees": done,
        "seconds": t_total,
        "sample": f"{done} of {f.ntree} trees (seeded random order) at n={f.n}, {t_total:.1f} s: testreebag + "
                  f"votes + cpu_varimp over {f.p} features + find_terminal_node + dense-branch pair counts; "
                  f"rate = the forest's {U} pair updates / ({per_tree:.3f} s per tree x {f.ntree} trees)"}


def run_reference(args):
    """The reference arm: the reference's own CPU path (CpuTrees) on all host
    cores over the same forest as the repository arm.

    The forest's trees are taken in a seeded random order and dealt out in
    equal blocks over the warm-up and timed steps, so that the timed steps
    together cover most of the forest once (about 150 s at n = 50,000 on 16
    cores); a step is one block.  Rate = the timed trees' exact pair updates
    over their summed wall time.  This process loads only the reference's
    build (oracle/_ref) and the oracle: the forest comes from `cached_forest`
    (a child process grows it when it is not on disk yet)."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    n, T = args.n, args.trees
    X, y, f, _ = cached_forest(n, T)
    Ut = tree_pair_updates(X, y, f)
    U = int(Ut.sum())
    run = CpuTrees(X, y, f)
    nsteps = args.warmup + args.steps
    block = max(1, T // nsteps)
    t_tot, u_tot, trees = 0.0, 0, 0
    for s in range(nsteps):
        dt, du = 0.0, 0
        for k in range(s * block, (s + 1) * block):
            dt += run.tree_seconds(k)
            du += int(Ut[run.order[k % T]])
        if s >= args.warmup:
            t_tot += dt
            u_tot += du
            trees += block
    value = u_tot / t_tot
    cores = run.cores if run.kind == "reference" else 1
    line = {"metric": "prox pair-updates/s", "value": value, "unit": "pair-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded mixed-type cover-shaped generator; forest grown by the library's "
                    "restatement of the reference grower)",
            "impl": "reference", "config": exact_config(n, f.p, T, U),
            "parallelism": f"host cores (OpenMP, {cores} threads)",
            "cpu_baseline": {"value": value, "unit": "pair-updates/s", "cores": cores, "kind": run.kind,
                             "sample": f"{trees} of the {T} trees (seeded random order, {block} per step) at n={n}: "
                                       "testreebag + votes + cpu_varimp over all features + find_terminal_node "
                                       "(the reference's own build) + dense-branch pair counts into one "
                                       "upper-triangle array; rate = those trees' exact pair updates "
                                       f"({u_tot}) / their summed time ({t_tot:.1f} s)"},
            "e2e": {"value": value, "unit": "pair-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_lowrank(args):
    """Low-rank proximity + MDS, the mixed form against the plain FP32 form,
    both timed end to end on the device, with the relative Frobenius error of
    each against the exact FP64 proximity on a seeded 20,000-row subsample.

    lowrank: n=200,000 cover-shaped rows, 2,000 trees, rank 64, factors INT8
             with per-column scales, 3-D MDS from the quantised factors.
    large:   n=1,000,000 Gaussian-mixture rows with 1% injected outliers, 500
             trees (mtry 5, nodesize 5), rank 32, factors FP8 e4m3 with
             per-column scales, 3-D MDS and outlier scores from the factors.
    mixed = BF16 sketch storage with FP32 accumulation, tcgen05 BF16 MDS
    products with one FP32 refinement step; FP32 = the same algorithm in FP32."""
    import torch

    from rfx_b200 import abi, synth

    large = args.workload == "large"
    if large:
        n = args.n if args.n is not None else 1_000_000
        T = args.trees if args.trees is not None else 500
        k, fmt, mtry, minnd, nclass = 32, 2, 5, 5, 4
        X, y, outl = synth.large_gmm(n, return_outliers=True)
        cat = np.ones(X.shape[1], np.int32)
        gen = "Gaussian mixture, 8 components, 4 classes, 1% uniform outliers in a 10x box, seed 20251006"
    else:
        n = args.n if args.n is not None else 200_000
        T = args.trees if args.trees is not None else 2000
        k, fmt, mtry, minnd, nclass = 64, 1, MTRY, 1, 7
        X, y = synth.mixed_cover(n, seed=synth.SEED_BASE + 3)
        cat = synth.detect_categorical(X)
        gen = "mixed-type cover-shaped generator, seed 20251004"
    t0 = time.time()
    f = abi.grow_forest(X, y, T, mtry, minnd, cat=cat, nclass=nclass)
    grow_s = time.time() - t0
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    ctx.route_oob()

    # forms: 0 = FP32, 1 = mixed with BF16 sketch storage and BF16 tensor-core
    # factor-MDS products, 3 = mixed with FP8 e4m3 sketch storage and FP8
    # E4M3 tensor-core factor-MDS products (both mixed forms end the MDS with
    # one FP32 refinement step); the FP8 form's MDS with BF16 products is
    # timed on its own below for comparison
    forms = (0, 1, 3)
    phases = {p: {} for p in forms}

    def run(precision, trees_per_pass=0):
        torch.cuda.synchronize()
        ctx.profile(True)
        t = time.perf_counter()
        A, ev = ctx.lowrank(k, oversample=16, power_iters=1, precision=precision, trees_per_pass=trees_per_pass)
        t1 = time.perf_counter()
        ctx.lowrank_quantize(fmt)
        t2 = time.perf_counter()
        C, _ = ctx.mds_from_factors(3, use_quantized=True, precision=precision)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        o = ctx.outlier_scores(use_quantized=True) if large else None
        t4 = time.perf_counter()
        st, _ = ctx.profile_read()
        phases[precision] = {"factors_s": t1 - t, "quantize_s": t2 - t1, "mds_s": t3 - t2,
                             "operator_product_ms_avg": st["lowrank_product"], "orth_ms_avg": st["lowrank_orth"],
                             "mds_ms": st["mds_factors"], "route_ms": max(st["route"], 0.0),
                             "leaf_lists_ms": max(st["leaf_lists"], 0.0)}
        if large:
            phases[precision]["outlier_s"] = t4 - t3
        return t4 - t, A, C, o

    run(1)  # warm-up (module load, allocations; builds the leaf keys and member lists once)
    once_ms = {key: phases[1][key] for key in ("route_ms", "leaf_lists_ms")}
    run(0)
    run(3)
    times = {p: [] for p in forms}
    best = {p: None for p in forms}
    res = {}
    clocks = Clocks(0)
    clocks.start()
    for rep in range(max(1, args.steps)):
        for prec in forms:
            dt, A, C, o = run(prec)
            times[prec].append(dt)
            res[prec] = (A, C, o)
            # phases of the fastest repetition of each form
            if best[prec] is None or dt <= min(times[prec]):
                best[prec] = dict(phases[prec])
    # the plain form: FP32 with one tree per pass of the leaf sums (the
    # per-tree structure of the reference's GPU accumulation), timed once
    t_plain, A_plain, _, _ = run(0, trees_per_pass=1)
    # the MDS of the FP8 form's factors with BF16 tensor-core products
    # (precision 1 of the MDS call), after one untimed call
    ctx.lowrank(k, oversample=16, power_iters=1, precision=3)
    ctx.lowrank_quantize(fmt)
    ctx.mds_from_factors(3, use_quantized=True, precision=1)
    torch.cuda.synchronize()
    t = time.perf_counter()
    C_b16, _ = ctx.mds_from_factors(3, use_quantized=True, precision=1)
    torch.cuda.synchronize()
    t_mds_b16 = time.perf_counter() - t
    clk = clocks.stop()
    phases = best
    # exact FP64 proximity on a seeded subsample
    m = min(20_000, n)
    rng = np.random.default_rng(7)
    sub = np.sort(rng.choice(n, size=m, replace=False))
    fs = f.subset(range(T))
    fs.n = m
    fs.nin = np.ascontiguousarray(f.nin[:, sub])
    ctx_s = abi.Context(0)
    ctx_s.load(fs, X[sub], y[sub])
    dev = torch.device("cuda", 0)
    Ssub = torch.empty(m * (m + 1) // 2, dtype=torch.int32, device=dev)
    ctx_s.proximity_upper(Ssub)
    Psub = torch.empty((m, m), dtype=torch.float32, device=dev)
    ctx_s.finishprox(Ssub, Psub, full=True)
    ctx_s.synchronize()
    del Ssub
    Mx = Psub.double()
    Mx.fill_diagonal_(0.0)
    nrm = float(torch.linalg.norm(Mx))
    errs = {}

    def sub_err(A):
        As = torch.from_numpy(A[sub]).to(dev).double()
        R = Mx - As @ As.T
        R.fill_diagonal_(0.0)
        return float(torch.linalg.norm(R)) / nrm

    for prec in forms:
        errs[prec] = sub_err(res[prec][0])
    err_plain = sub_err(A_plain)
    # rank truncation against algorithm error: the best rank-k approximation of
    # the subsample's own exact matrix (top-k positive eigenpairs, FP64) in the
    # same metric, and the eigenvalue-tail estimate of the rank that reaches
    # 1e-2 on the subsample
    w, V = torch.linalg.eigh(Mx)
    order = torch.argsort(w, descending=True)
    wk = w[order[:k]].clamp(min=0.0)
    Ak = V[:, order[:k]] * wk.sqrt()
    Rk = Mx - Ak @ Ak.T
    Rk.fill_diagonal_(0.0)
    floor_k = float(torch.linalg.norm(Rk)) / nrm
    del Ak, Rk, V
    wpos = w[order].clamp(min=0.0)
    tail = (float(torch.sum(w * w)) - torch.cumsum(wpos * wpos, 0)).clamp(min=0.0).sqrt() / nrm
    hit = torch.nonzero(tail <= 1e-2)
    rank_1e2 = int(hit[0]) + 1 if hit.numel() else None
    # the range finder with more power iterations (FP32 form), same rank
    sweep = {}
    for q_it in (1, 2, 3):
        Aq, _ = ctx.lowrank(k, oversample=16, power_iters=q_it, precision=0)
        sweep[str(q_it)] = sub_err(Aq)
    def procrustes(Cm, C32):
        U, _, Vt = np.linalg.svd(Cm.T @ C32)
        return float(np.sqrt(np.mean((Cm @ (U @ Vt) - C32) ** 2)) / np.sqrt(np.mean(C32 ** 2)))

    procs = {p: procrustes(res[p][1], res[0][1]) for p in (1, 3)}
    proc_mds_b16 = procrustes(C_b16, res[0][1])
    ctx_s.close()
    ctx.close()
    t32 = min(times[0])
    # the headline mixed form: the faster of the two whose factor error is
    # the FP32 form's to 1 % (relative)
    same = [p for p in (1, 3) if abs(errs[p] - errs[0]) <= 0.01 * errs[0]]
    mix = min(same, key=lambda p: min(times[p])) if same else 1
    tmx = min(times[mix])
    proc = procs[mix]
    qname = "FP8 e4m3" if fmt == 2 else "INT8"
    line = {"metric": f"n={n // 1000}K rank-{k} prox+MDS sec, mixed vs FP32 form @same err", "value": tmx,
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": args.steps,
            "dtype": ("fp8+fp32" if mix == 3 else "bf16+fp32") + " (mixed) / fp32", "data": f"synthetic ({gen})",
            "config": {"workload": f"low-rank proximity + 3D MDS{' + outlier scores' if large else ''}: n={n} "
                                   f"p={X.shape[1]} c={nclass} ntree={T} mtry={mtry} nodesize={minnd} rank={k} "
                                   f"oversample=16 power_iters=1, {qname} per-column factors",
                       "forest_grow_s": round(grow_s, 1), "per_forest_once_ms": once_ms,
                       "timed": f"factors (range finder), {qname} quantisation, 3-D MDS from the quantised factors"
                                f"{', outlier scores' if large else ''}; leaf keys and member lists are built once "
                                "per loaded forest (per_forest_once_ms)"},
            "fp32_seconds": t32, "mixed_seconds": tmx, "speedup_mixed_vs_fp32": t32 / tmx,
            "mixed_form": "FP8 e4m3 sketch storage" if mix == 3 else "BF16 sketch storage",
            "rel_frobenius_err_fp32": errs[0], "rel_frobenius_err_mixed": errs[mix],
            "mixed_bf16_seconds": min(times[1]), "mixed_fp8_seconds": min(times[3]),
            "plain_fp32_seconds": t_plain, "speedup_mixed_vs_plain_fp32": t_plain / tmx,
            "rel_frobenius_err_plain_fp32": err_plain,
            "plain_note": ("plain = the FP32 form with one tree per pass of the leaf sums (the per-tree structure "
                           "of the reference's GPU accumulation); fp32 = the same algorithm batched, 4 GB of leaf "
                           "sums per pass"),
            "rel_frobenius_err_mixed_bf16": errs[1], "rel_frobenius_err_mixed_fp8": errs[3],
            "mds_procrustes_rel_mixed_bf16_vs_fp32": procs[1], "mds_procrustes_rel_mixed_fp8_vs_fp32": procs[3],
            "mds_fp8_products_seconds": phases[3]["mds_s"], "mds_bf16_products_seconds_fp8_form": t_mds_b16,
            "mds_procrustes_rel_bf16_products_fp8_form_vs_fp32": proc_mds_b16,
            "err_subsample_rows": m, "rel_frobenius_err_best_rank_k_on_subsample": floor_k,
            "rank_for_1e-2_on_subsample_eigen_tail": rank_1e2,
            "rel_frobenius_err_fp32_by_power_iters": sweep,
            "err_note": ("errors: ||M - A A^T||_F / ||M||_F over the subsample's off-diagonal entries, M = exact "
                         "P - I (FP64); best_rank_k = top-k positive eigenpairs of the subsample's own M (a lower "
                         "bound for any rank-k factors restricted to the subsample); rank_for_1e-2 from the "
                         "eigenvalue tail (diagonal kept)"),
            "mds_procrustes_rel_mixed_vs_fp32": proc,
            "phases_fp32": phases[0], "phases_mixed": phases[mix], "phases_mixed_bf16": phases[1],
            "phases_mixed_fp8": phases[3]}
    if large:
        o = res[mix][2]
        top = np.argsort(-o)[: len(outl)]
        line["outlier_recall_top1pct"] = float(np.isin(top, outl).mean())
    if clk:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)
    return 0


def run_rows(args):
    """The path's other rows, each timed on the device by the library's stage
    events (mean over the timed launches, inputs and outputs in HBM):
    finishprox (full n x n and packed upper) and test-set prediction at
    n = 50,000 / 1,000 trees (the exact workload's forest), and the
    full-matrix 3-D MDS at n = 2,000 (500 trees, 13 Gaussian features, the
    reference's CPU-runnable size) and at n = 50,000."""
    import torch

    from rfx_b200 import abi, synth

    hbm, peak_src = peaks()
    dev = torch.device("cuda", 0)
    reps = max(args.steps, 1)
    warm = max(args.warmup, 3)

    def timed(ctx, stage, fn):
        ctx.profile(True)
        for _ in range(warm):
            fn()
        ctx.synchronize()
        tot = 0.0
        for _ in range(reps):
            fn()
            ctx.synchronize()
            tot += ctx.profile_read()[0][stage]
        ctx.profile(False)
        return tot / reps

    rows = {}
    n = args.n if args.n is not None else 50_000
    T = args.trees if args.trees is not None else 1000
    X, y, f, grow_s = make_forest(n, T, 0, 1, lambda: None)
    ctx = abi.Context(0)
    ctx.load(f, X, y)
    L = n * (n + 1) // 2
    S = torch.empty(L, dtype=torch.int32, device=dev)
    ctx.proximity_upper(S)
    ctx.synchronize()
    # SM clocks and throttle reasons sampled over the n = 50,000 rows below
    clocks = Clocks(0)
    clocks.start()
    for full in (True, False):
        P = torch.empty((n, n) if full else (L,), dtype=torch.float32, device=dev)
        ms = timed(ctx, "finishprox", lambda: ctx.finishprox(S, P, full=full))
        nbytes = 4 * L + 4 * (n * n if full else L) + 4 * n
        rows["finishprox_full" if full else "finishprox_upper"] = {
            "ms": ms, "alg_bytes": nbytes, "achieved_gbs": nbytes / ms / 1e6, "frac": nbytes / ms / 1e6 / hbm,
            "unit": "bytes: S read 4 B + P write 4 B per entry"}
        del P
    # test set: the training rows with Gaussian noise on the continuous columns
    rng = np.random.default_rng(7)
    Xt = X.copy()
    Xt[:, :10] += rng.normal(0.0, 0.5, size=(n, 10)).astype(np.float32)
    Xt_d = torch.from_numpy(Xt).to(dev)
    votes = torch.empty((n, f.nclass), dtype=torch.int32, device=dev)
    ms = timed(ctx, "predict", lambda: ctx.predict_votes(Xt_d, votes))
    walks = n * T
    nbytes = 4 * n * f.p + 4 * n * f.nclass + 16 * int(f.offs[-1])
    rows["predict"] = {"ms": ms, "walks_per_s": walks / ms * 1e3, "alg_bytes": nbytes,
                       "achieved_gbs": nbytes / ms / 1e6, "frac": nbytes / ms / 1e6 / hbm,
                       "unit": "walk = one (test row, tree); bytes: X rows + votes + one pass over the 16-byte nodes"}
    if not args.no_mds:
        Pd = torch.empty((n, n), dtype=torch.float32, device=dev)
        ctx.finishprox(S, Pd, full=True)
        del S
        coords = torch.empty((n, 3), dtype=torch.float64, device=dev)
        ms = timed(ctx, "mds_full", lambda: ctx.mds3d_full(Pd, coords))
        rows[f"mds_full_n{n}"] = {"ms": ms, "unit": "whole call: centring into an n x n FP64 matrix, subspace "
                                                    "iteration for the top 3 eigenpairs"}
        del Pd, coords
    ctx.close()
    clk = clocks.stop()  # (the n = 2,000 case below grows its forest on the host first)
    if args.no_mds:
        line = {"metric": "per-row device time (finishprox, predict)", "value": rows["finishprox_full"]["ms"],
                "unit": f"ms (finishprox full, n={n})", "higher_is_better": False, "n_gpus": 1, "steps": reps,
                "warmup": warm, "dtype": "int32 counts, fp64 normalisation, fp32 outputs",
                "data": "synthetic (seeded cover-shaped generator)",
                "config": {"workload": f"rows a5/a9: finishprox, predict at n={n} ntree={T}",
                           "forest_grow_s": round(grow_s, 2), "peak_hbm_gbs": hbm, "peak_source": peak_src},
                "rows": rows, "clocks": clk}
        print(json.dumps(line), flush=True)
        return 0
    X1, y1 = synth.gaussian_classes(2000, 13, 3)
    f1 = abi.grow_forest(X1, y1, 500, 3, 1, nclass=3)
    ctx = abi.Context(0)
    ctx.load(f1, X1, y1)
    n1 = f1.n
    S1 = torch.empty(n1 * (n1 + 1) // 2, dtype=torch.int32, device=dev)
    ctx.proximity_upper(S1)
    P1 = torch.empty((n1, n1), dtype=torch.float32, device=dev)
    ctx.finishprox(S1, P1, full=True)
    c1 = torch.empty((n1, 3), dtype=torch.float64, device=dev)
    ms = timed(ctx, "mds_full", lambda: ctx.mds3d_full(P1, c1))
    rows["mds_full_n2000"] = {"ms": ms, "unit": "whole call, n = 2,000, 500 trees"}
    ctx.close()
    line = {"metric": "per-row device time (finishprox, predict, full-matrix MDS)", "value": rows["finishprox_full"]["ms"],
            "unit": f"ms (finishprox full, n={n})", "higher_is_better": False, "n_gpus": 1, "steps": reps,
            "warmup": warm, "dtype": "int32 counts, fp64 normalisation and MDS, fp32 outputs",
            "data": "synthetic (seeded cover-shaped and Gaussian generators)",
            "config": {"workload": f"rows a5/a7/a9: finishprox, predict at n={n} ntree={T}; full-matrix 3-D MDS "
                                   f"at n={n} and n=2000", "forest_grow_s": round(grow_s, 2),
                       "peak_hbm_gbs": hbm, "peak_source": peak_src},
            "rows": rows, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """64 independent forests of uneven shape (n in [1000, 50000], p in
    [8, 100] with 30% noise features, 2..10 classes, 300 trees, mtry =
    floor(sqrt(p))): OOB votes and error, exact INT32 pair counts and
    permutation importance for every forest, replayed as one captured CUDA
    graph, against the same work as 64 sequential one-forest runs (each
    synchronised before the next)."""
    import torch

    from rfx_b200 import abi, synth

    count = args.forests
    T = args.trees if args.trees is not None else 300
    specs = synth.uneven_forests(count)
    t0 = time.time()
    forests = []
    for sp in specs:
        f = abi.grow_forest(sp["X"], sp["y"], T, sp["mtry"], 1, nclass=int(sp["y"].max()) + 1)
        forests.append((sp["X"], sp["y"], f))
    grow_s = time.time() - t0
    dev = torch.device("cuda", 0)
    ctxs, items = [], []
    for X, y, f in forests:
        ctx = abi.Context(0)
        ctx.load(f, X, y)
        ctxs.append(ctx)
        n, p, c = f.n, f.p, f.nclass
        z = lambda k, dt=torch.int32: torch.zeros(k, dtype=dt, device=dev)
        items.append(dict(ctx=ctx, impn=False, votes=z(n * c), nout=z(n), oob_error=z(1, torch.float32),
                          oob_pred=z(n), S=z(n * (n + 1) // 2), avimp=z(p, torch.float32),
                          sqsd=z(p, torch.float32)))
    g = abi.BatchGraph(items)  # eager pass + capture
    U = 0
    for ctx in ctxs:
        U += ctx.pair_updates()
    stream = torch.cuda.Stream(device=dev)

    def graph_once():
        g.launch(stream.cuda_stream)

    for _ in range(args.warmup):
        graph_once()
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        graph_once()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    graph_ms = e0.elapsed_time(e1) / args.steps

    # the same work as sequential one-forest runs through the plain entry points
    def sequential_once(lat):
        for it in items:
            ctx = it["ctx"]
            t = time.perf_counter()
            ctx.route_oob(it["votes"], it["nout"])
            ctx.oob_summary(it["oob_error"], it["oob_pred"])
            ctx.proximity_upper(it["S"])
            ctx.varimp(False, it["avimp"], it["sqsd"])
            ctx.synchronize()
            lat.append((time.perf_counter() - t) * 1000.0)

    lat = []
    sequential_once(lat)  # warm-up
    lat = []
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(max(1, min(args.steps, 3))):
        sequential_once(lat)
    seq_ms = (time.perf_counter() - t) * 1000.0 / max(1, min(args.steps, 3))
    g.close()
    for ctx in ctxs:
        ctx.close()
    ns = [f.n for _, _, f in forests]
    line = {"metric": f"batch prox pair-updates/s ({count} uneven forests, one CUDA graph)", "value": U / (graph_ms / 1e3),
            "unit": "pair-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": graph_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic (seeded Gaussian clusters, 30% noise features)",
            "config": {"workload": f"{count} forests: n in [1000, 50000] (sum {sum(ns)}), p in [8, 100], 2..10 "
                                   f"classes, ntree={T}, mtry=floor(sqrt(p)); OOB votes/error, exact INT32 S, "
                                   "permutation importance per forest", "forest_grow_s": round(grow_s, 1),
                       "pair_updates_per_step": U, "l2": "outputs far larger than L2 (S "
                       f"{sum(n * (n + 1) // 2 * 4 for n in ns) / 1e9:.1f} GB per step)"},
            "gpu_launches": g.kernel_nodes,
            "sequential_ms_per_step": seq_ms, "speedup_graph_vs_sequential": seq_ms / graph_ms,
            "per_forest_latency_ms_sequential": {"mean": float(np.mean(lat)), "max": float(np.max(lat))}}
    if clk:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=None, help="samples (default 50000; 200000 for --workload lowrank)")
    ap.add_argument("--trees", type=int, default=None, help="trees (default 1000; 2000 for --workload lowrank)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mds", action="store_true", help="rows workload: finishprox and predict only")
    ap.add_argument("--workload", default="exact", choices=["exact", "lowrank", "large", "batch", "rows"])
    ap.add_argument("--forests", type=int, default=64, help="forests in the batch workload")
    ap.add_argument("--grow-forest", default=None, metavar="PATH",
                    help="grow the exact workload's forest and save it to PATH (used by the forest cache)")
    args = ap.parse_args()
    if args.grow_forest:
        grow_forest_file(args.n or N_SAMPLES, args.trees or N_TREES, args.grow_forest)
        return 0
    if args.workload in ("lowrank", "large"):
        return run_lowrank(args)
    if args.workload == "batch":
        args.warmup = max(args.warmup, 3)
        return run_batch(args)
    if args.workload == "rows":
        return run_rows(args)
    args.n = N_SAMPLES if args.n is None else args.n
    args.trees = N_TREES if args.trees is None else args.trees
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    from rfx_b200 import abi

    X, y, f, grow_s = make_forest(args.n, args.trees, rank, ws, barrier)
    n, p, T = f.n, f.p, f.ntree
    ctx = abi.Context(local)
    ctx.load(f, X, y)
    L = n * (n + 1) // 2
    dev = torch.device("cuda", local)
    S = torch.empty(L, dtype=torch.int32, device=dev)
    avimp = torch.empty(p, dtype=torch.float32, device=dev)
    sqsd = torch.empty(p, dtype=torch.float32, device=dev)
    qimp = torch.empty(n, dtype=torch.float32, device=dev)
    qimpm = torch.empty(n * p, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def step():
        ctx.proximity_upper(S)
        ctx.varimp(True, avimp, sqsd, qimp, qimpm)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    U = ctx.pair_updates()
    ctx.profile(True)
    _, launches0 = ctx.profile_read()
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    ctx.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    stage_ms, launches1 = ctx.profile_read()
    gpu_launches = launches1 - launches0
    ctx.profile(False)
    # whole-job throughput: every replica's pair updates over the slowest replica's time
    ms_max = replica_reduce(ms, "max", dev)
    U_all = replica_reduce(U, "sum", dev)
    value = U_all / (ms_max / 1000.0)

    # roofline of the dominant kernel
    hbm, peak_src = peaks()
    kernels = {k: v for k, v in stage_ms.items() if v > 0}
    # the pair counts of one call are two stages when the hub leaves run on
    # the tensor cores: the hub GEMM (its byte tiles) and the row kernel that
    # starts from them and writes S; the roofline takes them together
    stages = dict(kernels)
    if "pair_hubs" in stages and "pair_counts" in stages:
        stages["pair_counts"] += stages.pop("pair_hubs")
    dom = max(stages, key=stages.get)
    alg_bytes = {
        # S written once + leaf keys read + bag flags read
        "pair_counts": L * 4 + T * n * 4 + T * n * 1,
        # per (tree, sample): bag flag + key written; X rows for OOB walks
        "route": T * n * (1 + 4),
        "leaf_lists": T * n * (4 + 4) * 2,
        # OOB (tree, sample) units: flag byte + flip words written, joob, perm
        "varimp_tree": T * n * (1 + 8 * ((p + 63) // 64)) + 2 * 4 * T * n,
        "varimp_sample": T * n * (1 + 1 + 8 * ((p + 63) // 64)) + n * p * 4,
        "varimp_feature": T * p * 4,
    }
    achieved = alg_bytes.get(dom, 0) / (stages[dom] / 1000.0) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"{dom}_dram.json")
    if os.path.exists(prof):
        with open(prof) as fh:
            d = json.load(fh)
        traffic = d.get("dram_bytes_per_launch_fullsize")
    roofline = {"kernel": dom + (" (hub GEMM + row kernel)" if dom == "pair_counts" and "pair_hubs" in kernels else ""),
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_src,
                "alg_bytes_per_launch": alg_bytes.get(dom, 0), "kernel_ms": stages[dom]}

    line = {"metric": "prox pair-updates/s", "value": value, "unit": "pair-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded mixed-type cover-shaped generator; forest grown by the library's "
                    "restatement of the reference grower)",
            "config": exact_config(n, p, T, U),
            "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU", "forest_obtain_s": round(grow_s, 2),
            "roofline": roofline, "gpu_launches": gpu_launches,
            "breakdown_ms": {k: round(v, 4) for k, v in kernels.items()},
            "tuned_shapes": abi.tuned_shapes()}
    if clk:
        line["clocks"] = clk

    # end to end through the public API with host buffers
    if not args.no_e2e:
        pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
        Sh = pin((L,), torch.int32)
        av_h, sq_h = pin((p,), torch.float32), pin((p,), torch.float32)
        qi_h, qm_h = pin((n,), torch.float32), pin((n * p,), torch.float32)
        Xh = pin(X.shape, torch.float32)
        Xh[...] = X
        yh = pin(y.shape, torch.int32)
        yh[...] = y
        fh = f.subset(range(T))
        for k in ("offs", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass", "nin", "cat"):
            a = getattr(fh, k)
            b = pin(a.shape, {np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32,
                              np.dtype(np.float32): torch.float32}[a.dtype])
            b[...] = a
            setattr(fh, k, b)
        h2d = X.nbytes + y.nbytes + sum(getattr(fh, k).nbytes for k in
                                        ("offs", "nodestatus", "bestvar", "xbestsplit", "treemap", "nodeclass",
                                         "nin", "cat"))
        d2h = Sh.nbytes + av_h.nbytes + sq_h.nbytes + qi_h.nbytes + qm_h.nbytes
        ctx2 = abi.Context(local)

        def e2e_step():
            ctx2.load(fh, Xh, yh)
            ctx2.proximity_upper(Sh)
            ctx2.varimp(True, av_h, sq_h, qi_h, qm_h)

        e2e_step()
        barrier()
        t0 = time.perf_counter()
        ke = max(1, min(args.steps, 3))
        for _ in range(ke):
            e2e_step()
        te = (time.perf_counter() - t0) / ke
        ctx2.close()
        te = replica_reduce(te, "max", dev)
        line["e2e"] = {"value": U_all / te, "unit": "pair-updates/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h), "ms_per_step": te * 1000.0, "steps": ke}

    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, info = cpu_baseline_run(X, y, f, pair_updates=U)
        line["cpu_baseline"] = {"value": v, "unit": "pair-updates/s", "cores": info["cores"], "kind": info["kind"],
                                "sample": info["sample"]}
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
