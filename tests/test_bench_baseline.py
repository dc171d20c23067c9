"""bench.py's CPU legs on small cases: the forest's pair-update count (the
metric's unit) equals the sum of the oracle's pair counts, and the sampled
per-tree runner accumulates into one array exactly what a whole-forest
analysis does."""
import os
import sys

import numpy as np

from rfx_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _forest(n=600, T=24):
    from rfx_b200 import abi

    X, y = synth.mixed_cover(n, seed=31)
    y = np.unique(y, return_inverse=True)[1].astype(np.int32)
    f = abi.grow_forest(X, y, T, 7, 1, nclass=int(y.max()) + 1, cat=synth.detect_categorical(X))
    return X, y, f


def test_forest_pair_updates_is_the_sum_of_pair_counts(built):
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as orc

    X, y, f = _forest()
    S = orc.analyse(X, y, f, do_imp=False, impn=False, do_prox=True)["S"]
    assert bench.forest_pair_updates(X, y, f) == int(S.astype(np.int64).sum())


def test_sampled_trees_accumulate_the_forest_counts(built):
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as orc

    X, y, f = _forest(n=300, T=10)
    run = bench.CpuTrees(X, y, f)
    for k in range(f.ntree):
        assert run.tree_seconds(k) > 0.0
    assert sorted(run.order.tolist()) == list(range(f.ntree))
    S = orc.analyse(X, y, f, do_imp=False, impn=False, do_prox=True)["S"]
    assert np.array_equal(run.S, S)
    v, info = bench.cpu_baseline_run(X, y, f, budget_s=0.0, min_trees=3)
    assert v > 0 and info["trees"] == 3


def test_reference_arm_prints_the_contract_line(built):
    """`bench.py --impl reference` on a small forest: one JSON line with the
    contract's keys, the reference arm's own e2e and cpu_baseline."""
    import json
    import subprocess

    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "600",
                        "--trees", "8", "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] >= 3
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert "workload" in d["config"]


def test_reference_arm_maps_no_library_of_this_package(built):
    """The reference arm's process runs the reference's build and the oracle
    only: the forest comes from a child process through the numpy loader, so
    librfx_b200.so is never mapped into it; both arms print the same config."""
    import json
    import subprocess

    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--n', '500', '--trees', '6', "
            "'--steps', '2', '--warmup', '3']; sys.path.insert(0, %r); import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'maps_rfx': 'librfx_b200' in maps, 'maps_pyrfx': '_rfx.' in maps}))" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    line, maps = lines[0], lines[-1]
    assert maps == {"maps_rfx": False, "maps_pyrfx": False}
    sys.path.insert(0, ROOT)
    import bench

    X, y, f, _ = bench.cached_forest(500, 6)
    U = bench.forest_pair_updates(X, y, f)
    assert line["config"] == json.loads(json.dumps(bench.exact_config(500, f.p, 6, U)))
