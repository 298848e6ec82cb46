"""bench.py's reference arm on the CPU: the JSON line a benchmark harness parses (keys, types, the
reference-arm fields) and the silent exit of ranks other than 0 under a multi-rank launch."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    p = _run({"RANK": "0"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 1 and d["warmup"] == 0
    assert d["value"] > 0 and d["higher_is_better"] is True and d["unit"] == "solve/s"
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_silently():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]


def test_near_pair_count_and_interaction_count_are_exact():
    """The bench's exact counts: near-field pairs from the library's leaf sort equal a brute
    force over the leaves and their neighbours; the M2L pairs of a full level equal the
    interaction lists of the oracle's tree."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    from oracle.oracle import Oracle, levsta
    rng = np.random.default_rng(3)
    x = rng.random((3000, 3)) - 0.5
    lev = 3
    g = bench.leaf_counts(x, lev)
    assert g.sum() == 3000
    m = 2 ** lev
    want = 0
    for i in np.ndindex(m, m, m):
        lo = [max(0, a - 1) for a in i]
        hi = [min(m, a + 2) for a in i]
        want += g[i] * g[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]].sum()
    assert bench.near_pairs(g) == want
    tree = Oracle("d").build_tree(x, 4)
    for l in (2, 3, 4):
        assert bench.interactions_per_level(l) == int(tree.iinter[levsta(l):levsta(l + 1)].sum()), l
