"""bench.py's host side without a GPU: the reference arm's JSON line for a
workload it can run on the host cores, the explicit line for workloads
without a standalone reference arm, and the algorithmic-byte counts behind
the roofline fields."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + list(args), capture_output=True,
                       text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_reference_arm_line_for_the_fisher_workload():
    line = _bench("--impl", "reference", "--workload", "fisher_l1", "--steps", "1", "--warmup", "0")
    assert line["impl"] == "reference" and line["unit"] == "Fisher entries/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] == 1


def test_serve_reference_arm_serves_the_same_trace():
    """The serve reference arm: the reference CPU engine on the first requests
    of the same seeded trace, FIFO over the host threads; p50 latency."""
    line = _bench("--impl", "reference", "--workload", "serve", "--steps", "1", "--warmup", "0")
    assert line["impl"] == "reference" and line["unit"] == "s" and line["value"] > 0
    assert line["higher_is_better"] is False and line["config"]["workload"] == "serve"
    assert line["cpu_baseline"]["kind"] in ("reference", "port")


def test_cv_reference_arm_runs_the_reference_driver():
    """The cv_grid reference arm: the reference's grid-search driver on a
    bounded sample (4 folds at the smallest variance and the refit)."""
    line = _bench("--impl", "reference", "--workload", "cv_grid", "--small", "--steps", "1", "--warmup", "0")
    assert line["impl"] == "reference" and line["unit"] == "fits/s" and line["value"] > 0
    assert line["config"]["workload"] == "cv_grid_small"
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_fisher_and_mm_byte_counts():
    sys.path.insert(0, ROOT)
    import bench
    from ccd_b200.data import INDICATOR, INTERCEPT, MODEL_CONDITIONAL_LOGISTIC, MODEL_LOGISTIC, CyclopsData, build_columns
    K = 10
    cols = [(None, None), (np.array([1, 3], np.int32), None), (np.array([0, 2, 4], np.int32), None)]
    cs, r, vs, v, fm = build_columns(K, cols, [INTERCEPT, INDICATOR, INDICATOR])
    d = CyclopsData(MODEL_LOGISTIC, np.zeros(K), cs, r, vs, v, fm, np.zeros(3, np.int32), np.ones(3))
    idx = np.arange(3, dtype=np.int32)
    # one pass (3 columns < 8 slots): scatter entries x (row id + 8-byte slot) + gather of every column
    ent = np.array([K, 2, 3.0])
    per = np.array([0, 4, 4.0])
    want = float(np.sum(ent * (per + 8)) + np.sum(ent * (per + 64 + 32)))
    assert bench.fisher_bytes(d, idx) == want
    d2 = CyclopsData(MODEL_CONDITIONAL_LOGISTIC, np.zeros(K), cs[1:] - cs[1], r, vs[1:], v, fm[1:],
                     np.zeros(2, np.int32), np.ones(2), stratum=np.zeros(K, np.int64))
    assert bench.mm_cycle_bytes(d2) == 5 * (4 + 16 + 4 + 16)
