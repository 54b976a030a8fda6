"""The trace summarisers (ccd_b200/trace.py) on synthetic traces in the
engine's file layouts: the level-to-level gaps, spans and phase medians they
report are the ones put in."""
import numpy as np

from ccd_b200 import trace


def test_sweep_trace_summary(tmp_path):
    # two CTAs, three levels; level L opens at 10 us * L + 1 us and ends 6 us later
    segs = np.zeros(4, trace.SEG)
    segs["level"] = [0, 1, 1, 2]
    segs["n_warp"] = [1, 1, 0, 1]
    segs["n_cta"] = [0, 0, 1, 0]
    segs["t0"] = [0, 1, 0, 1]
    cta_seg = np.array([0, 2, 4], np.int64)
    tasks = np.zeros(3, trace.TASK)
    base = 1_000_000
    rows = []
    for L in segs["level"]:
        start = base + 10_000 * L
        rows.append([start, start + 1_000, start + 7_000])
    tr = np.array(rows, np.int64)
    tr2 = np.array([[r[1] + 2_000, r[1] + 5_000] for r in rows], np.int64)
    path = tmp_path / "t.bin"
    with open(path, "wb") as fh:
        fh.write(np.array([len(segs), len(tasks)], np.int64).tobytes())
        fh.write(segs.tobytes())
        fh.write(cta_seg.tobytes())
        fh.write(tasks.tobytes())
        fh.write(tr.astype(np.uint64).tobytes())
        fh.write(tr2.astype(np.uint64).tobytes())
    out = trace.summarise(str(path))
    assert "segments 4, tasks 3, CTAs 2, levels 3" in out
    assert "level-to-level detection: median 4.00 us" in out  # next open (10+1) - previous end (7)
    assert "level span (open -> last arrival): median 6.00 us" in out
    assert "warp-only segments: 3, median phase1 2.00 us, phase2 3.00 us, tail 1.00 us" in out


def test_batch_trace_summary(tmp_path):
    # three columns, phases of 100, 200, 300, 400, 0 SM clocks; columns 1,000 clocks apart
    t = np.array([[c * 1000 + o for o in (1, 101, 301, 601, 1001, 1001)] for c in range(3)], np.int64)
    path = tmp_path / "b.bin"
    t.tofile(path)
    out = trace.summarise_batch(str(path), sm_mhz=1000.0)
    assert "columns traced: 3" in out
    assert "median column 1.00 us" in out
    assert "gather + FP32 terms" in out and "share  20.0%" in out
