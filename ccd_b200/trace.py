"""Summarise a sweep timestamp trace written by the engine.

Setting ``CCDB_TRACE_FILE=<path>`` before a fused findMode makes libccdb write,
for the first sweep, the schedule (segments, tasks) and per CTA segment the
global timer at: wait start, level open, end of the CTA-wide phase, end of
the warp phase, arrival.  ``python -m ccd_b200.trace <path>`` prints where the
time of a sweep goes: level-to-level detection, per-level span, and the phase
breakdown by segment kind.

``CCDB_BATCH_TRACE_FILE=<path>`` does the same for the mixed-precision batched
engine: CTA 0's SM clock at six points of every column of one sweep
(``CCDB_BATCH_TRACE_SWEEP``, default 1).  ``python -m ccd_b200.trace --batch
<path> [sm_mhz]`` prints the per-phase breakdown.

The default sweeps write their own formats to the same ``CCDB_TRACE_FILE``
(the last findMode of the process wins):

* ``--cluster <path>``: the cluster sweep, per level and CTA of the first
  sweep the global timer at entry, opening, end of phase A and release;
* ``--group <path>``: the group sweep (Cox), CTA 0's global timer at eight
  points of each of the first 4,096 nonzero steps;
* ``--resident <path> [sm_mhz]``: the resident sweep, SM clock stamps of the
  first 4,096 batches.
"""
from __future__ import annotations

import sys

import numpy as np

SEG = np.dtype([("level", "i4"), ("n_chunk", "i4"), ("n_cta", "i4"), ("n_warp", "i4"), ("t0", "i8")])
TASK = np.dtype([("col", "i4"), ("kind", "i2"), ("warp", "i2"), ("chunk", "i4"), ("nchunks", "i4"),
                 ("part_base", "i4"), ("p0", "i4"), ("p1", "i4"), ("pad", "i4")])


def load(path: str):
    raw = open(path, "rb").read()
    ns, nt = np.frombuffer(raw[:16], np.int64)
    off = 16
    segs = np.frombuffer(raw[off:off + SEG.itemsize * ns], SEG)
    off += SEG.itemsize * ns
    rest = len(raw) - off - TASK.itemsize * nt - 40 * ns
    G = rest // 8 - 1
    cta_seg = np.frombuffer(raw[off:off + 8 * (G + 1)], np.int64)
    off += 8 * (G + 1)
    tasks = np.frombuffer(raw[off:off + TASK.itemsize * nt], TASK)
    off += TASK.itemsize * nt
    allt = np.frombuffer(raw[off:], np.uint64).astype(np.int64)
    return segs, cta_seg, tasks, allt[:3 * ns].reshape(-1, 3), allt[3 * ns:5 * ns].reshape(-1, 2)


def summarise(path: str) -> str:
    segs, cta_seg, tasks, tr, tr2 = load(path)
    ns = len(segs)
    t0 = tr[tr[:, 0] > 0, 0].min()
    tr = tr - t0
    tr2 = np.where(tr2 > 0, tr2 - t0, 0)
    L = segs["level"]
    nl = int(L.max()) + 1
    first = np.full(nl, 1 << 62)
    last = np.zeros(nl, np.int64)
    for i in range(ns):
        first[L[i]] = min(first[L[i]], tr[i, 1])
        last[L[i]] = max(last[L[i]], tr[i, 2])
    gap = first[1:] - last[:-1]
    span = last - first
    out = [f"segments {ns}, tasks {len(tasks)}, CTAs {len(cta_seg) - 1}, levels {nl}",
           f"sweep span {last[-1] / 1e3:.1f} us, {last[-1] / 1e3 / nl:.2f} us per level",
           f"level-to-level detection: median {np.median(gap) / 1e3:.2f} us",
           f"level span (open -> last arrival): median {np.median(span) / 1e3:.2f} us, "
           f"p90 {np.percentile(span, 90) / 1e3:.2f} us"]
    p1 = tr2[:, 0] - tr[:, 1]
    p2 = np.where(tr2[:, 1] > 0, tr2[:, 1] - tr2[:, 0], 0)
    p3 = tr[:, 2] - np.maximum(tr2[:, 0], tr2[:, 1])
    kinds = (("CTA-task segments", (segs["n_cta"] > 0) & (segs["n_warp"] == 0) & (segs["n_chunk"] == 0)),
             ("warp-only segments", (segs["n_warp"] > 0) & (segs["n_cta"] == 0) & (segs["n_chunk"] == 0)),
             ("split-column segments", segs["n_chunk"] > 0))
    for name, sel in kinds:
        if sel.sum():
            out.append(f"{name}: {int(sel.sum())}, median phase1 {np.median(p1[sel]) / 1e3:.2f} us, "
                       f"phase2 {np.median(p2[sel]) / 1e3:.2f} us, tail {np.median(p3[sel]) / 1e3:.2f} us")
    return "\n".join(out)


BATCH_PHASES = ("issue (stage, prefetch, metadata)", "gather + FP32 terms", "group reduction",
                "step + update", "cp.async wait + barrier")


def summarise_batch(path: str, sm_mhz: float = 1965.0) -> str:
    tr = np.fromfile(path, np.int64).reshape(-1, 6)
    cols = np.nonzero(tr[:, 0])[0]
    t = tr[cols]
    per = np.diff(t, axis=1)  # five phases
    span = np.diff(t[:, 0])
    us = 1.0 / sm_mhz
    out = [f"columns traced: {len(cols)}; sweep span {(t[-1, 5] - t[0, 0]) * us / 1e3:.2f} ms; "
           f"median column {np.median(span) * us:.2f} us (mean {span.mean() * us:.2f} us)"]
    for name, col in zip(BATCH_PHASES, per.T):
        out.append(f"  {name:34s} median {np.median(col) * us:7.3f} us  mean {col.mean() * us:7.3f} us  "
                   f"share {col.sum() / per.sum():6.1%}")
    return "\n".join(out)


def summarise_cluster(path: str) -> str:
    """Level timing of the cluster sweep's first sweep."""
    raw = open(path, "rb").read()
    nl, C = (int(v) for v in np.frombuffer(raw[:16], np.int64))
    rest = len(raw) - 16
    J = (rest - nl - 32 * nl * C) // 4
    off = 16 + 4 * J
    split = np.frombuffer(raw[off:off + nl], np.uint8)
    off += nl
    tr = np.frombuffer(raw[off:], np.uint64).reshape(nl, C, 4).astype(np.int64)
    entry, opened, done_a, rel = (tr[..., i] for i in range(4))
    period = np.diff(opened.max(axis=1)) / 1e3
    phase_a = (done_a - opened).max(axis=1) / 1e3
    lag = (opened[1:].max(axis=1) - rel[:-1].max(axis=1)) / 1e3
    plain = split[:-1] == 0
    lines = [f"levels {nl}, CTAs {C}, split levels {int(split.sum())}",
             f"level period median {np.median(period):.2f} us (plain {np.median(period[plain]):.2f}, "
             f"split {np.median(period[~plain]) if (~plain).any() else 0:.2f})",
             f"slowest CTA's phase A median {np.median(phase_a):.2f} us",
             f"last release to every CTA opened median {np.median(lag):.2f} us",
             f"sweep {(rel.max() - opened.min()) / 1e3:.1f} us"]
    return "\n".join(lines)


def summarise_group(path: str) -> str:
    """Per-stage timing of the group sweep's nonzero steps (Cox)."""
    t = np.fromfile(path, dtype=np.uint64).reshape(-1, 8).astype(np.int64)
    t = t[t[:, 0] > 0]
    d = np.diff(t, axis=1) / 1e3
    names = ["gradients of the batch + barrier", "rows + barrier", "denominators + barrier",
             "rebuild phase 1 + barrier", "rebuild phase 2 + barrier", "rebuild phase 3 + barrier"]
    lines = [f"nonzero steps traced {len(t)}"]
    lines += [f"{n}: median {np.median(d[:, i]):.2f} us" for i, n in enumerate(names)]
    lines.append(f"one nonzero step: median {np.median(np.diff(t[:, 0])) / 1e3:.2f} us")
    return "\n".join(lines)


def summarise_resident(path: str, sm_mhz: float = 1965.0) -> str:
    """Per-batch timing of the resident sweep."""
    t = np.fromfile(path, dtype=np.int64).reshape(-1, 8)
    t = t[t[:, 0] != 0]
    long_col = t[:, 5] == -1
    b = t[~long_col]
    us = lambda x: x / sm_mhz
    lines = [f"batches {len(b)}, long columns {int(long_col.sum())}, "
             f"batches ending at a nonzero step {int((b[:, 6] < b[:, 5]).sum())}",
             f"batch median {np.median(us(b[:, 4] - b[:, 0])):.2f} us: gradients "
             f"{np.median(us(b[:, 1] - b[:, 0])):.2f}, decision {np.median(us(b[:, 2] - b[:, 1])):.2f}, "
             f"update {np.median(us(b[:, 3] - b[:, 2])):.2f}, barrier {np.median(us(b[:, 4] - b[:, 3])):.2f}"]
    if long_col.any():
        L = t[long_col]
        lines.append(f"long column median {np.median(us(L[:, 4] - L[:, 0])):.2f} us")
    return "\n".join(lines)


if __name__ == "__main__":
    if sys.argv[1] == "--batch":
        print(summarise_batch(sys.argv[2], *(float(a) for a in sys.argv[3:4])))
    elif sys.argv[1] == "--cluster":
        print(summarise_cluster(sys.argv[2]))
    elif sys.argv[1] == "--group":
        print(summarise_group(sys.argv[2]))
    elif sys.argv[1] == "--resident":
        print(summarise_resident(sys.argv[2], *(float(a) for a in sys.argv[3:4])))
    else:
        print(summarise(sys.argv[1]))
