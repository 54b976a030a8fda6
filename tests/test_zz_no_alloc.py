"""The allocation-free gradient entry point (ccdb_column_gradient_hessian_noalloc).

It serves callers that cannot allocate device memory -- code running inside a
CUDA graph capture, hosts whose device memory belongs to a pool they must not
grow, embedders given a fixed arena.  This test gives it device buffers it did
not allocate (made here with torch), calls it through the C ABI twice in a row
for every column, and checks each result against the regular entry point
(ccdb_compute_gradient_hessian) on the same state, within the gradient
tolerance the other GPU tests use.  The file sorts last so that a run stopping
at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import DENSE, INTERCEPT, MODEL_LOGISTIC, MODEL_POISSON, SPARSE

pytestmark = pytest.mark.gpu

GH_TOL = 1e-10


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("model,kw", [
    (MODEL_LOGISTIC, dict(seed=90, K=700, P=12)),
    (MODEL_POISSON, dict(seed=91, K=500, P=9, formats=("sparse", "dense", "indicator"))),
])
def test_noalloc_matches_regular_entry_point(gpu_ctx, model, kw, weighted):
    """weighted: random non-negative row weights (zeros included), the
    cross-validation case, against the regular entry point on a weighted fit."""
    import torch
    d = synthetic.small(model, **kw)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    rng = np.random.default_rng(5)
    w = np.where(rng.random(d.K) < 0.2, 0.0, rng.uniform(0.2, 2.0, d.K)) if weighted else np.ones(d.K)
    if weighted:
        f.set_weights(w)
    beta = rng.normal(0, 0.2, size=d.J)
    f.set_beta(beta)
    want = np.array([f.compute_gradient_and_hessian(j) for j in range(d.J)])

    # the same state, in buffers the caller owns: {xBeta, e, denominator, weight} per row
    xb = torch.tensor(f.get_xbeta(), dtype=torch.float64, device="cuda")
    e = torch.exp(xb)
    denom = (1.0 + e) if model == MODEL_LOGISTIC else e.clone()
    state = torch.stack([xb, e, denom, torch.tensor(w, dtype=torch.float64, device="cuda")],
                        dim=1).contiguous()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = native.lib()
    for j in range(d.J):
        fmt = int(d.fmt[j])
        r = d.rows[d.col_start[j]:d.col_start[j + 1]]
        v = d.vals[d.val_start[j]:d.val_start[j + 1]]
        n = d.K if fmt in (DENSE, INTERCEPT) else len(r)
        rows_t = torch.tensor(r, dtype=torch.int32, device="cuda") if len(r) else None
        vals_t = torch.tensor(v, dtype=torch.float64, device="cuda") if len(v) else None
        if fmt in (DENSE, INTERCEPT):
            x = v if fmt == DENSE else np.ones(d.K)
            xjy = float(np.sum(x * d.y * w))
        else:
            x = v if fmt == SPARSE else np.ones(len(r))
            xjy = float(np.sum(x * d.y[r] * w[r]))
        for call in range(2):  # two calls in a row share (and overwrite) the scratch
            out.zero_()
            rc = lib.ccdb_column_gradient_hessian_noalloc(
                model, fmt, n, C.c_void_p(rows_t.data_ptr() if rows_t is not None else 0),
                C.c_void_p(vals_t.data_ptr() if vals_t is not None else 0), C.c_void_p(state.data_ptr()),
                xjy, C.c_void_p(out.data_ptr()), stream)
            assert rc == native.OK, lib.ccdb_last_error()
            torch.cuda.current_stream().synchronize()
            g, h = out.tolist()
            g0, h0 = want[j]
            assert abs(g - g0) <= GH_TOL * max(1.0, abs(g0)), (j, call, g, g0)
            assert abs(h - h0) <= GH_TOL * max(1.0, abs(h0)), (j, call, h, h0)


def test_noalloc_rejects_columns_beyond_its_scratch(gpu_ctx):
    import torch
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    state = torch.zeros(4, dtype=torch.float64, device="cuda")
    lib = native.lib()
    rc = lib.ccdb_column_gradient_hessian_noalloc(MODEL_LOGISTIC, INTERCEPT, (1 << 24) + 1, None, None,
                                                  C.c_void_p(state.data_ptr()), 0.0,
                                                  C.c_void_p(out.data_ptr()), None)
    assert rc == native.ERR_INVALID
    assert b"scratch" in lib.ccdb_last_error()
