"""The serving loop on the GPU: every served result equals the same request
fitted alone (same engine and arguments), bit for bit."""
import numpy as np
import pytest

from ccd_b200 import native, serve, synthetic

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone(gpu_ctx):
    stream = synthetic.serving_stream(12, seed=5, rate=500.0, K_range=(1e3, 5e3), J_range=(50, 400))
    srv = serve.Server(hbm_budget=8e9, slots=4)
    try:
        done = serve.replay(srv, stream)
    finally:
        srv.close()
    assert all(c.error is None for c in done), [c.error for c in done if c.error]
    assert srv.peak_running >= 2  # requests were admitted while others ran
    args = native.ModeFindingArguments()  # the server's default arguments
    alone_ctx = native.Context(0)
    alone_ctx.set_max_ctas(max(1, alone_ctx.sm_count // 4))  # the slots' grid size
    for c, (_, d) in zip(done, stream):
        alone = native.fit_model(alone_ctx, d, args)
        assert c.flag == alone.return_flag and c.iterations == alone.iterations, c.rid
        assert np.array_equal(c.beta, alone.beta), c.rid
    alone_ctx.close()
    s = serve.latency_summary(done)
    assert s["failed"] == 0 and s["p99_s"] >= s["p50_s"] > 0
