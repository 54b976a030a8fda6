"""Profile-likelihood bounds on the GPU: inference.profile_bounds driving a
native.Fit (warm-started refits with the profiled coefficient fixed, through
the C ABI) against the reference's CcdInterface::profileModel.  The bounds
agree to the root finder's tolerance (1e-3); the evaluations are the same
objective calls."""
import numpy as np
import pytest

from ccd_b200 import inference, native, synthetic
from ccd_b200.data import GRADIENT, MODEL_LOGISTIC, PRIOR_NORMAL
from oracle import checker

from .golden_io import load_known

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not checker.reference_available(), reason="reference engine not built")]


@pytest.mark.parametrize("make,cols,kw", [
    (lambda: load_known("dobson_dense")[0], [0, 1, 2, 3, 4], {}),
    (lambda: synthetic.small(MODEL_LOGISTIC, seed=161, K=300, P=5, prior=PRIOR_NORMAL), [1, 3],
     dict(override_no_regularization=True, include_penalty=True)),
])
def test_gpu_profile_matches_the_reference(gpu_ctx, make, cols, kw):
    d = make()
    ref = checker.ReferenceEngine(d)
    ref.fit(GRADIENT, 1e-6)
    lo, up, _ = ref.profile(cols, **kw)
    m = native.Matrix(gpu_ctx, d)
    f = native.Fit(gpu_ctx, m, d)
    args = native.ModeFindingArguments(convergence_type=GRADIENT, tolerance=1e-6)
    mode = f.find_mode(args)
    glo, gup, _ = inference.profile_bounds(inference.NativeProfileBackend(f, args), d, cols, **kw)
    assert np.max(np.abs(glo - lo)) <= 2e-3 and np.max(np.abs(gup - up)) <= 2e-3
    # the fit is back at its mode with its own fixed set
    np.testing.assert_allclose(f.get_beta(), mode.beta, rtol=0, atol=0)
