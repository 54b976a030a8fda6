"""Host logic of native.Fit.fold_instances, over a stand-in for the C library
(no GPU): per instance the fold's weights, the instance's per-column prior
variances, a cold start (the offset at 1), the held-out predictive
log-likelihood only for a successful fit, and the handle left unweighted."""
import ctypes as C

import numpy as np
import pytest

from ccd_b200 import native, synthetic
from ccd_b200.data import MODEL_POISSON


class FakeLib:
    def __init__(self, J, K, flags):
        self.J, self.K, self.flags = J, K, list(flags)
        self.weights, self.fits, self.pred = [], [], []

    def _arr(self, p, n):
        return None if not p else np.ctypeslib.as_array((C.c_double * n).from_address(p)).copy()

    def ccdb_set_weights(self, h, w):
        self.weights.append(self._arr(w.value if isinstance(w, C.c_void_p) else w, self.K))
        return 0

    def ccdb_find_mode(self, h, ma_ref, b, res_ref):
        ma = ma_ref._obj
        pv = self._arr(ma.prior_var, self.J)
        beta = np.ctypeslib.as_array((C.c_double * self.J).from_address(b.value))
        self.fits.append((pv, beta.copy(), self.weights[-1]))
        beta[:] = 0.5  # the "fitted" coefficients
        res = res_ref._obj
        res.return_flag = self.flags.pop(0)
        res.iterations, res.device_seconds = 3, 0.25
        return 0

    def ccdb_get_predictive_log_likelihood(self, h, w, out_ref):
        held = self._arr(w.value if isinstance(w, C.c_void_p) else w, self.K)
        self.pred.append(held)
        out_ref._obj.value = -float(held.sum())
        return 0


@pytest.fixture
def fit(monkeypatch):
    d = synthetic.small(MODEL_POISSON, seed=5, K=40, P=3, offset=True)
    fake = FakeLib(d.J, d.K, flags=[0, 1, 0])
    monkeypatch.setattr(native, "lib", lambda: fake)
    f = native.Fit.__new__(native.Fit)
    f.h, f.d = C.c_void_p(1), d
    yield f, fake, d
    f.h = None  # no handle to release: the library never made one


def test_instances_get_their_folds_variances_and_a_cold_start(fit):
    f, fake, d = fit
    fold = np.arange(d.K) % 3
    var = np.tile(d.prior_var, (3, 1))
    var[:, 1:] = np.array([[0.1], [0.2], [0.3]])
    beta, out, secs = f.fold_instances(var, [0, 1, 2], fold)
    assert len(fake.fits) == 3 and secs == pytest.approx(0.75)
    for i, (pv, start, w) in enumerate(fake.fits):
        np.testing.assert_array_equal(pv, var[i])
        np.testing.assert_array_equal(w, (fold != i).astype(float))
        assert start[0] == 1.0 and not start[1:].any()  # offset fixed at 1, the rest cold
    # held-out LL only where the fit succeeded (flags 0, 1, 0)
    assert [o["flag"] for o in out] == [0, 1, 0]
    assert np.isnan(out[1]["pred_loglik"]) and len(fake.pred) == 2
    np.testing.assert_array_equal(fake.pred[0], (fold == 0).astype(float))
    assert out[0]["pred_loglik"] == -float((fold == 0).sum())
    np.testing.assert_array_equal(beta, 0.5)
    assert fake.weights[-1] is None  # left unweighted


def test_variances_must_be_one_row_per_instance(fit):
    f, _, d = fit
    with pytest.raises(ValueError):
        f.fold_instances(np.ones(d.J), [0], np.zeros(d.K, int))
