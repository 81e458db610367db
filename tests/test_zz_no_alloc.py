"""The allocation-free GLM entry point (ut_glm_logjoint_gradient_noalloc).

It serves callers that cannot allocate device memory when they need a gradient
(a host whose device memory all comes from its own pool or a fixed budget, or a
latency-critical loop that cannot take the synchronisation an allocation may
imply): every buffer comes from the caller and the only scratch is the
library's fixed 16 MiB device array.  This file is collected last so that a run
stopping at the first failure has already run every other test.

Checked here, through the C ABI on a GPU: two calls in a row each agree with
the workspace entry point (ut_logjoint_gradient_device) on the same inputs,
within the density tests' tolerances (logjoint 1e-5 relative, gradient 1e-5 of
the chain's max |g|), and a batch larger than the fixed scratch is rejected.
"""
import numpy as np
import pytest

from uncertaintea_b200 import _native as nat
from uncertaintea_b200.device import DeviceBatchedWorkspace
from uncertaintea_b200.models import BernoulliLogitGLM, logistic_regression_data

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _call(design, y, P, intercept, m, params, totals, grads):
    lib = nat.load()
    return lib.ut_glm_logjoint_gradient_noalloc(
        nat.ptr(design), nat.ptr(y), int(y.shape[0]), P, 1 if intercept else 0, m.intercept_mu, m.intercept_sigma,
        m.coef_mu, m.coef_sigma, nat.ptr(params), int(params.shape[0]), nat.ptr(totals), nat.ptr(grads), None)


@pytest.mark.parametrize("intercept", [True, False])
def test_noalloc_matches_workspace_entry_point_twice(intercept):
    N, D, C = 20_000, 50, 300
    X, y, _ = logistic_regression_data(N, D, 17, x_scale=0.2)
    m = BernoulliLogitGLM(D, intercept=intercept)
    P = m.num_params()
    ws = DeviceBatchedWorkspace(m, C, args=(X,), constraints={"y": y})
    design = np.concatenate([np.ones((N, 1), np.float32), X], axis=1) if intercept else X
    d_design = torch.from_numpy(np.ascontiguousarray(design, dtype=np.float32)).cuda()
    d_y = torch.from_numpy(y.astype(np.float32)).cuda()
    rng = np.random.default_rng(3)
    for call in range(2):
        q = torch.from_numpy(rng.standard_normal((C, P)).astype(np.float32)).cuda()
        ref_t, ref_g = ws.logjoint_gradient_device(q)
        tot = torch.full((C,), float("nan"), device="cuda")
        grd = torch.full((C, P), float("nan"), device="cuda")
        nat.check(_call(d_design, d_y, P, intercept, m, q, tot, grd))
        torch.cuda.synchronize()
        t, g, rt, rg = (x.double().cpu().numpy() for x in (tot, grd, ref_t, ref_g))
        assert np.all(np.isfinite(t)) and np.all(np.isfinite(g)), call
        assert np.max(np.abs(t - rt) / np.abs(rt)) <= 1e-5, call
        scale = np.max(np.abs(rg), axis=1)
        assert np.max(np.max(np.abs(g - rg), axis=1) / scale) <= 1e-5, call
    ws.close()


def test_noalloc_rejects_batches_beyond_the_fixed_scratch():
    P, C = 64, 70_000                       # C * (P + 1) > 4,194,304
    d_design = torch.zeros((8, P), device="cuda")
    d_y = torch.zeros(8, device="cuda")
    q = torch.zeros((C, P), device="cuda")
    tot = torch.zeros(C, device="cuda")
    grd = torch.zeros((C, P), device="cuda")
    m = BernoulliLogitGLM(P)
    status = _call(d_design, d_y, P, False, m, q, tot, grd)
    assert status == nat.UT_ERR_ARGUMENT
    assert "exceeds the fixed scratch" in nat.last_error()
