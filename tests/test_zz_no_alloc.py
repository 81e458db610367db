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
the chain's max |g|), and a few chains with the FP64 oracle; the second call
leaves the device's free memory unchanged (nothing is allocated); a batch so
large that the scratch, not the SM count, sets the observation split count
(C * (P + 1) above half of the scratch) agrees too; and a batch larger than the
fixed scratch is rejected.
"""
import numpy as np
import pytest

import oracle
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


def _check_against_workspace_and_oracle(N, D, C, intercept, seed, calls=2):
    X, y, _ = logistic_regression_data(N, D, seed, x_scale=0.2)
    m = BernoulliLogitGLM(D, intercept=intercept)
    P = m.num_params()
    ws = DeviceBatchedWorkspace(m, C, args=(X,), constraints={"y": y})
    om = oracle.OracleModel(ws.lowered)
    design = np.concatenate([np.ones((N, 1), np.float32), X], axis=1) if intercept else X
    d_design = torch.from_numpy(np.ascontiguousarray(design, dtype=np.float32)).cuda()
    d_y = torch.from_numpy(y.astype(np.float32)).cuda()
    rng = np.random.default_rng(3)
    qs = [torch.from_numpy(rng.standard_normal((C, P)).astype(np.float32)).cuda() for _ in range(calls)]
    refs = [ws.logjoint_gradient_device(q) for q in qs]
    tot = torch.empty(C, device="cuda")
    grd = torch.empty((C, P), device="cuda")
    torch.cuda.synchronize()
    for call in range(calls):
        tot.fill_(float("nan"))
        grd.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        nat.check(_call(d_design, d_y, P, intercept, m, qs[call], tot, grd))
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call > 0:
            # the first call on the device did its one-time set-up; later calls
            # leave the device's free memory exactly as it was
            assert free_after == free_before, (call, free_before, free_after)
        (ref_t, ref_g) = refs[call]
        t, g, rt, rg = (x.cpu().double().numpy() for x in (tot, grd, ref_t, ref_g))
        assert np.all(np.isfinite(t)) and np.all(np.isfinite(g)), call
        assert np.max(np.abs(t - rt) / np.abs(rt)) <= 1e-5, call
        scale = np.max(np.abs(rg), axis=1)
        assert np.max(np.max(np.abs(g - rg), axis=1) / scale) <= 1e-5, call
        idx = np.unique(np.linspace(0, C - 1, 6).astype(int))
        t64, g64 = om.logjoint_gradient_f64(qs[call][idx].cpu().double().numpy())
        assert np.max(np.abs(t[idx] - t64) / np.abs(t64)) <= 1e-5, call
        assert np.max(np.max(np.abs(g[idx] - g64), axis=1) / np.max(np.abs(g64), axis=1)) <= 1e-5, call
    ws.close()


@pytest.mark.parametrize("intercept", [True, False])
def test_noalloc_matches_workspace_entry_point_twice(intercept):
    _check_against_workspace_and_oracle(20_000, 50, 300, intercept, 17)


def test_noalloc_split_count_set_by_the_scratch_limit():
    """C * (P + 1) = 40000 * 102 > 4,194,304 / 2: the scratch holds one split's
    partials only, so the observation split count is the scratch's, not the
    SM-count plan's."""
    _check_against_workspace_and_oracle(3_000, 100, 40_000, True, 19)


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
