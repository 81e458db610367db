"""Warmup adaptation on the device (ut_warmup_adapt, ut_dual_averaging_final)
against the host restatement of the reference's adaptation
(src/inference/nuts/adaptation.jl:1-28, 56-65, 225-260;
hmc_support.jl:635-652): the same step sizes and running-variance weights,
iteration after iteration, for per-chain and shared dual averaging; and a
NUTS run whose warmup adapts on the device against the same run adapting on
the host."""
import numpy as np
import pytest

from uncertaintea_b200 import _native as nat
from uncertaintea_b200.inference import (DualAveraging, _mass_adaptation_weights, _mean_batched_adaptation_probability,
                                         _window_progress)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("per_chain", [True, False])
def test_device_dual_averaging_and_weights_match_the_host(lib, per_chain):
    C, P, window, iters = 300, 7, 50, 40
    r = np.random.default_rng(4)
    steps0 = r.uniform(0.05, 0.3, C) if per_chain else 0.12
    host = DualAveraging(steps0, 0.8)
    from uncertaintea_b200.inference import DeviceDualAveraging
    dev = DeviceDualAveraging(host, "cuda")
    var_state = torch.zeros(2 * P + 3, dtype=torch.float64, device="cuda")
    w_dev = torch.empty(C, dtype=torch.float64, device="cuda")
    step = torch.empty(C, dtype=torch.float32, device="cuda")
    for it in range(iters):
        ap = r.uniform(0, 1, C).astype(np.float32)
        ap[r.random(C) < 0.05] = np.nan
        acc = (r.random(C) < 0.6).astype(np.uint8)
        div = (r.random(C) < 0.05).astype(np.uint8)
        count = float(it * 3)
        var_state[2 * P] = count
        apd, accd, divd = (torch.from_numpy(x).cuda() for x in (ap, acc, div))
        nat.check(lib.ut_warmup_adapt(nat.ptr(apd), nat.ptr(accd), nat.ptr(divd), C, P, nat.ptr(var_state), window,
                                      nat.ptr(w_dev), nat.ptr(dev.state), 1 if per_chain else 0, 1, 0.8,
                                      nat.ptr(step), None))
        torch.cuda.synchronize()
        apd64, dv = ap.astype(np.float64), div.astype(bool)
        stat = np.where(dv, 0.0, apd64) if per_chain else _mean_batched_adaptation_probability(apd64, dv)
        want = np.broadcast_to(host.update(stat), (C,)).astype(np.float32)
        got = step.cpu().numpy()
        if per_chain:
            np.testing.assert_allclose(got, want, rtol=1e-6)
        else:
            # the shared mean sums 300 terms in a different order: float64 last bits
            np.testing.assert_allclose(got, want, rtol=1e-6)
        w_want = _mass_adaptation_weights(_window_progress(int(count), window), acc.astype(bool), apd64, dv)
        np.testing.assert_allclose(w_dev.cpu().numpy(), w_want, rtol=1e-15, atol=0)
    nat.check(lib.ut_dual_averaging_final(nat.ptr(dev.state), C, 1 if per_chain else 0, nat.ptr(step), None))
    torch.cuda.synchronize()
    np.testing.assert_allclose(step.cpu().numpy(), np.broadcast_to(host.final(), (C,)).astype(np.float32), rtol=1e-6)


def test_nuts_warmup_on_the_device_matches_the_host_path(lib):
    """The same NUTS run (seeded) with warmup adapting on the device and on the
    host.  The adaptation arithmetic agrees to the last bits of float64 (the
    test above), but a last-bit difference in one step size sends that chain
    down another trajectory, so individual chains' final step sizes differ;
    their distribution over the 128 chains (median and deciles), the shared
    mass and the posterior means (within 5 MCSE) agree."""
    from uncertaintea_b200 import BernoulliLogitGLM, batched_nuts, ess, logistic_regression_data
    X, y, _ = logistic_regression_data(500, 5, 2)
    kw = dict(num_chains=128, num_samples=300, num_warmup=300, rng=5)
    a = batched_nuts(BernoulliLogitGLM(5), (X,), {"y": y}, device_adaptation=True, **kw)
    b = batched_nuts(BernoulliLogitGLM(5), (X,), {"y": y}, device_adaptation=False, **kw)
    qs = (0.1, 0.5, 0.9)
    np.testing.assert_allclose(np.quantile(a.step_size, qs), np.quantile(b.step_size, qs), rtol=0.1)
    np.testing.assert_allclose(a.inverse_mass_matrix, b.inverse_mass_matrix, rtol=0.2)
    ua, ub = a.unconstrained.reshape(-1, 5), b.unconstrained.reshape(-1, 5)
    mcse = np.sqrt(ua.var(0) / ess(a, space="unconstrained") + ub.var(0) / ess(b, space="unconstrained"))
    assert np.all(np.abs(ua.mean(0) - ub.mean(0)) <= 5 * mcse)
    assert len(a.mass_adaptation_windows) == len(b.mass_adaptation_windows)
