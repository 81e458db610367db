"""Statistical gates of the device samplers (the reference's own gate for the
device path, test/uncertaintea/core/device_persistent_nuts.jl:58-139 and
device_chees.jl:43-173): split R-hat, few divergences, and posterior means of
different samplers agreeing within 5 Monte-Carlo standard errors.

R-hat thresholds: 1.01 where the run is long enough for it (NUTS on the GLM,
NUTS on a weakly identified hierarchical model).  Fixed-length HMC and ChEES
on 300 draws per chain reach ~10-30 effective draws per chain on the GLM, and
the non-centred form on informative groups (20 observations per group, large
tau) mixes mu slowly; split R-hat of those runs is bounded at 1.05 / 1.3
instead, with the reason stated at the assertion."""
import numpy as np
import pytest

from uncertaintea_b200 import (BernoulliBeta, BernoulliLogitGLM, HierarchicalNormalNoncentered, LognormalGammaNormal,
                               NormalKnownScale, NormalLocationScale, batched_advi,
                               batched_chees, batched_hmc, batched_meads, batched_nuts, ess, gauss_data, hierarchical_data,
                               logistic_regression_data, rhat, variational_mean, variational_samples)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glm_runs(lib):
    X, y, beta = logistic_regression_data(1000, 10, 1)
    m = BernoulliLogitGLM(10)
    kw = dict(num_chains=256, num_samples=300, num_warmup=300, rng=np.random.default_rng(11))
    hmc = batched_hmc(m, (X,), {"y": y}, step_size=0.05, num_leapfrog_steps=8, **kw)
    kw["rng"] = np.random.default_rng(12)
    nuts = batched_nuts(m, (X,), {"y": y}, **kw)
    kw["rng"] = np.random.default_rng(13)
    chees = batched_chees(m, (X,), {"y": y}, **kw)
    return hmc, nuts, chees


def _mean_mcse(res):
    d = res.constrained
    e = ess(res)
    return d.mean(axis=(0, 1)), d.std(axis=(0, 1)) / np.sqrt(e)


def test_glm_samplers_converge(glm_runs):
    for res in glm_runs:
        assert np.all(np.isfinite(res.constrained))
        assert res.divergent.mean() < 0.01, res.sampler
        # NUTS: 1.01; fixed-length HMC / ChEES with ~10-30 effective draws per chain: 1.05
        limit = 1.01 if res.sampler == "nuts" else 1.05
        assert np.max(rhat(res)) < limit, (res.sampler, rhat(res))


def test_glm_samplers_agree(glm_runs):
    hmc, nuts, chees = glm_runs
    (m1, s1), (m2, s2), (m3, s3) = _mean_mcse(hmc), _mean_mcse(nuts), _mean_mcse(chees)
    assert np.all(np.abs(m1 - m2) <= 5 * np.hypot(s1, s2))
    assert np.all(np.abs(m2 - m3) <= 5 * np.hypot(s2, s3))


def test_chees_adapts_trajectory(glm_runs):
    chees = glm_runs[2]
    assert np.isfinite(chees.trajectory_length) and chees.trajectory_length > 0
    # the step size targets the HARMONIC mean accept (0.651), so the arithmetic mean sits above it
    assert 0.5 < chees.accept_prob.mean() < 0.99


def test_nuts_tree_diagnostics(glm_runs):
    nuts = glm_runs[1]
    assert np.all((nuts.tree_depth >= 1) & (nuts.tree_depth <= 10))
    assert np.all(nuts.integration_steps >= 1)
    assert 0.6 < nuts.accept_prob.mean() < 0.98


def test_hierarchical_nuts_weakly_identified(lib):
    """Eight-schools-like data (one noisy observation per group): the regime the
    non-centred parameterisation is for; NUTS and HMC must agree."""
    y, sig, sizes, _ = hierarchical_data(8, 1, 21, mu_scale=5.0, tau_scale=2.5, sigma_range=(8.0, 16.0))
    m = HierarchicalNormalNoncentered(8)
    res = batched_nuts(m, (sig, sizes), {"y": y}, num_chains=512, num_samples=500, num_warmup=500,
                       rng=np.random.default_rng(5))
    assert np.max(rhat(res)) < 1.01, rhat(res)
    assert res.divergent.mean() < 0.01
    hmc = batched_hmc(m, (sig, sizes), {"y": y}, num_chains=512, num_samples=500, num_warmup=500,
                      num_leapfrog_steps=12, rng=np.random.default_rng(6))
    (m1, s1), (m2, s2) = _mean_mcse(res), _mean_mcse(hmc)
    assert np.all(np.abs(m1 - m2) <= 5 * np.hypot(s1, s2))


def _exact_mu_tau_moments(y, sig, sizes, mu_scale=5.0, tau_scale=2.5):
    """Posterior means of mu and tau with theta integrated out analytically:
    ybar_j | mu, tau ~ N(mu, sqrt(tau^2 + sigma_j^2 / n_j)), on a fine 2-D grid."""
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    ybar = np.array([y[s:s + n].astype(np.float64).mean() for s, n in zip(starts, sizes)])
    se2 = sig.astype(np.float64) ** 2 / sizes
    mu = np.linspace(ybar.mean() - 8, ybar.mean() + 8, 801)[:, None]
    lt = np.linspace(np.log(ybar.std()) - 2.5, np.log(ybar.std()) + 2.5, 801)[None, :]
    tau = np.exp(lt)
    lp = -0.5 * (mu / mu_scale) ** 2 - np.log1p((tau / tau_scale) ** 2) + lt   # prior x |d tau / d log tau|
    for j in range(len(ybar)):
        v = tau ** 2 + se2[j]
        lp = lp - 0.5 * np.log(v) - 0.5 * (ybar[j] - mu) ** 2 / v
    w = np.exp(lp - lp.max())
    w /= w.sum()
    return float((w * mu).sum()), float((w * tau).sum())


def test_hierarchical_nuts_informative_groups(lib):
    """Hierarchical data shape (64 groups x 20 observations, y from the prior at
    seed 7).  The group effects are pinned by the data; mu and tau move slowly
    along the non-centred ridge, so the check is against the exact marginal
    posterior means of mu and tau, within 5 Monte-Carlo standard errors."""
    y, sig, sizes, _ = hierarchical_data(64, 20, 7)
    m = HierarchicalNormalNoncentered(64)
    res = batched_nuts(m, (sig, sizes), {"y": y}, num_chains=1024, num_samples=500, num_warmup=500,
                       rng=np.random.default_rng(5))
    r = rhat(res)
    assert np.max(r[2:]) < 1.02, r[2:]      # theta_j mix fast
    assert res.divergent.mean() < 0.02
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    ybar = np.array([y[s:s + n].mean() for s, n in zip(starts, sizes)])
    theta = res.constrained[:, :, 2:].mean(axis=(0, 1))
    assert np.max(np.abs(theta - ybar)) < 1.0
    mu_ex, tau_ex = _exact_mu_tau_moments(y, sig, sizes)
    mean, mcse = _mean_mcse(res)
    assert abs(mean[0] - mu_ex) <= 5 * mcse[0], (mean[0], mu_ex, mcse[0])
    assert abs(mean[1] - tau_ex) <= 5 * mcse[1], (mean[1], tau_ex, mcse[1])


def _exact_gauss_moments(y, mu_loc=0.0, mu_scale=1.0, shape=2.0, rate=1.0):
    """Posterior means of mu and s of the normal location/scale model on a fine
    2-D grid over (mu, log s)."""
    y = y.astype(np.float64)
    n, ybar, sd = len(y), y.mean(), y.std()
    mu = np.linspace(ybar - 8 * sd / np.sqrt(n) - 1, ybar + 8 * sd / np.sqrt(n) + 1, 1201)[:, None]
    ls = np.linspace(np.log(sd) - 1.5, np.log(sd) + 1.5, 1201)[None, :]
    s = np.exp(ls)
    ss = n * (sd ** 2 + (ybar - mu) ** 2)   # sum_i (y_i - mu)^2
    lp = -0.5 * ((mu - mu_loc) / mu_scale) ** 2 + (shape - 1) * ls - rate * s + ls - n * ls - 0.5 * ss / s ** 2
    w = np.exp(lp - lp.max())
    w /= w.sum()
    return float((w * mu).sum()), float((w * s).sum())


@pytest.mark.parametrize("strategy", ["persistent", "masked"])
def test_gauss_nuts_matches_exact_posterior(lib, strategy):
    """The normal location/scale family (the reference's gaussian scaling model)
    under both device NUTS strategies: R-hat < 1.01 and posterior means of mu and
    s within 5 Monte-Carlo standard errors of the grid-integrated posterior."""
    y, _ = gauss_data(50, 13)
    m = NormalLocationScale()
    res = batched_nuts(m, (50,), {"y": y}, num_chains=512, num_samples=400, num_warmup=400,
                       tree_strategy=strategy, rng=np.random.default_rng(3))
    assert np.max(rhat(res)) < 1.01, rhat(res)
    assert res.divergent.mean() < 0.01
    mu_ex, s_ex = _exact_gauss_moments(y)
    mean, mcse = _mean_mcse(res)
    assert abs(mean[0] - mu_ex) <= 5 * mcse[0], (mean[0], mu_ex, mcse[0])
    assert abs(mean[1] - s_ex) <= 5 * mcse[1], (mean[1], s_ex, mcse[1])


# The reference's conjugate gate (device_persistent_nuts.jl:33-38, device_chees.jl:26-32):
# mu ~ normal(0, 1), y ~ normal(mu, 1) observed at y = 0.3; posterior normal(0.15, sqrt(0.5)).
CONJ_MEAN, CONJ_SD = 0.15, np.sqrt(0.5)


@pytest.mark.parametrize("strategy", ["persistent", "masked"])
def test_conjugate_gauss_nuts_gate(lib, strategy):
    """The reference's persistent-NUTS gate (device_persistent_nuts.jl:58-72; 64
    chains, 1000 draws after 500 warmup): mean and sd within 0.03 of the exact
    posterior, R-hat < 1.01, no divergences -- for both device tree strategies
    (its persistent-vs-masked check, :74-100, compares the same moments)."""
    res = batched_nuts(NormalKnownScale(), (1,), {"y": np.array([0.3])}, num_chains=64, num_samples=1000,
                       num_warmup=500, tree_strategy=strategy, rng=np.random.default_rng(511))
    d = res.constrained[..., 0]
    assert np.all(np.isfinite(d))
    assert abs(d.mean() - CONJ_MEAN) <= 0.03, d.mean()
    assert abs(d.std() - CONJ_SD) <= 0.03, d.std()
    assert np.max(rhat(res)) < 1.01, rhat(res)
    assert res.divergent.sum() == 0


def test_conjugate_gauss_chees_gate(lib):
    """The reference's device ChEES gate (device_chees.jl:45-79; 16 chains, 2000
    draws after 600 warmup, the default trajectory-gradient estimator): mean
    within 0.05 and sd within 0.08 of the exact posterior, R-hat < 1.05, and the
    trajectory length T finite, in (0.5, 200) at the end of warmup, with a tail
    (last 150 warmup iterations) whose max/min ratio is below 3."""
    trace = []
    res = batched_chees(NormalKnownScale(), (1,), {"y": np.array([0.3])}, num_chains=16, num_samples=2000,
                        num_warmup=600, rng=np.random.default_rng(161), _trajectory_trace=trace)
    d = res.constrained[..., 0]
    assert np.all(np.isfinite(d))
    assert abs(d.mean() - CONJ_MEAN) <= 0.05, d.mean()
    assert abs(d.std() - CONJ_SD) <= 0.08, d.std()
    assert np.max(rhat(res)) < 1.05, rhat(res)
    assert len(trace) == 600 and np.all(np.isfinite(trace))
    assert 0.5 < trace[-1] < 200.0, trace[-1]
    tail = np.asarray(trace[-150:])
    assert tail.max() / tail.min() < 3.0


def test_gauss_masked_nuts_stranding_gate(lib):
    """The reference's per-chain stranding gate (device_perchain_stranding.jl):
    normal location/scale with 400 observations (mu 0.3, s 1.2), masked NUTS
    from prior draws with per-chain step sizes and a pooled mass, 64 chains,
    200 warmup + 500 draws: aggregate divergence < 1%, no chain more than 50%
    divergent, posterior mean of s within 0.25 of 1.2, R-hat < 1.2."""
    ys = 0.3 + 1.2 * np.random.default_rng(137).standard_normal(400)
    res = batched_nuts(NormalLocationScale(), (400,), {"y": ys}, num_chains=64, num_samples=500, num_warmup=200,
                       tree_strategy="masked", rng=np.random.default_rng(2024))
    div = np.asarray(res.divergent, dtype=bool)
    assert div.mean() < 0.01, div.mean()
    assert div.mean(axis=1).max() < 0.5
    d = res.constrained
    assert np.all(np.isfinite(d))
    assert abs(d[:, :, 1].mean() - 1.2) <= 0.25, d[:, :, 1].mean()
    assert np.all(rhat(res) < 1.2), rhat(res)


def test_summary_and_warnings_on_device_hmc(lib):
    """The reference's diagnostics test (mcmc_diagnostics_ess_mcse.jl:1-80) on
    device HMC: mu ~ normal(0, 1), y ~ normal(mu, 1) at y = 0.4, 4 chains of
    300 + 300.  MCSE of the mean is sd / sqrt(ess); tail ESS and quantile MCSEs
    are finite; per-chain statistics are opt-in and average to the mean; the
    clean run has no warnings; a step of 16 without adaptation diverges and
    raises them."""
    from uncertaintea_b200 import check_diagnostics, has_warnings, summarize
    m, cons = NormalKnownScale(), {"y": np.array([0.4])}
    ch = batched_hmc(m, (1,), cons, num_chains=4, num_samples=300, num_warmup=300, rng=np.random.default_rng(2024))
    sm = summarize(ch)
    p = sm["parameters"][0]
    assert abs(p["mcse_mean"] - p["sd"] * np.sqrt(1 / p["ess"])) <= 1e-12
    assert np.isfinite(p["mcse_mean"]) and np.isfinite(p["ess_tail"]) and p["ess_tail"] > 0
    assert len(p["mcse_quantiles"]) == len(sm["quantiles"])
    assert all(np.isfinite(v) and v >= 0 for v in p["mcse_quantiles"])
    assert p["per_chain_means"] is None and p["per_chain_sds"] is None
    pc = summarize(ch, per_chain=True)["parameters"][0]
    assert len(pc["per_chain_means"]) == 4 and len(pc["per_chain_sds"]) == 4
    assert abs(np.mean(pc["per_chain_means"]) - pc["mean"]) <= 1e-8
    w = check_diagnostics(ch)
    assert len(w.num_divergent) == 4 and len(w.ebfmi) == 4 and list(w.treedepth_hits) == [0, 0, 0, 0]
    assert w.high_rhat_parameters == [] and w.low_ess_parameters == [] and not has_warnings(w)
    bad = batched_hmc(m, (1,), cons, num_chains=4, num_samples=200, num_warmup=0, step_size=16.0,
                      adapt_step_size=False, adapt_mass_matrix=False, rng=np.random.default_rng(7))
    ws = summarize(bad)["warnings"]
    assert np.any(ws.num_divergent > 0) and has_warnings(ws)


def test_chees_forward_velocity_adapts_trajectory(lib):
    """trajectory_velocity="forward" (the ChEES criterion's own derivative): T
    settles to a finite value with a stable tail (the reference's gate on its
    ChEES T trace, device_chees.jl:70-79) and the posterior agrees with NUTS."""
    X, y, _ = logistic_regression_data(1000, 10, seed=1)
    m = BernoulliLogitGLM(10)
    trace = []
    ch = batched_chees(m, (X,), {"y": y}, num_chains=256, num_samples=400, num_warmup=400,
                       trajectory_velocity="forward", rng=np.random.default_rng(9), _trajectory_trace=trace)
    assert len(trace) == 400 and np.all(np.isfinite(trace))
    tail = np.asarray(trace[-150:])
    assert tail.max() / tail.min() < 3.0
    assert np.max(rhat(ch)) < 1.05
    nuts = batched_nuts(m, (X,), {"y": y}, num_chains=256, num_samples=400, num_warmup=400,
                        rng=np.random.default_rng(10))
    (m1, s1), (m2, s2) = _mean_mcse(ch), _mean_mcse(nuts)
    assert np.all(np.abs(m1 - m2) <= 5 * np.hypot(s1, s2))
    with pytest.raises(ValueError, match="trajectory_velocity"):
        batched_chees(m, (X,), {"y": y}, num_chains=4, num_samples=1, trajectory_velocity="backward")


def test_advi_on_the_gauss_model(lib):
    """Device mean-field ADVI (the reference's device gate, device_hmc_advi.jl:130-147):
    the fitted mean of mu matches the exact posterior mean, the ELBO's last quartile
    beats its first, and the fitted scale of mu is near the posterior SD."""
    y, _ = gauss_data(50, 13)
    m = NormalLocationScale()
    res = batched_advi(m, (50,), {"y": y}, num_iterations=600, num_particles=256, learning_rate=0.05,
                       rng=np.random.default_rng(46))
    assert np.all(np.isfinite(res.elbo_history)) and res.elbo_history.shape == (600,)
    q = len(res.elbo_history) // 4
    assert res.elbo_history[-q:].mean() > res.elbo_history[:q].mean()
    mu_ex, s_ex = _exact_gauss_moments(y)
    mean = variational_mean(res)
    assert abs(mean[0] - mu_ex) < 0.05, (mean, mu_ex)
    assert abs(mean[1] - s_ex) < 0.1 * s_ex, (mean, s_ex)
    sd_mu = np.exp(res.best_log_scale[0])
    assert 0.5 * s_ex / np.sqrt(50) < sd_mu < 2.0 * s_ex / np.sqrt(50)
    draws = variational_samples(res, num_samples=2000, rng=np.random.default_rng(1))
    assert draws.shape == (2, 2000) and np.all(draws[1] > 0)


def test_advi_on_the_glm_matches_nuts_means(lib):
    """On the 1000x10 logistic regression (a near-Gaussian posterior) the mean-field
    location matches the NUTS posterior means within 0.25 posterior SD."""
    X, y, _ = logistic_regression_data(1000, 10, seed=1)
    m = BernoulliLogitGLM(10)
    res = batched_advi(m, (X,), {"y": y}, num_iterations=1500, num_particles=128, learning_rate=0.02,
                       rng=np.random.default_rng(3))
    nuts = batched_nuts(m, (X,), {"y": y}, num_chains=256, num_samples=300, num_warmup=300,
                        rng=np.random.default_rng(4))
    d = nuts.constrained.reshape(-1, 10)
    loc = variational_mean(res)
    assert np.all(np.abs(loc - d.mean(0)) < 0.25 * d.std(0)), (loc, d.mean(0), d.std(0))


def test_meads_on_the_gauss_model(lib):
    """MEADS (no warmup adaptation; the reference's gate on its conjugate model,
    batched_meads.jl:71-98): R-hat, the posterior means of mu and s within 5 MCSE
    of the grid-integrated posterior, finite adaptation trace in range."""
    y, _ = gauss_data(50, 13)
    trace = []
    res = batched_meads(NormalLocationScale(), (50,), {"y": y}, num_chains=256, num_samples=1500, num_warmup=500,
                        rng=np.random.default_rng(11), _adapt_trace=trace)
    assert len(trace) == 2000
    assert all(0.0 < t["step"] <= 1.0 and 0.0 <= t["damping"] <= 1.0 for t in trace)
    assert np.max(rhat(res)) < 1.02, rhat(res)
    assert np.min(ess(res)) > 400
    mu_ex, s_ex = _exact_gauss_moments(y)
    mean, mcse = _mean_mcse(res)
    assert abs(mean[0] - mu_ex) <= 5 * mcse[0], (mean[0], mu_ex, mcse[0])
    assert abs(mean[1] - s_ex) <= 5 * mcse[1], (mean[1], s_ex, mcse[1])
    ist = res.integration_steps
    assert set(np.unique(ist)) <= {0, 1} and abs((ist == 0).mean() - 0.25) < 0.01


def test_meads_on_the_glm_matches_nuts(lib):
    X, y, _ = logistic_regression_data(1000, 10, seed=1)
    m = BernoulliLogitGLM(10)
    res = batched_meads(m, (X,), {"y": y}, num_chains=512, num_samples=1000, num_warmup=500,
                        rng=np.random.default_rng(12))
    assert np.max(rhat(res)) < 1.02
    assert res.divergent.mean() < 0.01
    nuts = batched_nuts(m, (X,), {"y": y}, num_chains=256, num_samples=400, num_warmup=400,
                        rng=np.random.default_rng(13))
    (m1, s1), (m2, s2) = _mean_mcse(res), _mean_mcse(nuts)
    assert np.all(np.abs(m1 - m2) <= 5 * np.hypot(s1, s2))


def test_bernoulli_beta_nuts_matches_the_conjugate_posterior(lib):
    """Beta(2, 3) prior, Bernoulli data: the posterior is Beta(2 + S, 3 + n - S);
    NUTS mean of p within 5 MCSE of it, and MEADS agrees too."""
    z = (np.random.default_rng(17).random(200) < 0.35).astype(np.float32)
    S, n = float(z.sum()), 200
    exact = (2 + S) / (5 + n)
    m = BernoulliBeta()
    res = batched_nuts(m, (n,), {"z": z}, num_chains=512, num_samples=400, num_warmup=400,
                       rng=np.random.default_rng(18))
    assert np.max(rhat(res)) < 1.01
    mean, mcse = _mean_mcse(res)
    assert abs(mean[0] - exact) <= 5 * mcse[0], (mean[0], exact, mcse[0])
    med = batched_meads(m, (n,), {"z": z}, num_chains=256, num_samples=800, num_warmup=400,
                        rng=np.random.default_rng(19))
    mean2, mcse2 = _mean_mcse(med)
    assert abs(mean2[0] - exact) <= 5 * mcse2[0], (mean2[0], exact, mcse2[0])


def test_lognormal_gamma_nuts_matches_grid_posterior(lib):
    """The lognormal/gamma family under NUTS: posterior means of a and b within 5
    MCSE of a fine grid over (log a, log b)."""
    from scipy import stats
    y = (1.5 + 2.0 * np.random.default_rng(21).standard_normal(40)).astype(np.float32).astype(np.float64)
    m = LognormalGammaNormal()
    res = batched_nuts(m, (40,), {"y": y}, num_chains=512, num_samples=400, num_warmup=400,
                       rng=np.random.default_rng(22))
    assert np.max(rhat(res)) < 1.01
    ua = np.linspace(-2.5, 1.5, 801)[:, None]
    ub = np.linspace(-2.0, 1.8, 801)[None, :]
    a, b = np.exp(ua), np.exp(ub)
    s = np.exp(a)
    ss = ((y[None, None, :] - b[..., None]) ** 2).sum(-1)
    lp = (stats.norm(0, 1).logpdf(ua) + stats.gamma(3.0, scale=0.5).logpdf(b) + ub
          - len(y) * a - 0.5 * ss / s ** 2)
    w = np.exp(lp - lp.max())
    w /= w.sum()
    ea, eb = float((w * a).sum()), float((w * b).sum())
    mean, mcse = _mean_mcse(res)
    assert abs(mean[0] - ea) <= 5 * mcse[0], (mean[0], ea, mcse[0])
    assert abs(mean[1] - eb) <= 5 * mcse[1], (mean[1], eb, mcse[1])


def test_seed_reproducibility(lib):
    X, y, _ = logistic_regression_data(200, 3, 4)
    m = BernoulliLogitGLM(3)
    a = batched_nuts(m, (X,), {"y": y}, num_chains=32, num_samples=20, num_warmup=20, rng=np.random.default_rng(3))
    b = batched_nuts(m, (X,), {"y": y}, num_chains=32, num_samples=20, num_warmup=20, rng=np.random.default_rng(3))
    assert np.array_equal(a.unconstrained, b.unconstrained)


def test_argument_validation(lib):
    X, y, _ = logistic_regression_data(50, 2, 4)
    m = BernoulliLogitGLM(2)
    with pytest.raises(ValueError):
        batched_nuts(m, (X,), {"y": y}, num_chains=4, num_samples=5, tree_strategy="hybrid")
    with pytest.raises(ValueError):
        batched_chees(m, (X,), {"y": y}, num_chains=4, num_samples=5, jitter_amount=1.5)
    with pytest.raises(ValueError):
        batched_hmc(m, (X,), {"y": y}, num_chains=4, num_samples=5, precision=np.float64)
    with pytest.raises(ValueError):
        batched_hmc(m, (X,), {"y": y}, num_chains=0, num_samples=5)


def test_masked_nuts_on_the_large_glm(lib):
    """Lockstep NUTS over the tensor-core batched gradient on the 100000x100 design
    (100000 x 100, 256 chains): R-hat < 1.01 and posterior means within 5 MCSE of
    a ChEES run on the same model."""
    X, y, _ = logistic_regression_data(100000, 100, 3, x_scale=0.1)
    m = BernoulliLogitGLM(100)
    nuts = batched_nuts(m, (X,), {"y": y}, num_chains=256, num_samples=300, num_warmup=300, tree_strategy="masked",
                        rng=5)
    assert np.max(rhat(nuts, space="unconstrained")) < 1.01
    chees = batched_chees(m, (X,), {"y": y}, num_chains=256, num_samples=300, num_warmup=300, rng=6)
    a, b = nuts.unconstrained.reshape(-1, 100), chees.unconstrained.reshape(-1, 100)
    ea, eb = ess(nuts, space="unconstrained"), ess(chees, space="unconstrained")
    se = np.sqrt(a.var(0) / ea + b.var(0) / eb)
    assert np.all(np.abs(a.mean(0) - b.mean(0)) < 5 * se)
    assert nuts.tree_depth.min() >= 1 and nuts.gradient_evaluations > 0


def _mixing(draws_sc_p):
    """Min bulk ESS per draw and max rank-normalised R-hat of (S, C, P) draws
    (the reference's estimators, diagnostics.jl:550-612)."""
    import torch
    from uncertaintea_b200.multi import rank_split_rhat, split_ess
    x = torch.from_numpy(np.ascontiguousarray(draws_sc_p, dtype=np.float64))
    S, C, _ = x.shape
    return float(split_ess(x).min()) / (S * C), float(rank_split_rhat(x).max())


@pytest.mark.parametrize("config", [1, 2])
def test_slow_mixing_is_the_models_not_the_devices(lib, config):
    """Configs 1 and 2 fail the R-hat < 1.01 gate after 1000 + 1000 iterations.
    The oracle's own sampler -- an independent CPU restatement of the same
    iteration, here with other random streams -- runs 64 chains for 600
    iterations from the device run's post-warmup positions with the device's
    adapted mass and steps.  Its mixing (min ESS per draw) matches the device's
    on the same 64 chains and draw count (within a factor of 2.5; both R-hats
    are printed), so the slow mixing belongs to the model, data and settings:
    config 1's fixed trajectory (8 x 0.05) nearly matches half a period of the
    posterior's stiffest direction, and config 2's non-centred form sits on a
    ridge of informative groups."""
    import oracle
    C, S = 64, 600
    if config == 1:
        X, y, _ = logistic_regression_data(1000, 10, seed=1)
        m, args, cons = BernoulliLogitGLM(10), (X,), {"y": y}
        ch = batched_hmc(m, args, cons, num_chains=256, num_samples=S, num_warmup=1000, step_size=0.05,
                         num_leapfrog_steps=8, adapt_step_size=False, rng=1)
    else:
        yh, sig, sizes, _ = hierarchical_data(64, 20, 7)
        m, args, cons = HierarchicalNormalNoncentered(64), (sig, sizes), {"y": yh}
        ch = batched_nuts(m, args, cons, num_chains=512, num_samples=S, num_warmup=1000, max_tree_depth=10, rng=7)
    dev = ch.unconstrained[:C].transpose(1, 0, 2)                  # (S, C, P) of the first 64 chains
    om = oracle.OracleModel(m.lower(args, cons))
    q = np.ascontiguousarray(ch.unconstrained[:C, 0, :], dtype=np.float32)
    t, g = om.logjoint_gradient_f32(q)
    im = np.asarray(ch.inverse_mass_matrix, dtype=np.float32).reshape(-1)
    step = np.ascontiguousarray(np.asarray(ch.step_size, dtype=np.float32)[:C])
    draws = np.empty((S, C, q.shape[1]))
    for it in range(S):
        coord = 900_000 + it                                        # streams the device run never used
        if config == 1:
            om.hmc_iteration(q, g, t, im, step, 8, coord)
        else:
            om.nuts_iteration(q, g, t, im, step, 10, coord)
        draws[it] = q
    e_dev, r_dev = _mixing(dev)
    e_orc, r_orc = _mixing(draws)
    print(f"config {config}: device ESS/draw {e_dev:.4g} R-hat {r_dev:.4f}; "
          f"oracle ESS/draw {e_orc:.4g} R-hat {r_orc:.4f}")
    assert 1 / 2.5 < e_orc / e_dev < 2.5, (e_dev, e_orc, r_dev, r_orc)
