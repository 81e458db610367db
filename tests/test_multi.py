"""Uneven batching: many hierarchical models in one batched persistent-NUTS
launch (no counterpart in the reference).

CPU: the warmup action schedule and the device split-ESS against the
reference-restated estimator.  GPU (through the C ABI): one multi-model NUTS
iteration against the oracle's per-model NUTS (same Philox keys: chain c of a
model is keyed by its global chain index), bitwise independence of the launch
configuration, graph replay and the autotuner, and an end-to-end run.

Tolerances: the NUTS iteration as the single-model parity test (the same
tree depth, step count, moved and divergent flags for >= 95% of chains; their
positions within rtol 1e-3, atol 1e-3).  Configurations, graph replay and
autotuning: bit-identical states.
"""
import numpy as np
import pytest

import oracle
from uncertaintea_b200.diagnostics import _split_chain_draws, _split_ess_of
from uncertaintea_b200.models import HierarchicalNormalNoncentered, hierarchical_data
from uncertaintea_b200.multi import ACT_FINAL, ACT_WELFORD, ACT_WINDOW_END, split_ess, warmup_actions


def _models(spec, seed=0, sigma_range=(0.5, 2.0)):
    """spec: list of (J, group sizes) -> [(model, args, constraints)]."""
    out = []
    for i, (J, sizes) in enumerate(spec):
        y, sig, sz, _ = hierarchical_data(J, sizes, seed + i, sigma_range=sigma_range)
        out.append((HierarchicalNormalNoncentered(J), (sig, sz), {"y": y}))
    return out


def _near_mode(model_args, C, rng):
    (m, (sig, sizes), cons) = model_args
    y = cons["y"]
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    ybar = np.array([y[s:s + n].mean() if n > 0 else 0.0 for s, n in zip(starts, sizes)])
    mu0, tau0 = ybar.mean(), max(ybar.std(), 0.1)
    q = np.empty((C, m.num_groups + 2), dtype=np.float32)
    q[:, 0] = mu0 + 0.1 * rng.standard_normal(C)
    q[:, 1] = np.log(tau0) + 0.02 * rng.standard_normal(C)
    q[:, 2:] = (ybar - mu0) / tau0 + 0.05 * rng.standard_normal((C, m.num_groups))
    return q


# ------------------------------------------------------------------ CPU -----
def test_warmup_actions_follow_the_windowed_schedule():
    from uncertaintea_b200.inference import _warmup_schedule
    for W in (0, 1, 15, 150, 1000):
        a = warmup_actions(W)
        assert a.shape == (W,)
        if W == 0:
            continue
        s = _warmup_schedule(W)
        ends = np.nonzero(a & ACT_WINDOW_END)[0] + 1
        assert list(ends) == list(s.slow_window_ends)
        assert a[-1] & ACT_FINAL and not np.any(a[:-1] & ACT_FINAL)
        if s.slow_window_ends:
            wel = np.nonzero(a & ACT_WELFORD)[0] + 1
            assert wel[0] == s.initial_buffer + 1 and wel[-1] == s.slow_window_ends[-1]
            assert len(wel) == s.slow_window_ends[-1] - s.initial_buffer


def test_split_ess_matches_the_reference_estimator():
    torch = pytest.importorskip("torch")
    r = np.random.default_rng(0)
    for S, C, P, phi in [(101, 4, 3, 0.7), (200, 8, 5, -0.3), (37, 3, 2, 0.95), (64, 16, 4, 0.0)]:
        x = np.zeros((S, C, P))
        x[0] = r.standard_normal((C, P))
        for s in range(1, S):
            x[s] = phi * x[s - 1] + r.standard_normal((C, P))
        got = split_ess(torch.from_numpy(x)).numpy()
        ref = np.array([_split_ess_of(_split_chain_draws(x[:, :, p].T)) for p in range(P)])
        np.testing.assert_allclose(got, ref, rtol=1e-10)


# ------------------------------------------------------------------ GPU -----
SPEC = [(3, [4, 0, 7]), (40, 12), (100, 5), (300, np.arange(300) % 9 + 1)]
CHAINS = [8, 5, 12, 6]


@pytest.mark.gpu
def test_multi_nuts_iteration_vs_oracle(lib):
    torch = pytest.importorskip("torch")
    from uncertaintea_b200.multi import MultiModelBatch
    models = _models(SPEC, seed=3)
    batch = MultiModelBatch(models, CHAINS, max_tree_depth=6)
    r = np.random.default_rng(1)
    qs = [_near_mode(ma, c, r) for ma, c in zip(models, CHAINS)]
    batch.set_positions(np.concatenate([q.reshape(-1) for q in qs]))
    step, seed = 0.02, 777
    batch.begin(0, 4, seed, initial_step=step, draws_capacity=0)  # no warmup: no step search, no adaptation
    v = batch.view()
    pos0 = v["position"].cpu().numpy().copy()
    grad0 = v["gradient"].cpu().numpy().copy()
    lj0 = v["logjoint"].cpu().numpy().copy()
    batch.run(1, use_graph=False)
    torch.cuda.synchronize()
    v = batch.view()
    pos1 = v["position"].cpu().numpy()
    depth, acc = v["tree_depth"].cpu().numpy(), v["accept_prob"].cpu().numpy()
    same_all = []
    for m, (ma, C) in enumerate(zip(models, CHAINS)):
        P = int(batch.P[m])
        a, b = int(batch.state_offsets[m]), int(batch.state_offsets[m + 1])
        c0, c1 = int(batch.chain_offsets[m]), int(batch.chain_offsets[m + 1])
        om = oracle.OracleModel(ma[0].lower(ma[1], ma[2]))
        q = pos0[a:b].reshape(C, P).copy()
        g = grad0[a:b].reshape(C, P).copy()
        t = lj0[c0:c1].copy()
        # the device's starting logjoint and gradient agree with the oracle's
        t64, g64 = om.logjoint_gradient_f64(q)
        assert np.max(np.abs(t - t64) / np.abs(t64)) < 1e-5
        ref = om.nuts_iteration(q, g, t, np.ones(P), np.full(C, step), 6, seed, chain_key_offset=c0)
        same = depth[c0:c1] == ref["tree_depth"]
        same &= v["divergent"].cpu().numpy()[c0:c1] == ref["divergent"]
        same &= v["integration_steps"].cpu().numpy()[c0:c1] == ref["integration_steps"]
        np.testing.assert_allclose(pos1[a:b].reshape(C, P)[same], q[same], rtol=1e-3, atol=1e-3)
        np.testing.assert_allclose(acc[c0:c1][same], ref["accept_prob"][same], atol=1e-3)
        same_all.append(same)
    assert np.concatenate(same_all).mean() >= 0.95
    batch.close()


def _run_state(models, chains, iters, config=None, use_graph=True, autotune_at=None, seed=11):
    torch = pytest.importorskip("torch")
    from uncertaintea_b200.multi import MultiModelBatch
    batch = MultiModelBatch(models, chains, max_tree_depth=8)
    r = np.random.default_rng(5)
    qs = [_near_mode(ma, c, r) for ma, c in zip(models, np.broadcast_to(chains, (len(models),)))]
    batch.set_positions(np.concatenate([q.reshape(-1) for q in qs]))
    if config is not None:
        for k in range(8):
            batch.configure(k, *config)
    batch.begin(6, iters - 6, seed, initial_step=0.05)
    if autotune_at is None:
        batch.run(iters, use_graph)
    else:
        batch.run(autotune_at, use_graph)
        before = batch.view()["position"].clone()
        timings = batch.autotune(2)
        assert torch.equal(before, batch.view()["position"])  # the trials leave the state as it was
        assert np.all(timings[batch.class_info()["chains"] > 0] > 0)
        batch.run(iters - autotune_at, use_graph)
    torch.cuda.synchronize()
    v = batch.view()
    out = {k: v[k].cpu().numpy().copy() for k in ("position", "step", "inverse_mass", "draws", "tree_depth")}
    batch.close()
    return out


@pytest.mark.gpu
def test_multi_results_do_not_depend_on_configuration_graph_or_autotuning(lib):
    models = _models(SPEC + [(64, 20), (520, 3)], seed=9)
    chains = [4, 7, 3, 5, 6, 2]
    ref = _run_state(models, chains, 14, config=(1, 0), use_graph=False)
    for kwargs in (dict(config=(4, 204800), use_graph=True), dict(config=(2, 204800), use_graph=False),
                   dict(config=None, use_graph=True, autotune_at=3)):
        got = _run_state(models, chains, 14, **kwargs)
        for k in ref:
            assert np.array_equal(ref[k], got[k]), (kwargs, k)


@pytest.mark.gpu
def test_batched_nuts_multi_end_to_end(lib):
    """Six weakly identified models (few observations per group, noisy
    groups: the regime the non-centred form suits) of different sizes and
    chain counts: every model mixes (R-hat < 1.1 after 300 draws, about 1.01
    as the single-model sampler gets on the same models), a model has a
    time-to-R-hat exactly when its R-hat fell below 1.01 at a checkpoint, and
    its posterior mean of mu agrees with a single-model batched_nuts run
    within 5 combined Monte-Carlo standard errors."""
    from uncertaintea_b200 import batched_nuts, batched_nuts_multi
    spec = [(8, 3), (30, [1, 2, 4] * 10), (64, 2), (120, 3), (250, 2), (400, 1)]
    models = _models(spec, seed=21, sigma_range=(4.0, 8.0))
    chains = [64, 32, 64, 48, 64, 64]
    res = batched_nuts_multi(models, chains_per_model=chains, num_warmup=400, num_samples=300, rng=3,
                             rhat_check_every=50)
    assert np.all(res.max_rhat < 1.1), res.max_rhat
    assert np.all(np.isfinite(res.time_to_rhat)[res.max_rhat < 1.01])  # the last checkpoint is the full run
    assert np.all(res.sampling_time_to_rhat <= res.time_to_rhat)
    assert np.all(res.min_ess > 100) and res.aggregate_ess_per_second > 0
    p50, _ = res.time_to_rhat_quantiles()
    assert p50 > 0
    for m in (0, 4):
        mm, args, cons = models[m]
        single = batched_nuts(mm, args, cons, num_chains=64, num_samples=300, num_warmup=400, rng=4)
        a = res.draws(m)[:, :, 0]
        b = single.unconstrained[:, :, 0]
        ea = float(split_ess(__import__("torch").from_numpy(a.T[:, :, None].copy()))[0])
        eb = float(split_ess(__import__("torch").from_numpy(b.T[:, :, None].copy()))[0])
        se = np.sqrt(a.var() / ea + b.var() / eb)
        assert abs(a.mean() - b.mean()) < 5 * se, (m, a.mean(), b.mean(), se)
    res.batch.close()


@pytest.mark.gpu
def test_stopped_model_keeps_its_state(lib):
    """ut_multi_set_stopped: a stopped model's positions, step sizes and
    adaptation state stay as they were through warmup and sampling
    iterations, its later draw rows repeat its last state, and the other
    models' iterations are bitwise those of a run without the stop (each
    chain's Philox key is its global chain index)."""
    torch = pytest.importorskip("torch")
    from uncertaintea_b200.multi import MultiModelBatch
    models = _models(SPEC, seed=4)
    ref = _run_state(models, CHAINS, 14, seed=13)
    batch = MultiModelBatch(models, CHAINS, max_tree_depth=8)
    r = np.random.default_rng(5)
    qs = [_near_mode(ma, c, r) for ma, c in zip(models, CHAINS)]
    batch.set_positions(np.concatenate([q.reshape(-1) for q in qs]))
    batch.begin(6, 8, 13, initial_step=0.05)
    batch.run(4, use_graph=False)
    torch.cuda.synchronize()
    a, b = int(batch.state_offsets[1]), int(batch.state_offsets[2])
    c0, c1 = int(batch.chain_offsets[1]), int(batch.chain_offsets[2])
    p0, p1 = int(batch.param_offsets[1]), int(batch.param_offsets[2])
    v = batch.view()
    before = {k: v[k].cpu().numpy().copy() for k in ("position", "step", "inverse_mass")}
    batch.set_stopped(np.array([0, 1, 0, 0], dtype=np.uint8))
    batch.run(10, use_graph=True)
    torch.cuda.synchronize()
    v = batch.view()
    after = {k: v[k].cpu().numpy() for k in ("position", "step", "inverse_mass")}
    assert np.array_equal(after["position"][a:b], before["position"][a:b])
    assert np.array_equal(after["step"][c0:c1], before["step"][c0:c1])
    assert np.array_equal(after["inverse_mass"][p0:p1], before["inverse_mass"][p0:p1])
    d = v["draws"].cpu().numpy()
    assert np.all(d[:, a:b] == before["position"][a:b][None, :])   # all 8 draws follow the stop
    others = np.ones(ref["position"].shape[0], dtype=bool)
    others[a:b] = False
    assert np.array_equal(after["position"][others], ref["position"][others])
    batch.close()


@pytest.mark.gpu
def test_per_model_stopping_run(lib):
    """batched_nuts_multi(stop_converged=True): converged models stop at the
    checkpoint that confirmed R-hat < 1.01 (rank-normalised, over their own
    draws), the others run to the cap, and each model's summary covers its
    own draws only."""
    from uncertaintea_b200 import batched_nuts_multi
    easy = _models([(8, 3), (30, 2), (64, 2)], seed=21, sigma_range=(4.0, 8.0))
    hard = _models([(200, 60)], seed=2, sigma_range=(0.5, 0.6))  # informative: slow in the non-centred form
    models = easy + hard
    cap = 400
    res = batched_nuts_multi(models, chains_per_model=32, num_warmup=300, num_samples=cap, rng=5,
                             rhat_check_every=50, stop_converged=True)
    own = res.draws_per_model
    stopped = np.isfinite(res.time_to_rhat)
    assert stopped[:3].any() and not stopped[3], res.max_rhat
    assert np.all(own[stopped] % 50 == 0) and np.all(own[stopped] <= cap)
    assert np.all(res.max_rhat[stopped] < 1.01)
    assert np.all(own[~stopped] == own.max())
    if (~stopped).any():
        assert own.max() == cap
    d = res.batch.view()["draws"].cpu().numpy()
    for m in np.flatnonzero(stopped & (own < own.max())):
        a, b = int(res.batch.state_offsets[m]), int(res.batch.state_offsets[m + 1])
        assert np.all(d[own[m]:own.max(), a:b] == d[own[m] - 1, a:b][None, :])
    res.batch.close()


@pytest.mark.gpu
def test_multi_validation(lib):
    from uncertaintea_b200 import BernoulliLogitGLM, logistic_regression_data
    from uncertaintea_b200.multi import MultiModelBatch
    X, y, _ = logistic_regression_data(50, 3, seed=0)
    with pytest.raises(ValueError):
        MultiModelBatch([(BernoulliLogitGLM(3), (X,), {"y": y})], 4)
    with pytest.raises(ValueError):
        MultiModelBatch(_models([(600, 2)]), 4)  # more than 544 parameters
    with pytest.raises(ValueError):
        MultiModelBatch(_models([(5, 3)]), 0)
    b = MultiModelBatch(_models([(5, 3)]), 4)
    with pytest.raises(ValueError):
        b.run(1)  # before begin
    with pytest.raises(ValueError):
        b.configure(0, 5, 0)
    b.close()
