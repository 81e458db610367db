"""CPU tests of the host-side logic: ChEES scalar helpers (pinned by the
reference's unit tests), warmup schedule, dual averaging, mass weights,
diagnostics."""
import math
import os

import numpy as np
import pytest

from uncertaintea_b200 import inference as inf
from uncertaintea_b200 import diagnostics as dg


def test_chees_steps_from_jitter_pins(pins):
    # batched_chees_adaptation.jl:50-52
    for p in pins["chees"]["steps_from_jitter"]:
        assert inf._chees_leapfrog_steps_from_jitter(p["jitter"], p["trajectory_length"], p["step_size"]) == p["steps"]


def test_chees_jitter_reconciliation():
    # batched_chees_adaptation.jl:27-49
    assert inf._chees_jitter_value(0.0, 1) == 1.0
    assert inf._chees_jitter_value(0.0, 7) == 1.0
    assert inf._chees_jitter_value(1.0, 1) == inf._halton_base2(1)
    for i in range(1, 21):
        assert 0.5 <= inf._chees_jitter_value(0.5, i) <= 1.0
    for L in (1, 3, 10, 12, 37, 100):
        for eps in (0.1, 0.037, 1.6, 0.9):
            assert inf._chees_jittered_leapfrog_steps(L * eps, eps, 0.0, 5) == L


def test_halton_sequence():
    assert [inf._halton_base2(i) for i in range(1, 8)] == [0.5, 0.25, 0.75, 0.125, 0.625, 0.375, 0.875]
    with pytest.raises(ValueError):
        inf._halton_base2(0)


def test_chees_adam_pin(pins):
    # batched_chees_adaptation.jl:55-67
    a = pins["chees"]["adam"]
    adam = inf.ChEESAdamState(a["learning_rate"], a["beta1"], a["beta2"], a["epsilon"])
    u1 = adam.ascend(a["constant_gradient"])
    assert u1 > 0
    for _ in range(200):
        u = adam.ascend(a["constant_gradient"])
    assert abs(u - a["limit"]) <= a["atol"]
    adam2 = inf.ChEESAdamState(a["learning_rate"], a["beta1"], a["beta2"], a["epsilon"])
    assert adam2.ascend(-3.0) < 0


def test_chees_harmonic_mean_pin(pins):
    # batched_chees_adaptation.jl:69-76
    hm = inf._chees_harmonic_mean_accept(pins["chees"]["harmonic_mean_input"], [False, False, False])
    assert abs(hm - pins["chees"]["harmonic_mean_expected"]) < 1e-12
    assert inf._chees_harmonic_mean_accept([0.5, 0.0], [False, True]) == 0.5
    assert inf._chees_harmonic_mean_accept([0.5], [True]) == 0.0


def test_chees_trajectory_update_clip_and_revert():
    traj = inf.ChEESTrajectoryState(1.0, 0.0, inf.ChEESAdamState(0.5, 0.0, 0.95, 1e-8), 1, 0.5, 100)
    t = inf._chees_apply_trajectory_gradient(traj, 1e6, 1.0, 1.0, 0.1)
    assert math.isclose(math.log(t), 0.35, rel_tol=1e-12)  # first step: weight 1, clipped update
    traj2 = inf.ChEESTrajectoryState(5.0, math.log(5.0), inf.ChEESAdamState(0.5, 0.0, 0.95, 1e-8), 1, 0.5, 3)
    assert inf._chees_apply_trajectory_gradient(traj2, 1e6, 1.0, 1.0, 0.1) == pytest.approx(0.3)  # clamp to max*eps
    traj3 = inf.ChEESTrajectoryState(1.0, 0.0, inf.ChEESAdamState(0.5, 0.0, 0.95, 1e-8), 1, 0.5, 10)
    assert inf._chees_apply_trajectory_gradient(traj3, 1.0, 0.0, 1.0, 0.1) == pytest.approx(1.0)  # zero denom


def test_warmup_schedule():
    # adaptation.jl:103-136
    s = inf._warmup_schedule(1000)
    assert s.initial_buffer == 100 and s.terminal_buffer == 100
    assert s.slow_window_ends[0] == 125 and s.slow_window_ends[-1] == 900
    assert inf._warmup_schedule(0).slow_window_ends == []
    s10 = inf._warmup_schedule(10)
    assert s10.initial_buffer == 5 and s10.slow_window_ends == [10]
    s500 = inf._warmup_schedule(500)
    lens = [inf._warmup_window_length(s500, i + 1) for i in range(len(s500.slow_window_ends))]
    assert sum(lens) == 500 - s500.initial_buffer - s500.terminal_buffer
    assert lens[0] == 25


def test_dual_averaging_matches_scalar_recursion():
    da = inf.DualAveraging(np.array([0.1, 0.2]), 0.8)
    mu = math.log(10 * 0.1)
    hbar, lss, avg = 0.0, math.log(0.1), math.log(0.1)
    for it in range(1, 30):
        acc = 0.5 + 0.01 * it
        out = da.update(np.array([acc, acc]))
        eta = 1 / (it + 10.0)
        hbar = (1 - eta) * hbar + eta * (0.8 - acc)
        lss = mu - math.sqrt(it) / 0.05 * hbar
        eb = it ** -0.75
        avg = eb * lss + (1 - eb) * avg
        assert math.isclose(out[0], math.exp(lss), rel_tol=1e-12)
    assert math.isclose(da.final()[0], math.exp(avg), rel_tol=1e-12)


def test_mass_window_summaries_follow_the_reference(monkeypatch):
    """The warmup driver records one summary per slow window with the reference's
    fields (adaptation.jl:143-170) and summarize groups them (diagnostics.jl:411-448).
    The device running-variance update is replaced by a host weighted Welford
    update of the same state layout, so the driver runs on the CPU."""
    P, C, W = 3, 8, 300

    def host_update(self, positions, weights):
        st = self.state.numpy()
        x = np.asarray(positions, dtype=np.float64)
        for c in range(x.shape[0]):
            w = float(weights[c])
            if w <= 0:
                continue
            st[2 * P + 1] += w
            st[2 * P + 2] += w * w
            d = x[c] - st[:P]
            st[:P] += (w / st[2 * P + 1]) * d
            st[P:2 * P] += w * d * (x[c] - st[:P])
        self.count += int(np.count_nonzero(np.asarray(weights) > 0))

    monkeypatch.setattr(inf.DeviceRunningVariance, "update", host_update)
    drv = inf.WarmupDriver(None, P, W, 0.1, 0.8, adapt_step_size=False, adapt_mass_matrix=True,
                           mass_matrix_regularization=1e-3, mass_matrix_min_samples=10, device="cpu")
    rng = np.random.default_rng(0)
    scale = np.array([0.5, 1.0, 3.0])
    for it in range(1, W + 1):
        weights = np.where(np.arange(C) == it % C, 0.5, 1.0)
        drv.warmup_update(it, 0.8, rng.standard_normal((C, P)) * scale, weights, None)
    sched = drv.schedule
    wins = drv.mass_adaptation_windows
    assert [w["window"] for w in wins] == list(range(1, len(sched.slow_window_ends) + 1))
    for i, w in enumerate(wins, start=1):
        start = sched.initial_buffer + 1 if i == 1 else sched.slow_window_ends[i - 2] + 1
        length = sched.slow_window_ends[i - 1] - start + 1
        assert (w["start"], w["end"], w["window_length"]) == (start, sched.slow_window_ends[i - 1], length)
        assert w["samples"] == C * length
        assert w["weight_sum"] == pytest.approx(C * length - 0.5 * length)
        assert w["effective_count"] == pytest.approx(w["weight_sum"] ** 2 / ((C - 1) * length + 0.25 * length))
        assert w["mean_weight"] == pytest.approx(w["weight_sum"] / w["samples"])
        assert w["clip_scale_start"] == 8.0 and w["updated"]
        assert w["mass_min"] <= w["mass_mean"] <= w["mass_max"]
    last = wins[-1]
    mass = 1.0 / drv.inverse_mass_matrix   # the mass the last window left
    assert (last["mass_min"], last["mass_mean"], last["mass_max"]) == pytest.approx(
        (mass.min(), mass.mean(), mass.max()))
    assert np.argmin(drv.inverse_mass_matrix) == 0 and np.argmax(drv.inverse_mass_matrix) == 2   # variances learned

    class Fake:
        mass_adaptation_windows = wins
    groups = dg._mass_adaptation_diagnostics(Fake.mass_adaptation_windows, 4)
    assert [g["window_index"] for g in groups] == [w["window"] for w in wins]
    assert all(g["chains"] == 4 and g["updated_chains"] == 4 for g in groups)
    assert groups[0]["mean_effective_count"] == pytest.approx(wins[0]["effective_count"])


def test_per_chain_step_driver_restarts_at_window_ends(monkeypatch):
    """Shared pooled mass + per-chain dual-averaged steps (warmup.jl:362-473):
    each chain's step follows its own dual-averaging recursion on its own
    acceptance; at every slow-window end before the last warmup iteration the
    step search is re-run with the new mass, and dual averaging restarts from
    the steps it returns; finalisation gives each chain's averaged step."""
    P, C, W = 2, 5, 150

    def host_update(self, positions, weights):
        st = self.state.numpy()
        for c in range(len(weights)):
            st[2 * P + 1] += float(weights[c])
            st[2 * P + 2] += float(weights[c]) ** 2
        st[P:2 * P] += 1.0
        self.count += int(np.count_nonzero(np.asarray(weights) > 0))

    monkeypatch.setattr(inf.DeviceRunningVariance, "update", host_update)
    steps0 = np.array([0.05, 0.1, 0.2, 0.4, 0.8])
    drv = inf.PooledMassPerChainStepDriver(None, P, W, steps0, 0.8, adapt_step_size=True, adapt_mass_matrix=True,
                                           mass_matrix_regularization=1e-3, mass_matrix_min_samples=10,
                                           device="cpu")
    calls = []

    def refind(steps, inverse_mass):
        calls.append(np.array(inverse_mass))
        return np.asarray(steps) * 0.5

    refs = [inf.DualAveraging(np.array([s]), 0.8) for s in steps0]
    ends = set(drv.mass.schedule.slow_window_ends)
    rng = np.random.default_rng(1)
    for it in range(1, W + 1):
        acc = rng.uniform(0.3, 1.0, C)
        got = drv.warmup_update(it, acc, np.zeros((C, P)), np.ones(C), refind)
        want = np.array([refs[c].update(np.array([acc[c]]))[0] for c in range(C)])
        if it in ends and it < W:
            want = want * 0.5
            refs = [inf.DualAveraging(np.array([s]), 0.8) for s in want]
        assert np.allclose(got, want, rtol=1e-12), it
    assert len(calls) == len([e for e in ends if e < W])
    final = drv.warmup_finalize()
    assert np.allclose(final, [r.final()[0] for r in refs], rtol=1e-12)


def test_shared_step_driver_restarts_at_window_ends(monkeypatch):
    """The shared-step warmup driver (warmup.jl:262-330): one dual-averaged step
    on the pooled acceptance, the mass re-estimated at each slow-window end,
    the step re-searched with that mass (before the last warmup iteration) and
    dual averaging restarted from it; finalisation averages."""
    P, C, W = 2, 4, 120

    def host_update(self, positions, weights):
        st = self.state.numpy()
        for c in range(len(weights)):
            st[2 * P + 1] += float(weights[c])
            st[2 * P + 2] += float(weights[c]) ** 2
        st[P:2 * P] += np.array([0.5, 2.0])
        self.count += int(np.count_nonzero(np.asarray(weights) > 0))

    monkeypatch.setattr(inf.DeviceRunningVariance, "update", host_update)
    drv = inf.WarmupDriver(None, P, W, 0.3, 0.8, adapt_step_size=True, adapt_mass_matrix=True,
                           mass_matrix_regularization=1e-3, mass_matrix_min_samples=10, device="cpu")
    seen = []

    def refind(step, inverse_mass):
        seen.append(np.array(inverse_mass))
        return step * 2.0

    ref = inf.DualAveraging(0.3, 0.8)
    ends = set(drv.schedule.slow_window_ends)
    rng = np.random.default_rng(4)
    for it in range(1, W + 1):
        a = float(rng.uniform(0.4, 1.0))
        got = drv.warmup_update(it, a, np.zeros((C, P)), np.ones(C), refind)
        want = float(ref.update(a))
        if it in ends and it < W:
            want *= 2.0
            ref = inf.DualAveraging(want, 0.8)
            assert np.allclose(seen[-1], drv.inverse_mass_matrix)
        assert got == pytest.approx(want, rel=1e-12), it
    assert len(seen) == len([e for e in ends if e < W])
    assert drv.inverse_mass_matrix[1] > drv.inverse_mass_matrix[0]   # the larger second moment
    assert drv.warmup_finalize() == pytest.approx(float(ref.final()), rel=1e-12)


def test_draw_buffer_and_finish_layout():
    """Draws recorded per iteration come back as (chains, samples, ...) arrays,
    constrained through the model's transform, with the run's step sizes and
    mass; the diagnostics read that layout (host assembly on CPU tensors)."""
    import torch
    from uncertaintea_b200.models import NormalLocationScale

    class Run:
        pass

    run = Run()
    run.torch, run.device, run.C, run.P = torch, "cpu", 3, 2
    run.model, run.args, run.constraints = NormalLocationScale(), (4,), {"y": np.zeros(4)}
    for name, dt in (("position", torch.float32), ("logjoint", torch.float32), ("accept_prob", torch.float32),
                     ("energy", torch.float32), ("energy_error", torch.float32), ("accepted", torch.uint8),
                     ("divergent", torch.uint8)):
        setattr(run, name, torch.zeros((3, 2) if name == "position" else 3, dtype=dt))
    draws = inf._DrawBuffer(run, 6)
    for s_ in range(6):
        run.position.copy_(torch.tensor([[s_, 0.1 * s_], [10 + s_, 0.2], [20 + s_, -0.3]], dtype=torch.float32))
        run.logjoint.fill_(-float(s_))
        run.accept_prob.fill_(0.5)
        run.divergent.copy_(torch.tensor([0, s_ == 3, 0], dtype=torch.uint8))
        draws.record(s_, integration_steps=7)
    out = inf._finish("hmc", run, draws, 0.25, np.ones(2), [], 1.0, 2.0)
    assert out.unconstrained.shape == (3, 6, 2) and out.constrained.shape == (3, 6, 2)
    assert out.unconstrained[1, 4, 0] == 14.0 and out.logjoint[2, 5] == -5.0
    assert np.allclose(out.constrained[:, :, 1], np.exp(out.unconstrained[:, :, 1]))
    assert out.divergent.dtype == bool and out.divergent[1, 3] and out.divergent.sum() == 1
    assert np.all(out.integration_steps == 7) and np.all(out.step_size == 0.25)
    assert out.num_chains == 3 and out.num_samples == 6
    assert dg.rhat(out).shape == (2,) and dg.summarize(out)["diagnostics"]["divergence_rate"] == pytest.approx(1 / 18)


@pytest.mark.parametrize("velocity", ["reference", "forward"])
def test_chees_trajectory_adaptation_on_the_conjugate_model(velocity):
    """The reference's ChEES T-trace gate (device_chees.jl:70-79) on the oracle:
    16 chains of the conjugate gauss model (y = 0.3), trajectories and the
    cross-chain reduction from the oracle, the trajectory length adapted by the
    package's Adam update on log T.  T stays finite, ends in (0.5, 200) and its
    last 150 values vary by less than a factor 3, for both trajectory-gradient
    estimators."""
    import math
    import oracle
    from uncertaintea_b200.models import NormalKnownScale
    om = oracle.OracleModel(NormalKnownScale().lower((1,), {"y": np.array([0.3])}))
    C, eps, im = 16, 0.8, np.full(1, 0.5, dtype=np.float32)
    rng = np.random.default_rng(161)
    q = rng.normal(0, 1, size=(C, 1)).astype(np.float32)
    t, g = om.logjoint_gradient_f32(q)
    traj = inf.ChEESTrajectoryState(10 * eps, math.log(10 * eps), inf.ChEESAdamState(0.5, 0.0, 0.95, 1e-8), 1,
                                    0.5, 1000)
    trace = []
    for it in range(1, 401):
        jit = inf._chees_jitter_value(1.0, it)
        L = inf._chees_leapfrog_steps_from_jitter(jit, traj.trajectory_length, eps)
        init = q.copy()
        out = om.hmc_iteration(q, g, t, im, np.full(C, eps, np.float32), L, it, want_proposal=True)
        num, den = oracle.chees_reduce(init, out["proposal"], out["endpoint_momentum"], out["accept_prob"],
                                       out["divergent"], im)
        if velocity == "forward":
            num = -num
        inf._chees_apply_trajectory_gradient(traj, num, den, jit, eps)
        trace.append(traj.trajectory_length)
    trace = np.asarray(trace)
    assert np.all(np.isfinite(trace)) and 0.5 < trace[-1] < 200.0, trace[-1]
    assert trace[-150:].max() / trace[-150:].min() < 3.0
    assert abs(float(q.mean()) - 0.15) < 0.5     # the chains sit in the posterior (sd 0.71)


def test_mass_adaptation_weights():
    w = inf._mass_adaptation_weights(0.5, [True, False, False, False], [0.3, 0.3, np.nan, 0.9], [False, False, False, True])
    assert w[0] == 1.0 and w[2] == 0.0 and w[3] == 0.0
    assert w[1] == pytest.approx(1.0 + (0.3 - 1.0) * 0.5)


def test_diagnostics_iid_draws():
    rng = np.random.default_rng(0)

    class Fake:
        constrained = rng.standard_normal((8, 400, 2))
        unconstrained = constrained
        sampling_seconds = 2.0

    r = dg.rhat(Fake)
    e = dg.ess(Fake)
    assert np.all(np.abs(r - 1) < 0.02)
    assert np.all(e > 0.6 * 3200)
    assert dg.min_ess_per_second(Fake) == pytest.approx(np.min(e) / 2.0)
    rr = dg.rhat(Fake, method="rank")
    assert np.all(rr < 1.02)


def _rank_rhat_loops(chains):
    """The reference's rank-normalised R-hat of one parameter, restated with
    loops (diagnostics.jl:500-511 split matrix, :589-600 ranks of the
    column-major flattening by a stable sort, :602-612 bulk and folded)."""
    from statistics import NormalDist
    C, S = len(chains), len(chains[0])
    h = S // 2
    split = []
    for c in range(C):
        split.append(list(chains[c][:h]))
        split.append(list(chains[c][h:2 * h]))

    def rhat_of(m):
        means = [sum(r) / h for r in m]
        var = [sum((v - mu) ** 2 for v in r) / (h - 1) for r, mu in zip(m, means)]
        W = sum(var) / len(m)
        gm = sum(means) / len(m)
        B = h * sum((mu - gm) ** 2 for mu in means) / (len(m) - 1)
        return math.sqrt(max(((h - 1) / h * W + B / h) / W, 1.0))

    def rank_normal(m):
        flat = [m[i][j] for j in range(h) for i in range(len(m))]  # column-major
        order = sorted(range(len(flat)), key=lambda k: flat[k])   # stable
        ranks = [0] * len(flat)
        for pos, k in enumerate(order):
            ranks[k] = pos + 1
        n = len(flat)
        z = [NormalDist().inv_cdf((r - 0.375) / (n + 0.25)) for r in ranks]
        return [[z[j * len(m) + i] for j in range(h)] for i in range(len(m))]

    vals = sorted(v for r in split for v in r)
    n = len(vals)
    med = 0.5 * (vals[(n - 1) // 2] + vals[n // 2])
    folded = [[abs(v - med) for v in r] for r in split]
    return max(rhat_of(rank_normal(split)), rhat_of(rank_normal(folded)))


def test_rank_rhat_ties_follow_reference_order():
    """Repeated states (rejected proposals) tie; their ranks follow the
    reference's order, in the host diagnostics and the device gate alike."""
    import torch
    from uncertaintea_b200.multi import rank_split_rhat
    rng = np.random.default_rng(11)
    d = np.round(rng.standard_normal((5, 41, 2)), 1)   # (C, S, P) with many ties
    d[0] += 0.3

    class Fake:
        constrained = d
        unconstrained = d

    host = dg.rhat(Fake, method="rank")
    dev = rank_split_rhat(torch.from_numpy(d.transpose(1, 0, 2).copy())).numpy()
    for p in range(2):
        ref = _rank_rhat_loops(d[:, :, p].tolist())
        assert host[p] == pytest.approx(ref, rel=1e-12)
        assert dev[p] == pytest.approx(ref, rel=1e-12)


def test_fixed_step_chees_jitters_the_step_size_after_warmup():
    """With fixed_leapfrog_steps the Halton jitter moves from the step count to
    the step size, from the first sampling iteration on; the reference's rule
    (no fixed count) is unchanged."""
    for it in (1, 2, 3, 50, 51, 52, 77):
        j = inf._chees_jitter_value(1.0, it)
        eps, L, jit = inf._chees_iteration_step_and_steps(0.5, 3.0, 1.0, it, 50, 16)
        assert L == 16 and jit == j
        assert eps == (0.5 * j if it > 50 else 0.5)
        eps, L, _ = inf._chees_iteration_step_and_steps(0.5, 3.0, 1.0, it, 50)
        assert eps == 0.5 and L == inf._chees_leapfrog_steps_from_jitter(j, 3.0, 0.5)
    # jitter_amount = 0: no jitter anywhere
    assert inf._chees_iteration_step_and_steps(0.5, 3.0, 0.0, 77, 50, 16)[:2] == (0.5, 16)
    # the sampling-phase step sizes cover (0, eps): no fixed trajectory length repeats
    eps = [inf._chees_iteration_step_and_steps(0.5, 3.0, 1.0, it, 0, 16)[0] for it in range(1, 65)]
    assert len(set(eps)) == 64 and 0.0 < min(eps) and max(eps) < 0.5


def test_device_diagnostics_match_the_host_estimators():
    """The torch estimators the bench runs on the device (plain split R-hat,
    rank-normalised split R-hat, bulk ESS) agree with the host diagnostics,
    odd draw counts included."""
    import torch
    from uncertaintea_b200.multi import rank_split_rhat, split_ess, split_rhat
    rng = np.random.default_rng(12)
    for C, S in ((4, 101), (7, 64)):
        d = np.cumsum(rng.standard_normal((C, S, 3)), axis=1) * 0.1 + rng.standard_normal((C, S, 3))

        class Fake:
            constrained = d
            unconstrained = d

        x = torch.from_numpy(d.transpose(1, 0, 2).copy())
        np.testing.assert_allclose(split_rhat(x).numpy(), dg.rhat(Fake), rtol=1e-12)
        np.testing.assert_allclose(rank_split_rhat(x).numpy(), dg.rhat(Fake, method="rank"), rtol=1e-12)
        np.testing.assert_allclose(split_ess(x).numpy(), dg.ess(Fake), rtol=1e-9)


def test_bench_diagnostics_and_gate_prefixes_match_the_host_estimators():
    """bench.py's sampler rows compute rank R-hat, split R-hat and bulk ESS a
    few parameters at a time with the torch estimators (on the device when
    there is one); chunking and prefixes give the host diagnostics' values."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    rng = np.random.default_rng(3)
    d = np.cumsum(rng.standard_normal((6, 300, 37)), axis=1) * 0.05 + rng.standard_normal((6, 300, 37))

    class Fake:
        constrained = d
        unconstrained = d
        sampling_seconds = 2.0

    rr, rs, e = bench._device_diagnostics(Fake, chunk=5)
    np.testing.assert_allclose(rr, dg.rhat(Fake, "unconstrained", method="rank"), rtol=1e-12)
    np.testing.assert_allclose(rs, dg.rhat(Fake, "unconstrained"), rtol=1e-12)
    np.testing.assert_allclose(e, dg.ess(Fake, "unconstrained"), rtol=1e-9)

    class Half:
        constrained = d[:, :151]
        unconstrained = d[:, :151]

    rows = bench._gate_prefixes(Fake, [151, 300, 400])
    assert [r["draws"] for r in rows] == [151, 300]
    assert rows[0]["max_rank_rhat"] == pytest.approx(np.max(dg.rhat(Half, "unconstrained", method="rank")), rel=1e-12)
    assert rows[0]["min_ess"] == pytest.approx(np.min(dg.ess(Half, "unconstrained")), rel=1e-9)
    assert rows[1]["min_ess_per_s"] == pytest.approx(np.min(e) / 2.0, rel=1e-9)


def test_diagnostics_detect_disagreeing_chains():
    rng = np.random.default_rng(1)

    class Fake:
        constrained = rng.standard_normal((4, 200, 1)) + np.arange(4)[:, None, None]
        unconstrained = constrained

    assert dg.rhat(Fake)[0] > 1.1


def test_split_ess_matches_direct_sum():
    """FFT autocovariance == the reference's direct autocovariance sum (diagnostics.jl:541-583)."""
    rng = np.random.default_rng(3)
    x = np.cumsum(rng.standard_normal((6, 101)), axis=1) * 0.1 + rng.standard_normal((6, 101))
    split = dg._split_chain_draws(x)
    M, S = split.shape
    means, _, W, _, var_plus = dg._chain_stats(split)
    pair_sums = []
    for start in range(0, S, 2):
        s = 0.0
        for lag in range(start, min(start + 1, S - 1) + 1):
            ac = np.mean([np.sum((split[m, :S - lag] - means[m]) * (split[m, lag:] - means[m])) / S for m in range(M)])
            rho = 1.0 if lag == 0 else 1 - (W - ac) / var_plus
            s += min(rho, 1.0)
        if not s > 0:
            break
        pair_sums.append(s)
    for i in range(1, len(pair_sums)):
        pair_sums[i] = min(pair_sums[i], pair_sums[i - 1])
    tau = max(-1 + 2 * sum(pair_sums), 1.0)
    assert dg._split_ess_of(split) == pytest.approx(min(M * S, M * S / tau), rel=1e-9)


def test_summarize_matches_the_reference_formulas():
    """summarize (diagnostics.jl:662-712, summaries.jl:1-76) restated with direct
    loops: quantiles at position 1 + (n - 1) p, MCSE of the mean sd / sqrt(ess),
    tail ESS from the 5% / 95% indicators, order-statistic MCSE of the
    quantiles, per-chain means and SDs, quantile validation."""
    rng = np.random.default_rng(7)
    x = np.cumsum(rng.standard_normal((4, 301, 2)), axis=1) * 0.05 + rng.standard_normal((4, 301, 2))

    class Fake:
        constrained = x
        unconstrained = x
        accept_prob = rng.random((4, 301))
        divergent = rng.random((4, 301)) < 0.01
        step_size = np.array([0.1, 0.2, 0.3, 0.4])
        energy = rng.standard_normal((4, 301))
        tree_depth = np.zeros((4, 301), dtype=np.int32)

        @staticmethod
        def parameter_names():
            return ["a", "b"]

    out = dg.summarize(Fake, quantiles=(0.1, 0.5, 0.9), per_chain=True)

    def quant(sv, q):  # diagnostics.jl:486-497, 1-based
        n = len(sv)
        pos = 1 + (n - 1) * q
        lo, hi = int(np.floor(pos)), int(np.ceil(pos))
        return sv[lo - 1] if lo == hi else (1 - (pos - lo)) * sv[lo - 1] + (pos - lo) * sv[hi - 1]

    for p, row in enumerate(out["parameters"]):
        pooled = np.concatenate([x[c, :, p] for c in range(4)])
        sv = np.sort(pooled)
        n = pooled.size
        mean = sum(pooled) / n
        sd = np.sqrt(sum((v - mean) ** 2 for v in pooled) / (n - 1))
        assert row["parameter"] == "ab"[p]
        assert row["mean"] == pytest.approx(mean, rel=1e-12) and row["sd"] == pytest.approx(sd, rel=1e-12)
        assert row["quantiles"] == pytest.approx([quant(sv, q) for q in (0.1, 0.5, 0.9)], rel=1e-12)
        split = dg._split_chain_draws(x[:, :, p])
        ess_bulk = dg._split_ess_of(split)
        assert row["ess_bulk"] == pytest.approx(ess_bulk, rel=1e-12)
        assert row["mcse_mean"] == pytest.approx(sd * np.sqrt(1 / ess_bulk), rel=1e-12)
        ind = lambda t: dg._split_ess_of((split <= t).astype(float))  # noqa: E731
        assert row["ess_tail"] == pytest.approx(min(ind(quant(sv, 0.05)), ind(quant(sv, 0.95))), rel=1e-12)
        for q, th, m in zip((0.1, 0.5, 0.9), row["quantiles"], row["mcse_quantiles"]):
            e = ind(th)
            spread = np.sqrt(q * (1 - q) / e)
            ref = (quant(sv, min(q + spread, 1.0)) - quant(sv, max(q - spread, 0.0))) / 2
            assert m == pytest.approx(ref, rel=1e-12)
        for c in range(4):
            cm = sum(x[c, :, p]) / 301
            assert row["per_chain_means"][c] == pytest.approx(cm, rel=1e-12)
            assert row["per_chain_sds"][c] == pytest.approx(np.sqrt(sum((x[c, :, p] - cm) ** 2) / 300), rel=1e-12)
    dgn = out["diagnostics"]
    assert dgn["acceptance_rate"] == pytest.approx(Fake.accept_prob.mean())
    assert dgn["divergence_rate"] == pytest.approx(Fake.divergent.mean())
    assert dgn["mean_step_size"] == pytest.approx(0.25)
    assert dg.summarize(Fake)["parameters"][0]["per_chain_means"] is None
    # a parameter on one side of the tail threshold has NaN tail ESS (a constant indicator)
    class Const(Fake):
        constrained = np.ones((4, 301, 2))
        unconstrained = constrained
    assert np.isnan(dg.summarize(Const)["parameters"][0]["ess_tail"])
    for bad, msg in [((), "non-empty"), ((0.5, 1.5), r"lie in \[0, 1\]")]:
        with pytest.raises(ValueError, match=msg):
            dg.summarize(Fake, quantiles=bad)


def test_check_diagnostics_matches_the_reference_rules():
    """check_diagnostics / has_warnings (warnings.jl:7-86): per-chain divergence
    counts, E-BFMI, treedepth hits at the depth limit, high-R-hat and low-ESS
    parameters (non-finite values count), none of the latter below 4 draws."""
    rng = np.random.default_rng(2)
    C, S = 3, 200

    class Fake:
        constrained = rng.standard_normal((C, S, 2))
        unconstrained = constrained
        divergent = np.zeros((C, S), dtype=bool)
        energy = rng.standard_normal((C, S))
        tree_depth = np.full((C, S), 3)
        max_tree_depth = 10
        accept_prob = np.full((C, S), 0.8)
        step_size = np.full(C, 0.1)

        @staticmethod
        def parameter_names():
            return ["a", "b"]

    # the reference's hand-computed E-BFMI pins (mcmc_diagnostics_ess_mcse.jl:52-56)
    assert dg._ebfmi(np.array([1.0, 3.0, 2.0])) == pytest.approx(2.5, abs=1e-12)
    assert np.isnan(dg._ebfmi(np.array([1.0]))) and np.isnan(dg._ebfmi(np.array([5.0, 5.0, 5.0])))
    w = dg.check_diagnostics(Fake)
    ref = [np.sum(np.diff(e) ** 2) / np.sum((e - e.mean()) ** 2) for e in Fake.energy]
    assert w.ebfmi == pytest.approx(ref, rel=1e-12)
    assert not dg.has_warnings(w) and w.low_ess_parameters == [] and w.high_rhat_parameters == []

    class Bad(Fake):
        constrained = np.concatenate([rng.standard_normal((C, S, 1)),
                                      rng.standard_normal((C, S, 1)) + np.arange(C)[:, None, None] * 3], axis=2)
        unconstrained = constrained
        divergent = np.zeros((C, S), dtype=bool)
        divergent[1, :5] = True
        tree_depth = np.full((C, S), 10)
        energy = np.cumsum(rng.standard_normal((C, S)), axis=1)   # random walk: E-BFMI far below 0.3

    w = dg.check_diagnostics(Bad)
    assert list(w.num_divergent) == [0, 5, 0] and list(w.treedepth_hits) == [S, S, S]
    assert np.all(w.ebfmi < 0.3) and w.high_rhat_parameters == ["b"] and "b" in w.low_ess_parameters
    assert dg.has_warnings(w)
    assert dg.check_diagnostics(Bad, ess_threshold=0.0).low_ess_parameters == []

    class Short(Fake):
        constrained = np.ones((C, 3, 2))
        unconstrained = constrained
        energy = np.ones((C, 3))

    w = dg.check_diagnostics(Short)
    assert w.high_rhat_parameters == [] and np.all(np.isnan(w.ebfmi))
    assert isinstance(dg.summarize(Fake)["warnings"], dg.SamplerWarnings)
    text = str(dg.summarize(Fake))
    assert "parameter" in text and "rhat" in text and "warnings" not in text
    assert any(line.split()[0] == "a" for line in text.splitlines()[2:4])
    bad_text = str(dg.summarize(Bad))
    assert "warnings:" in bad_text and "divergences: 5 total" in bad_text and "high Rhat parameters: ['b']" in bad_text
    # the reference's diagnostics checks (diagnostics.jl:332-340, 384-402)
    with pytest.raises(ValueError, match="at least 4 samples"):
        dg.rhat(Short)
    with pytest.raises(ValueError, match="at least 4 samples"):
        dg.summarize(Short)
    with pytest.raises(ValueError, match="diagnostic space"):
        dg.ess(Fake, space="bogus")
    assert dg.rhat(Fake, space="unconstrained").shape == (2,)


class _OracleProbeRun:
    """The step-size searches of the device runner, driven by the oracle's
    leapfrog probe (the same log accept ratio the device probe returns) with
    one fixed momentum coordinate."""

    def __init__(self, C=2, P=4, seed=1):
        import oracle
        from uncertaintea_b200.models import BernoulliLogitGLM, logistic_regression_data
        X, y, _ = logistic_regression_data(200, P, seed)
        self.om = oracle.OracleModel(BernoulliLogitGLM(P).lower((X,), {"y": y}))
        self.C = C
        self.q = np.random.default_rng(seed).standard_normal((C, P)).astype(np.float32)
        self.lj, self.g = self.om.logjoint_gradient_f32(self.q)
        self.probes = []

    def next_probe_coord(self):
        return 12345

    def probe(self, trial_steps, inverse_mass, coord):
        ts = np.broadcast_to(np.asarray(trial_steps, dtype=np.float32), (self.C,)).copy()
        self.probes.append(ts)
        return self.om.leapfrog_probe(self.q.copy(), self.g.copy(), self.lj.copy(), np.asarray(inverse_mass), ts,
                                      coord).astype(np.float64)


def test_shared_step_search_stops_at_the_first_crossing():
    """The reference's shared step-search regression (warmup_driver_regression.jl:67-137):
    searches started from s0 and 2 s0 with the same momentum land on the same
    step, on the halving (or doubling) grid of their start, and the downward
    and upward searches bracket each other within a factor 4."""
    from uncertaintea_b200.inference import _DeviceRun
    run = _OracleProbeRun()
    search = lambda s0: _DeviceRun.find_reasonable_step_size(run, s0, np.ones(4), 1000.0)  # noqa: E731
    down, down2 = search(10.0), search(20.0)
    assert down == down2 and down < 10.0
    assert float(np.log2(10.0 / down)).is_integer() and float(np.log2(20.0 / down2)).is_integer()
    up, up2 = search(1e-4), search(2e-4)
    assert up == up2 and up > 1e-4 and float(np.log2(up / 1e-4)).is_integer()
    assert up / 4 <= down <= up * 4


def test_per_chain_step_search_equals_independent_searches():
    """The reference's vectorised per-chain search (warmup_driver_regression.jl:139-221)
    reproduces independent per-chain searches: each chain's step is the first
    crossing of log(0.5) along its own halving / doubling sequence."""
    import math
    from uncertaintea_b200.inference import _DeviceRun
    run = _OracleProbeRun(C=6, seed=3)
    starts = np.array([10.0, 1e-4, 0.5, 2.0, 1e-3, 40.0])
    got = _DeviceRun.find_reasonable_step_size_per_chain(run, starts, np.ones(4))
    for c in range(6):
        def lar(step):
            ts = np.full(6, step, dtype=np.float32)
            return float(run.om.leapfrog_probe(run.q.copy(), run.g.copy(), run.lj.copy(), np.ones(4), ts, 12345)[c])
        s = float(starts[c])
        d = 1.0 if lar(s) > math.log(0.5) else -1.0
        for _ in range(20):
            nxt = s * 2.0 ** d
            if nxt < 1e-8 or nxt > 1e3:
                break
            s = nxt
            v = lar(s)
            if (d > 0 and v <= math.log(0.5)) or (d < 0 and v >= math.log(0.5)):
                break
        assert got[c] == pytest.approx(s, rel=1e-12), c


# ---- mean-field ADVI host logic (vi.jl:179-227, guides.jl:51-57) -----------
def test_advi_entropy_clip_and_adam():
    from uncertaintea_b200 import vi
    ls = np.array([-1.0, 0.5, 2.0])
    assert vi._gaussian_entropy(ls) == pytest.approx(1.5 * (1 + math.log(2 * math.pi)) + 1.5, abs=1e-14)
    lg, sg = np.array([3.0, 0.0, 0.0]), np.array([0.0, 4.0, 0.0])
    assert vi._clip_advi_gradients(lg, sg, math.inf) == pytest.approx(5.0)
    assert vi._clip_advi_gradients(lg, sg, 1.0) == 1.0
    np.testing.assert_allclose(lg, [0.6, 0, 0]) and np.testing.assert_allclose(sg, [0, 0.8, 0])
    # Adam ascent, two steps against the scalar recursion
    p, m1, m2 = np.array([0.5]), np.zeros(1), np.zeros(1)
    ref, a, b = 0.5, 0.0, 0.0
    for it, g in enumerate([2.0, -1.0], start=1):
        vi._adam_ascent_step(p, m1, m2, np.array([g]), it, 0.05, 0.9, 0.999, 1e-8)
        a = 0.9 * a + 0.1 * g
        b = 0.999 * b + 0.001 * g * g
        ref += 0.05 * (a / (1 - 0.9 ** it)) / (math.sqrt(b / (1 - 0.999 ** it)) + 1e-8)
    assert p[0] == pytest.approx(ref, abs=1e-15)


def test_advi_on_the_conjugate_model_through_the_oracle():
    """Mean-field ADVI is exact for the conjugate gauss model (posterior
    normal(0.15, sqrt(0.5))): the oracle's ADVI step (Philox particles, mean
    gradients) with the package's gradient clip, entropy and Adam ascent
    reaches that location and scale, and the ELBO rises."""
    import oracle
    from uncertaintea_b200 import vi
    from uncertaintea_b200.models import NormalKnownScale
    om = oracle.OracleModel(NormalKnownScale().lower((1,), {"y": np.array([0.3])}))
    loc, ls = np.array([-1.0]), np.array([-1.0])
    m1, v1, m2, v2 = np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(1)
    locs, scales, elbo = [], [], []
    for it in range(1, 1501):
        r = om.advi_step(loc.astype(np.float32), np.exp(ls).astype(np.float32), 256, 7000 + it)
        lg = np.asarray(r["location_gradient"], dtype=np.float64).copy()
        sg = 1.0 + np.asarray(r["scale_gradient"], dtype=np.float64)
        vi._clip_advi_gradients(lg, sg, math.inf)
        elbo.append(float(np.mean(r["values"])) + vi._gaussian_entropy(ls))
        vi._adam_ascent_step(loc, m1, v1, lg, it, 0.02, 0.9, 0.999, 1e-8)
        vi._adam_ascent_step(ls, m2, v2, sg, it, 0.02, 0.9, 0.999, 1e-8)
        locs.append(loc[0])
        scales.append(math.exp(ls[0]))
    assert abs(np.mean(locs[-300:]) - 0.15) < 0.03, np.mean(locs[-300:])
    assert abs(np.mean(scales[-300:]) - math.sqrt(0.5)) < 0.05, np.mean(scales[-300:])
    assert np.mean(elbo[-100:]) > np.mean(elbo[:100])


def test_advi_validation_before_any_device_work():
    from uncertaintea_b200 import BernoulliLogitGLM, batched_advi
    m = BernoulliLogitGLM(3)
    X, y = np.zeros((4, 3)), np.zeros(4)
    for kw, msg in [(dict(guide="fullrank"), "CPU-only"), (dict(elbo="iwae"), "CPU-only"),
                    (dict(guide="bogus"), "guide must be"), (dict(num_iterations=0), "num_iterations > 0"),
                    (dict(num_particles=0), "num_particles > 0"), (dict(beta1=1.0), "beta1"),
                    (dict(gradient_clip=0.0), "gradient_clip > 0"), (dict(adtype="bogus"), "adtype must be"),
                    (dict(adtype="reverse"), "host-only path")]:
        args = dict(num_iterations=5)
        args.update(kw)
        with pytest.raises(ValueError, match=msg):
            batched_advi(m, (X,), {"y": y}, **args)


def test_nuts_validation_before_any_device_work():
    """batched_nuts rejects what the reference rejects (api_batched_nuts.jl:60-63,
    99-102) with its messages, before any device work."""
    from uncertaintea_b200 import BernoulliLogitGLM, batched_nuts
    m = BernoulliLogitGLM(3)
    X, y = np.zeros((4, 3)), np.zeros(4)
    for kw, msg in [(dict(adtype="bogus"), "adtype must be :auto, :forward, or :reverse"),
                    (dict(adtype="reverse"), "adtype=:reverse is a host-only path"),
                    (dict(tree_strategy="hybrid"), "requires tree_strategy=:masked or :persistent"),
                    (dict(tree_strategy="bogus"), "tree_strategy must be"),
                    (dict(persistent_gradient="bogus"), "persistent_gradient must be"),
                    (dict(max_tree_depth=0), "max_tree_depth must be >= 1"),
                    (dict(num_chains=0), "num_chains must be >= 1"),
                    (dict(init_strategy="bogus"), "init_strategy must be :prior or :uniform, got :bogus"),
                    (dict(init_max_retries=-1), "init_max_retries must be >= 0, got -1")]:
        args = dict(num_chains=4, num_samples=5, device_sync_per_leaf=True)
        args.update(kw)
        with pytest.raises(ValueError, match=msg):
            batched_nuts(m, (X,), {"y": y}, **args)


def test_init_validation_before_any_device_work():
    """init_robustness_batched.jl:62-69: a bad init_strategy or a negative retry
    budget is rejected up front by every sampler."""
    from uncertaintea_b200 import BernoulliLogitGLM, batched_chees, batched_hmc
    m = BernoulliLogitGLM(3)
    X, y = np.zeros((4, 3)), np.zeros(4)
    for fn, name in ((batched_hmc, "batched_hmc"), (batched_chees, "batched_chees")):
        with pytest.raises(ValueError, match=f"{name} init_strategy must be"):
            fn(m, (X,), {"y": y}, num_chains=2, num_samples=2, init_strategy="bogus")
        with pytest.raises(ValueError, match=f"{name} init_max_retries must be >= 0"):
            fn(m, (X,), {"y": y}, num_chains=2, num_samples=2, init_max_retries=-1)


def test_oracle_advi_step_consistency():
    """The oracle's ADVI step equals its own pieces: Philox noise at stream 5,
    particles location + scale * eps, means of the f64 gradients."""
    import oracle
    from uncertaintea_b200.models import NormalLocationScale, gauss_data
    y, _ = gauss_data(30, 2)
    om = oracle.OracleModel(NormalLocationScale().lower((30,), {"y": y}))
    loc, sc = np.array([0.3, -0.2], dtype=np.float32), np.array([0.2, 0.5], dtype=np.float32)
    r = om.advi_step(loc, sc, 16, 77)
    eps = np.stack([oracle.rand_normal(j, 77, 5, 0, 2) for j in range(16)])
    # one rounding (fused multiply-add): the f32 product is exact in f64
    fused = (loc.astype(np.float64) + sc.astype(np.float64) * eps.astype(np.float64)).astype(np.float32)
    np.testing.assert_array_equal(r["particles"], fused)
    t, g = om.logjoint_gradient_f64(r["particles"].astype(np.float64))
    np.testing.assert_allclose(r["values"], t, rtol=1e-5)
    np.testing.assert_allclose(r["location_gradient"], g.mean(0), rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(r["scale_gradient"], (g * sc * eps).mean(0), rtol=1e-4, atol=1e-4)


def test_meads_validation_before_any_device_work():
    """batched_meads argument errors (batched_meads.jl:59-69)."""
    from uncertaintea_b200 import BernoulliLogitGLM, batched_meads
    m = BernoulliLogitGLM(3)
    X, y = np.zeros((4, 3)), np.zeros(4)
    for kw, msg in [(dict(num_chains=4, num_folds=1), "num_folds must be >= 2"),
                    (dict(num_chains=6, num_folds=4), "num_chains >= 2 \\* num_folds"),
                    (dict(num_chains=8, num_samples=0), "num_samples must be > 0"),
                    (dict(num_chains=8, init_strategy="bogus"), "init_strategy")]:
        args = dict(num_chains=8, num_samples=10)
        args.update(kw)
        with pytest.raises(ValueError, match=msg):
            batched_meads(m, (X,), {"y": y}, **args)
