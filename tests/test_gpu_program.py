"""Step programs on the GPU, through the C ABI: the warp interpreter's
logjoint and reverse-mode gradient against the FP64 oracle's plan walk
(forward-mode duals) for every distribution and for composite models, the
program form of a fixed family against that family's kernel, sampler
iterations replayed against the oracle under the same Philox streams, and
batched NUTS posteriors against the dedicated hierarchical family.

Tolerances: logjoint 1e-5 relative; gradient elementwise
|g - g64| <= 1e-5 |g64| + 1e-6 m (m = the oracle's gradient magnitude, the
sum over the terms of |d term / d row|) and the per-chain norm bound."""
import ctypes

import numpy as np
import pytest

import oracle
from test_gpu_parity import _grad_ok, _lj_err, _nuts_call, _ref, _state
from test_program import _CASES, _eight_schools, _poisson_regression
from uncertaintea_b200 import _native as nat
from uncertaintea_b200.models import HierarchicalNormalNoncentered, NormalLocationScale, gauss_data
from uncertaintea_b200.program import Program, ProgramModel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _ws(model, C):
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    return DeviceBatchedWorkspace(model, C)


def _check(model, q, norm=True):
    ws = _ws(model, q.shape[0])
    assert ws.kernel_path() == "warp"
    t, g = ws.logjoint_gradient(q.T)
    t_only = ws.logjoint(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5 and _lj_err(t_only, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag, norm=norm)
    ws.close()


def _all_distributions(blocks=64, seed=11):
    """Every continuous family as a latent with latent-dependent arguments,
    then a loop of `blocks` blocks holding one observation of each of the 23
    families (arguments depending on the latents)."""
    r = np.random.default_rng(seed)
    p = Program()
    s = p.latent("s", "normal", 0.0, 0.3)        # a log-scale every argument depends on
    e = p.f("exp", s)
    for name, args, x, _ in _CASES:
        if name in ("bernoulli", "bernoullilogit", "poisson", "geometric", "negativebinomial", "binomial"):
            continue
        p.latent(f"x_{name}", name, *[a * e if k == len(args) - 1 else a for k, a in enumerate(args)])
    vals = []
    for _ in range(blocks):
        vals += [r.normal(0.3, 1.7), r.lognormal(0.2, 0.8), r.exponential(0.6), r.gamma(2.5, 1 / 1.5),
                 r.laplace(0.2, 0.9), 0.1 + 1.3 * r.standard_cauchy(), abs(r.normal(0, 1.4)),
                 abs(2.5 * r.standard_cauchy()), r.logistic(0.3, 0.7), r.gumbel(0.3, 0.7),
                 1.3 * r.weibull(2.2) ** -1.0, r.rayleigh(1.1), r.wald(1.2, 2.0), r.beta(2.0, 3.5),
                 0.2 + 1.3 * r.standard_t(4.5), 1 / r.gamma(3.0, 1 / 2.0), 1.4 * r.weibull(1.8),
                 float(r.random() < 0.3), float(r.random() < 0.6), float(r.poisson(3.2)),
                 float(r.geometric(0.3) - 1), float(r.negative_binomial(3.5, 0.4)), float(r.binomial(12, 0.35))]
    with p.loop(blocks, width=23):
        for k, (name, args, _, _) in enumerate(_CASES):
            if name == "binomial":
                p.observe(name, 12.0, p.f("exp", s - 1.0), row=k)
            elif name in ("bernoulli", "geometric"):
                p.observe(name, p.f("exp", s - 1.2), row=k)
            elif name == "negativebinomial":
                p.observe(name, 3.5 * e, p.f("exp", s - 0.9), row=k)
            else:
                p.observe(name, *[a * e if j == len(args) - 1 else a for j, a in enumerate(args)], row=k)
    return ProgramModel(p, np.array(vals))


def test_program_every_distribution_vs_oracle(lib):
    model = _all_distributions()
    r = np.random.default_rng(3)
    P = model.program.num_params
    q = np.zeros((64, P), dtype=np.float32)
    q[:, 0] = 0.1 * r.standard_normal(64)
    for lat in model.program.latents[1:]:
        name = lat.dist
        x = dict((c[0], c[2]) for c in _CASES)[name]
        u = np.log(x) if lat.transform == nat.UT_TRANSFORM_LOG else (
            np.log(x / (1 - x)) if lat.transform == nat.UT_TRANSFORM_LOGIT else x)
        q[:, lat.row] = u + 0.2 * r.standard_normal(64)
    # The shared log-scale's gradient sums terms from every family whose
    # magnitudes total m ~ 7e3 and cancel to ~7e2: its FP32 error (~1e-6 m)
    # is ~1.5e-5 of the chain's largest component, so only the elementwise
    # bound, which carries that cancellation, applies here.
    _check(model, q, norm=False)


@pytest.mark.parametrize("centred", [True, False])
def test_program_eight_schools_vs_oracle(lib, centred):
    model, _, _ = _eight_schools(centred)
    q = (np.random.default_rng(4).standard_normal((100, 10)) * np.r_[3.0, 0.7, [1.0] * 8]).astype(np.float32)
    _check(model, q)


def test_program_poisson_regression_many_blocks_vs_oracle(lib):
    """2000 loop iterations over the 32 lanes of each chain's warp."""
    model, _, _, _ = _poisson_regression(N=2000, seed=6)
    q = (np.array([0.3, 0.5, -0.2]) + 0.05 * np.random.default_rng(5).standard_normal((40, 3))).astype(np.float32)
    _check(model, q)


def test_program_nested_loops_glm_and_iid_normal_vs_oracle(lib):
    r = np.random.default_rng(9)
    J, K, N, D = 5, 7, 300, 6
    yv = r.standard_normal((J, K))
    X = r.standard_normal((N, D)) * 0.5
    yb = (r.random(N) < 0.5).astype(np.float64)
    p = Program()
    mu = p.latent("mu", "normal", 0.0, 3.0)
    beta = p.latent("beta", "normal", 0.0, 1.0)
    s = p.latent("s", "gamma", 2.0, 1.0)
    with p.loop(J, width=K, start=1) as j:
        with p.loop(K, width=1):
            p.observe("normal", mu + beta * j, s, row=0)
    a = p.latent("a", "normal", 0.0, 2.5)
    sg = p.latent("sigma", "halfnormal", 1.0)
    row = p.latent_iid_normal("w", D, 0.0, sg)
    p.glm_bernoulli_logit(row, D, N, intercept=a, offset=J * K)
    staged = np.concatenate([yv.reshape(-1), np.concatenate([X, yb[:, None]], axis=1).reshape(-1)])
    model = ProgramModel(p, staged)
    q = (0.4 * np.random.default_rng(2).standard_normal((33, p.num_params))).astype(np.float32)
    _check(model, q)


def test_program_form_of_the_gauss_family_matches_its_kernel(lib):
    """The normal location/scale model as a program and as its fixed family:
    the two device evaluations agree to FP32 rounding."""
    y, _ = gauss_data(3000, 3)
    p = Program()
    mu = p.latent("mu", "normal", 0.0, 1.0)
    s = p.latent("s", "gamma", 2.0, 1.0)
    with p.loop(3000, width=1):
        p.observe("normal", mu, s, row=0)
    q = (np.random.default_rng(2).standard_normal((64, 2)) * 0.3).astype(np.float32)
    w1 = _ws(ProgramModel(p, y), 64)
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    w2 = DeviceBatchedWorkspace(NormalLocationScale(), 64, args=(3000,), constraints={"y": y})
    t1, g1 = w1.logjoint_gradient(q.T)
    t2, g2 = w2.logjoint_gradient(q.T)
    np.testing.assert_allclose(t1, t2, rtol=2e-6)
    np.testing.assert_allclose(g1, g2, rtol=1e-4, atol=1e-4 * np.abs(g2).max())
    w1.close()
    w2.close()


@pytest.mark.parametrize("strategy", ["persistent", "lockstep"])
def test_program_nuts_iteration_vs_oracle(lib, strategy):
    """One NUTS iteration on the non-centred eight-schools program against
    the oracle's NUTS (same Philox streams): the same trees for >= 95% of
    chains, their states within 1e-3."""
    model, _, _ = _eight_schools(False)
    C = 128
    q = (np.random.default_rng(8).standard_normal((C, 10)) * 0.5 + np.r_[4.0, 1.0, [0.0] * 8]).astype(np.float32)
    ws = _ws(model, C)
    qd, g, t = _state(ws, q)
    qo, go, to = qd.cpu().numpy().copy(), g.cpu().numpy().copy(), t.cpu().numpy().copy()
    im, steps = np.ones(10), np.full(C, 0.2)
    fn = lib.ut_persistent_nuts_iteration if strategy == "persistent" else lib.ut_lockstep_nuts_iteration
    gpu = _nuts_call(fn, ws, qd, g, t, im, steps, 8, 31)
    ref = oracle.OracleModel(ws.lowered).nuts_iteration(qo, go, to, im, steps, 8, 31)
    same = (gpu["tree_depth"] == ref["tree_depth"]) & (gpu["integration_steps"] == ref["integration_steps"]) & \
        (gpu["moved"] == ref["moved"])
    assert same.mean() >= 0.95, same.mean()
    assert gpu["tree_depth"].max() >= 2
    ws.close()


def test_program_hmc_iteration_vs_oracle(lib):
    model, _, _, _ = _poisson_regression(N=400, seed=3)
    C = 96
    q = (np.array([0.3, 0.5, -0.2]) + 0.05 * np.random.default_rng(1).standard_normal((C, 3))).astype(np.float32)
    ws = _ws(model, C)
    qd, g, t = _state(ws, q)
    qo, go, to = qd.cpu().numpy().copy(), g.cpu().numpy().copy(), t.cpu().numpy().copy()
    f = lambda dt=torch.float32: torch.zeros(C, dtype=dt, device="cuda")  # noqa: E731
    im = torch.ones(3, device="cuda")
    st = torch.full((C,), 0.01, device="cuda")
    o = [f(), f(), f(), f(torch.uint8), f(torch.uint8)]
    buf = nat.HmcBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(im), nat.ptr(st), *[nat.ptr(x) for x in o],
                         None, None)
    nat.check(lib.ut_hmc_iteration(ws.handle, ctypes.byref(buf), 8, 77, 1000.0, None))
    torch.cuda.synchronize()
    ref = oracle.OracleModel(ws.lowered).hmc_iteration(qo, go, to, np.ones(3), np.full(C, 0.01), 8, 77)
    acc = o[3].cpu().numpy()
    same = acc == ref["accepted"]
    assert same.mean() >= 0.98
    np.testing.assert_allclose(qd.cpu().numpy()[same], qo[same], rtol=1e-3, atol=1e-4)
    ws.close()


def test_program_nuts_posterior_matches_the_hierarchical_family(lib):
    """Batched NUTS on the non-centred eight-schools model written as a
    program and as the hierarchical family (the same priors): posterior means
    of every unconstrained coordinate within 5 MCSE."""
    from uncertaintea_b200 import batched_nuts, ess
    model, y, s = _eight_schools(False)
    fam = HierarchicalNormalNoncentered(8, mu_loc=0.0, mu_scale=5.0, tau_scale=5.0)
    a = batched_nuts(model, (), None, num_chains=256, num_samples=400, num_warmup=400, rng=3)
    b = batched_nuts(fam, (s.astype(np.float32), np.ones(8, dtype=np.int64)), {"y": y.astype(np.float32)},
                     num_chains=256, num_samples=400, num_warmup=400, rng=4)
    ua, ub = a.unconstrained.reshape(-1, 10), b.unconstrained.reshape(-1, 10)
    mcse = np.sqrt(ua.var(0) / ess(a, space="unconstrained") + ub.var(0) / ess(b, space="unconstrained"))
    assert np.all(np.abs(ua.mean(0) - ub.mean(0)) <= 5 * mcse), (ua.mean(0), ub.mean(0), mcse)
