"""Step programs (the composable kernel description) on the CPU: the oracle's
plan walk against scipy's densities for every distribution of the reference's
scalar device families (math.jl:88-300) and the transforms (math.jl:1144-1159),
its forward-mode gradient against central finite differences on composite
models, the program form of a fixed family against that family's own oracle,
and the host compiler's checks (ut_program_report) through the library."""
import numpy as np
import pytest
from scipy import special, stats

import oracle
from uncertaintea_b200 import _native as nat
from uncertaintea_b200.models import NormalLocationScale, gauss_data
from uncertaintea_b200.program import Program, ProgramModel, report

# (name, args, observed value, scipy logpdf)
_CASES = [
    ("normal", (0.3, 1.7), -0.4, lambda a, x: stats.norm(a[0], a[1]).logpdf(x)),
    ("lognormal", (0.2, 0.8), 1.3, lambda a, x: stats.lognorm(a[1], scale=np.exp(a[0])).logpdf(x)),
    ("exponential", (1.7,), 0.6, lambda a, x: stats.expon(scale=1 / a[0]).logpdf(x)),
    ("gamma", (2.5, 1.5), 1.1, lambda a, x: stats.gamma(a[0], scale=1 / a[1]).logpdf(x)),
    ("laplace", (0.2, 0.9), -0.5, lambda a, x: stats.laplace(a[0], a[1]).logpdf(x)),
    ("cauchy", (0.1, 1.3), 2.0, lambda a, x: stats.cauchy(a[0], a[1]).logpdf(x)),
    ("halfnormal", (1.4,), 0.9, lambda a, x: stats.halfnorm(scale=a[0]).logpdf(x)),
    ("halfcauchy", (2.5,), 1.2, lambda a, x: stats.halfcauchy(scale=a[0]).logpdf(x)),
    ("logistic", (0.3, 0.7), -0.2, lambda a, x: stats.logistic(a[0], a[1]).logpdf(x)),
    ("gumbel", (0.3, 0.7), 0.8, lambda a, x: stats.gumbel_r(a[0], a[1]).logpdf(x)),
    ("frechet", (2.2, 1.3), 1.7, lambda a, x: stats.invweibull(a[0], scale=a[1]).logpdf(x)),
    ("rayleigh", (1.1,), 0.7, lambda a, x: stats.rayleigh(scale=a[0]).logpdf(x)),
    ("inversegaussian", (1.2, 2.0), 0.9, lambda a, x: stats.invgauss(a[0] / a[1], scale=a[1]).logpdf(x)),
    ("beta", (2.0, 3.5), 0.3, lambda a, x: stats.beta(a[0], a[1]).logpdf(x)),
    ("studentt", (4.5, 0.2, 1.3), 1.1, lambda a, x: stats.t(a[0], a[1], a[2]).logpdf(x)),
    ("inversegamma", (3.0, 2.0), 0.8, lambda a, x: stats.invgamma(a[0], scale=a[1]).logpdf(x)),
    ("weibull", (1.8, 1.4), 0.9, lambda a, x: stats.weibull_min(a[0], scale=a[1]).logpdf(x)),
    ("bernoulli", (0.3,), 1.0, lambda a, x: stats.bernoulli(a[0]).logpmf(x)),
    ("bernoullilogit", (0.4,), 0.0, lambda a, x: stats.bernoulli(special.expit(a[0])).logpmf(x)),
    ("poisson", (3.2,), 4.0, lambda a, x: stats.poisson(a[0]).logpmf(x)),
    ("geometric", (0.3,), 2.0, lambda a, x: stats.geom(a[0], loc=-1).logpmf(x)),
    ("negativebinomial", (3.5, 0.4), 5.0, lambda a, x: stats.nbinom(a[0], a[1]).logpmf(x)),
    ("binomial", (12.0, 0.35), 4.0, lambda a, x: stats.binom(a[0], a[1]).logpmf(x)),
]


def _eval(model, q):
    om = oracle.OracleModel(model.lower())
    t, g = om.logjoint_gradient_f64(np.atleast_2d(q))
    return t, g, om


@pytest.mark.parametrize("case", range(len(_CASES)))
def test_program_oracle_observed_density_matches_scipy(case):
    """One observed choice of each distribution with constant arguments, plus
    a standard normal latent so the program has a parameter."""
    name, args, x, ref = _CASES[case]
    p = Program()
    p.latent("u", "normal", 0.0, 1.0)
    p.observe(name, *args, row=0)
    t, g, _ = _eval(ProgramModel(p, [x]), [[0.25]])
    want = ref(args, float(np.float32(x))) + stats.norm.logpdf(0.25)   # the staged buffer is float32
    assert t[0] == pytest.approx(want, rel=1e-12, abs=1e-12)
    assert g[0, 0] == pytest.approx(-0.25, rel=1e-12)


@pytest.mark.parametrize("case", [c for c in range(len(_CASES)) if _CASES[c][0] not in
                                  ("bernoulli", "bernoullilogit", "poisson", "geometric", "negativebinomial",
                                   "binomial")])
def test_program_oracle_latent_density_transform_and_gradient(case):
    """The same distributions as latent values under their default transform:
    logjoint = logpdf(T(u)) + log|T'(u)|, gradient against central
    differences, and every argument made latent-dependent (scaled by
    exp(v)) so the argument adjoints are exercised too."""
    name, args, x, ref = _CASES[case]
    positive = name in ("lognormal", "exponential", "gamma", "halfnormal", "halfcauchy", "frechet", "rayleigh",
                        "inversegaussian", "inversegamma", "weibull")
    u = np.log(x) if positive else (np.log(x / (1 - x)) if name == "beta" else x)
    p = Program()
    v = p.latent("v", "normal", 0.0, 1.0)
    scaled = [a * p.f("exp", v) if k > 0 or name in ("exponential", "halfnormal", "halfcauchy", "rayleigh") else a
              for k, a in enumerate(args)]
    p.latent("x", name, *scaled)
    model = ProgramModel(p, [])
    q = np.array([[0.1, u]])
    t, g, om = _eval(model, q)
    va = [a * np.exp(0.1) if (k > 0 or name in ("exponential", "halfnormal", "halfcauchy", "rayleigh")) else a
          for k, a in enumerate(args)]
    lad = u if positive else (np.log(x) + np.log1p(-x) if name == "beta" else 0.0)
    assert t[0] == pytest.approx(ref(va, x) + lad + stats.norm.logpdf(0.1), rel=1e-10, abs=1e-10)
    h = 1e-6
    for r in range(2):
        e = np.zeros((1, 2))
        e[0, r] = h
        fd = (om.logjoint_gradient_f64(q + e, want_grad=False)[0] - om.logjoint_gradient_f64(q - e, want_grad=False)[0])
        assert g[0, r] == pytest.approx(fd[0] / (2 * h), rel=1e-6, abs=1e-7), (name, r)


def _eight_schools(centred):
    y = np.array([28, 8, -3, 7, -1, 1, 18, 12], dtype=np.float64)
    s = np.array([15, 10, 16, 11, 9, 11, 10, 18], dtype=np.float64)
    p = Program()
    mu = p.latent("mu", "normal", 0.0, 5.0)
    tau = p.latent("tau", "halfcauchy", 5.0)
    for j in range(8):
        if centred:
            theta = p.latent(f"theta[{j + 1}]", "normal", mu, tau)
        else:
            z = p.latent(f"z[{j + 1}]", "normal", 0.0, 1.0)
            theta = p.deterministic(mu + tau * z)
        p.observe("normal", theta, p.obs(2 * j + 1), row=2 * j)
    staged = np.stack([y, s], axis=1).reshape(-1)
    return ProgramModel(p, staged), y, s


@pytest.mark.parametrize("centred", [True, False])
def test_program_oracle_eight_schools_closed_form_and_gradient(centred):
    model, y, s = _eight_schools(centred)
    q = np.random.default_rng(1).standard_normal((3, 10))
    t, g, om = _eval(model, q)
    for c in range(3):
        mu, tau = q[c, 0], np.exp(q[c, 1])
        theta = q[c, 2:] if centred else mu + tau * q[c, 2:]
        want = stats.norm(0, 5).logpdf(mu) + stats.halfcauchy(scale=5).logpdf(tau) + q[c, 1]
        want += (stats.norm(mu, tau).logpdf(q[c, 2:]) if centred else stats.norm.logpdf(q[c, 2:])).sum()
        want += stats.norm(theta, s).logpdf(y).sum()
        assert t[c] == pytest.approx(want, rel=1e-12)
    h = 1e-6
    for r in range(10):
        e = np.zeros_like(q)
        e[:, r] = h
        fd = (om.logjoint_gradient_f64(q + e, want_grad=False)[0] - om.logjoint_gradient_f64(q - e, want_grad=False)[0])
        np.testing.assert_allclose(g[:, r], fd / (2 * h), rtol=1e-6, atol=1e-7)


def _poisson_regression(N=60, seed=2):
    r = np.random.default_rng(seed)
    # float32 values: the staged buffer holds float32
    x1, x2 = (r.standard_normal(N).astype(np.float32).astype(np.float64) for _ in range(2))
    yv = r.poisson(np.exp(0.3 + 0.5 * x1 - 0.2 * x2)).astype(np.float64)
    p = Program()
    a = p.latent("a", "normal", 0.0, 2.0)
    b1 = p.latent("b1", "normal", 0.0, 1.0)
    b2 = p.latent("b2", "normal", 0.0, 1.0)
    with p.loop(N, width=3):
        p.observe("poisson", p.f("exp", a + b1 * p.obs(1) + b2 * p.obs(2)), row=0)
    staged = np.stack([yv, x1, x2], axis=1).reshape(-1)
    return ProgramModel(p, staged), yv, x1, x2


def test_program_oracle_loop_poisson_regression():
    """A loop of observed Poisson counts with a log link over two covariate
    columns of each block (the broadcast-observation layout of
    DeviceBroadcastNormalChoiceStep, steps.jl:252-259)."""
    model, yv, x1, x2 = _poisson_regression()
    q = np.array([[0.2, 0.4, -0.1], [0.5, 0.1, 0.3]])
    t, g, om = _eval(model, q)
    for c in range(2):
        lam = np.exp(q[c, 0] + q[c, 1] * x1 + q[c, 2] * x2)
        want = stats.norm(0, 2).logpdf(q[c, 0]) + stats.norm.logpdf(q[c, 1:]).sum() + stats.poisson(lam).logpmf(yv).sum()
        assert t[c] == pytest.approx(want, rel=1e-12)
        r_ = yv - lam
        grad = np.array([r_.sum() - q[c, 0] / 4, (r_ * x1).sum() - q[c, 1], (r_ * x2).sum() - q[c, 2]])
        np.testing.assert_allclose(g[c], grad, rtol=1e-10)


def test_program_oracle_nested_loops_and_iterator():
    """Two nested loops (fixed trip counts, reference DeviceLoopStep semantics)
    whose iterator enters an expression: y_jk ~ normal(mu + beta * j, s)."""
    J, K = 3, 4
    r = np.random.default_rng(5)
    yv = r.standard_normal((J, K)).astype(np.float32).astype(np.float64)
    p = Program()
    mu = p.latent("mu", "normal", 0.0, 3.0)
    beta = p.latent("beta", "normal", 0.0, 1.0)
    s = p.latent("s", "gamma", 2.0, 1.0)
    with p.loop(J, width=K, start=1) as j:
        with p.loop(K, width=1):
            p.observe("normal", mu + beta * j, s, row=0)
    model = ProgramModel(p, yv.reshape(-1))
    q = np.array([[0.3, -0.2, 0.1]])
    t, g, om = _eval(model, q)
    sv = np.exp(0.1)
    want = (stats.norm(0, 3).logpdf(0.3) + stats.norm.logpdf(-0.2) + stats.gamma(2.0).logpdf(sv) + 0.1 +
            sum(stats.norm(0.3 - 0.2 * (jj + 1), sv).logpdf(yv[jj]).sum() for jj in range(J)))
    assert t[0] == pytest.approx(want, rel=1e-12)


def test_program_form_of_the_gauss_family_matches_its_oracle():
    """mu ~ normal(0, 1), s ~ gamma(2, 1) (log), y_i ~ normal(mu, s) written as a
    program gives the dedicated family's oracle values and gradients."""
    y, _ = gauss_data(50, 3)
    p = Program()
    mu = p.latent("mu", "normal", 0.0, 1.0)
    s = p.latent("s", "gamma", 2.0, 1.0)
    with p.loop(50, width=1):
        p.observe("normal", mu, s, row=0)
    q = np.random.default_rng(2).standard_normal((5, 2)) * 0.5
    t1, g1, _ = _eval(ProgramModel(p, y), q)
    t2, g2 = oracle.OracleModel(NormalLocationScale().lower((50,), {"y": y})).logjoint_gradient_f64(q)
    np.testing.assert_allclose(t1, t2, rtol=1e-12)
    np.testing.assert_allclose(g1, g2, rtol=1e-10, atol=1e-12)


def test_program_glm_and_iid_normal_steps_match_a_direct_sum():
    r = np.random.default_rng(7)
    N, D = 40, 3
    X = r.standard_normal((N, D)).astype(np.float32).astype(np.float64)
    yv = (r.random(N) < 0.4).astype(np.float64)
    p = Program()
    a = p.latent("a", "normal", 0.0, 2.5)
    sg = p.latent("sigma", "halfnormal", 1.0)
    row = p.latent_iid_normal("beta", D, 0.0, sg)
    p.glm_bernoulli_logit(row, D, N, intercept=a)
    staged = np.concatenate([X, yv[:, None]], axis=1).reshape(-1)
    q = np.array([[0.2, -0.3, 0.5, -0.4, 0.1]])
    t, g, om = _eval(ProgramModel(p, staged), q)
    sv = np.exp(-0.3)
    eta = 0.2 + X @ q[0, 2:]
    want = (stats.norm(0, 2.5).logpdf(0.2) + stats.halfnorm(scale=1).logpdf(sv) - 0.3 +
            stats.norm(0, sv).logpdf(q[0, 2:]).sum() + (yv * eta - np.logaddexp(0, eta)).sum())
    assert t[0] == pytest.approx(want, rel=1e-12)
    h = 1e-6
    for k in range(5):
        e = np.zeros_like(q)
        e[0, k] = h
        fd = om.logjoint_gradient_f64(q + e, want_grad=False)[0] - om.logjoint_gradient_f64(q - e, want_grad=False)[0]
        assert g[0, k] == pytest.approx(fd[0] / (2 * h), rel=1e-6, abs=1e-7)
    mag = om.gradient_magnitude_f64(q)
    assert np.all(mag >= np.abs(g) * (1 - 1e-12))


def test_program_report_accepts_and_rejects(lib):
    model, _, _ = _eight_schools(False)
    ok, issues = report(model)
    assert ok and issues == []

    def bad(build, rows, needle):
        p = Program()
        build(p)
        ok, issues = report(ProgramModel(p, np.zeros(rows)))
        assert not ok and any(needle in i for i in issues), issues

    def latent_in_loop(p):
        with p.loop(2, width=1):
            p.steps.append(dict(kind=nat.UT_STEP_CHOICE, dist=1, arg=[p.expr(0.0).index, p.expr(1.0).index, -1, -1],
                                value_source=0, obs_offset=0, transform=0, binding_slot=-1, count=0, width=0, body=0,
                                iterator_slot=-1, iterator_start=0))
        p.num_params = 1
    bad(latent_in_loop, 2, "latent choice inside a loop")

    def read_before_write(p):
        p.latent("m", "normal", 0.0, 1.0)
        p.num_slots += 1
        p.observe("normal", p._node("slot", p.num_slots - 1), 1.0, row=0)
    bad(read_before_write, 1, "read before it is written")

    def row_outside(p):
        p.latent("m", "normal", 0.0, 1.0)
        p.observe("normal", 0.0, 1.0, row=5)
    bad(row_outside, 3, "outside its block")

    def leaf_outside(p):
        m = p.latent("m", "normal", 0.0, 1.0)
        with p.loop(2, width=2):
            p.observe("normal", m + p.obs(2), 1.0, row=0)
    bad(leaf_outside, 4, "observation leaf outside its block")

    def loop_too_long(p):
        p.latent("m", "normal", 0.0, 1.0)
        with p.loop(4, width=2):
            p.observe("normal", 0.0, 1.0, row=0)
    bad(loop_too_long, 7, "loop blocks outside")

    def uncovered(p):
        p.latent("m", "normal", 0.0, 1.0)
        p.num_params = 2
    bad(uncovered, 0, "parameter row 1 is read by no latent step")

    def discrete_latent(p):
        p.latent("k", "poisson", 3.0)
    bad(discrete_latent, 0, "discrete distribution's value must be observed")

    def huge_expr(p):
        m = p.latent("m", "normal", 0.0, 1.0)
        e = m
        for _ in range(30):
            e = e * m
        p.observe("normal", e, 1.0, row=0)
    bad(huge_expr, 1, "more than 48 nodes")

    def deep(p):
        p.latent("m", "normal", 0.0, 1.0)
        with p.loop(1, 1):
            with p.loop(1, 1):
                with p.loop(1, 1):
                    with p.loop(1, 1):
                        with p.loop(1, 1):
                            p.observe("normal", 0.0, 1.0, row=0)
    bad(deep, 1, "nest at most 4 deep")


def _host_math(tmp_path):
    """The device interpreter's distribution math compiled for the host."""
    import ctypes
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = str(tmp_path / "program_math.so")
    subprocess.run(["nvcc", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-o", lib,
                    os.path.join(root, "tests", "c_host", "program_math.cu")], check=True)
    h = ctypes.CDLL(lib)
    h.prog_dist_host.restype = ctypes.c_float
    h.prog_dist_host.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_float,
                                 ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    h.prog_digamma_host.restype = ctypes.c_float
    h.prog_digamma_host.argtypes = [ctypes.c_float]
    return h


def test_device_distribution_math_matches_scipy_and_its_derivatives(tmp_path):
    """Every distribution of the device interpreter (compiled for the host):
    the float32 log-density against scipy in float64, and each partial
    derivative (arguments and value) against float64 central differences of
    scipy's density, at several argument points."""
    import ctypes
    h = _host_math(tmp_path)
    r = np.random.default_rng(0)
    discrete = ("bernoulli", "bernoullilogit", "poisson", "geometric", "negativebinomial", "binomial")
    for name, args, x, ref in _CASES:
        code = nat.DISTRIBUTIONS[name]
        for trial in range(4):
            a = np.array(args, dtype=np.float64)
            if trial:   # perturb the continuous arguments (binomial trials stay integral)
                scale = np.where(np.arange(a.size) == 0 if name == "binomial" else False, 0.0, 0.15)
                a = a * np.exp(scale * r.standard_normal(a.size))
            a32 = (ctypes.c_float * 3)(*[float(np.float32(v)) for v in a] + [0.0] * (3 - a.size))
            da = (ctypes.c_float * 3)()
            dx = ctypes.c_float()
            x32 = float(np.float32(x))
            lp = h.prog_dist_host(code, a32, x32, da, ctypes.byref(dx))
            av = np.array([a32[k] for k in range(a.size)], dtype=np.float64)
            want = ref(av, x32)
            assert lp == pytest.approx(want, rel=2e-6, abs=2e-6), (name, trial)
            for k in range(a.size):
                if name == "binomial" and k == 0:
                    continue
                e = np.zeros_like(av)
                e[k] = 1e-6 * max(1.0, abs(av[k]))
                fd = (ref(av + e, x32) - ref(av - e, x32)) / (2 * e[k])
                assert da[k] == pytest.approx(fd, rel=2e-4, abs=2e-4 * max(1.0, abs(fd))), (name, trial, k)
            if name not in discrete:
                hx = 1e-6 * max(1.0, abs(x32))
                fd = (ref(av, x32 + hx) - ref(av, x32 - hx)) / (2 * hx)
                assert dx.value == pytest.approx(fd, rel=2e-4, abs=2e-4 * max(1.0, abs(fd))), (name, trial, "x")


def test_device_digamma_against_scipy(tmp_path):
    h = _host_math(tmp_path)
    for x in [1e-3, 0.05, 0.3, 0.5, 1.0, 1.7, 2.5, 4.0, 5.9, 6.0, 7.5, 12.0, 50.0, 1e3, 1e5]:
        assert h.prog_digamma_host(x) == pytest.approx(special.digamma(x), rel=3e-6, abs=3e-6), x


def _reference_logpdf_pins():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pins.json")
    with open(path) as f:
        return json.load(f)["logpdf"]


@pytest.mark.parametrize("pin", _reference_logpdf_pins(), ids=lambda p: f"{p['family']}@{p['x']}")
def test_program_oracle_matches_the_reference_tests_logpdf_pins(pin):
    """The reference's own scalar log-density tests (test/uncertaintea/core/
    dist_*.jl: `logpdf(family(args), x) ≈ closed form` and `== -Inf` outside the
    support, extracted by tests/golden/make_golden.py) hold for the oracle's
    plan walk, which the device's step programs are tested against: the
    parameterisations (rate or scale, failures or trials, shape order) are the
    reference's.  The staged observation is float32, so values agree to 1e-6."""
    p = Program()
    p.latent("u", "normal", 0.0, 1.0)
    p.observe(pin["family"], *pin["args"], row=0)
    t, _, _ = _eval(ProgramModel(p, [pin["x"]]), [[0.25]])
    got = float(t[0]) - stats.norm.logpdf(0.25)
    if np.isinf(pin["logpdf"]):
        assert got == pin["logpdf"], (pin["source"], got)
    else:
        assert abs(got - pin["logpdf"]) <= 1e-6 * max(1.0, abs(pin["logpdf"])), (pin["source"], got)
