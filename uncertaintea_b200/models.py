"""Model specifications and their lowering to the fixed kernel description.

The reference lowers a ``@tea static`` model's execution plan into an
``isbits`` ``DeviceExecutionPlan`` (src/device/plan/lowering.jl:1360) and
stages its observations into a dense buffer (src/device/staging.jl:499).  A
``TeaModelSpec`` here plays the role of that already-parsed model: it names a
kernel-description family and its priors, and ``lower(args, constraints)``
produces the ``PlanDesc`` plus the staged observation buffer that
``ut_workspace_create`` takes.

Calls mirror the reference: ``args`` carries the model's data arguments and
``constraints`` the observed choices, e.g. for the logistic regression
``args = (X,)`` and ``constraints = {"y": y}``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as nat


@dataclass
class Lowered:
    plan: nat.PlanDesc
    observed: np.ndarray            # float32, staged rows (one shared column)
    trip_counts: np.ndarray         # int32 (may be empty)
    loop_starts: np.ndarray         # int32 (may be empty)
    num_params: int


class TeaModelSpec:
    """Base class: a model whose density lowers to a device kernel description."""

    name = "model"

    def parameter_names(self, args=(), constraints=None):
        raise NotImplementedError

    def lower(self, args=(), constraints=None) -> Lowered:
        raise NotImplementedError

    def num_params(self, args=(), constraints=None) -> int:
        return len(self.parameter_names(args, constraints))

    def constrain(self, unconstrained: np.ndarray, args=(), constraints=None) -> np.ndarray:
        """Unconstrained draws (..., P) -> constrained values (..., P_constrained)."""
        return np.asarray(unconstrained)

    def initial_positions(self, rng: np.random.Generator, num_chains: int, args=(), constraints=None,
                          init_strategy: str = "prior") -> np.ndarray:
        raise NotImplementedError


def _observed_value(constraints, key):
    if constraints is None or key not in constraints:
        raise ValueError(f"missing observed choice {key!r} in constraints")
    return np.asarray(constraints[key], dtype=np.float64)


@dataclass
class BernoulliLogitGLM(TeaModelSpec):
    """``beta ~ iid normal(coef_mu, coef_sigma)`` (+ optional intercept),
    ``y_i ~ bernoullilogit(intercept + x_i . beta)``.

    args = (X,) with X of shape (N, D) (observation-major; the reference's own
    covariate matrix is D x N, ``X[:, i]`` being observation i -- pass
    ``X.T`` of such a matrix).  constraints = {"y": y} with y in {0, 1}.
    """

    num_coefs: int
    intercept: bool = False
    coef_mu: float = 0.0
    coef_sigma: float = 1.0
    intercept_mu: float = 0.0
    intercept_sigma: float = 2.5
    name: str = "bernoulli_logit_glm"

    def parameter_names(self, args=(), constraints=None):
        names = ["alpha"] if self.intercept else []
        return names + [f"beta[{d + 1}]" for d in range(self.num_coefs)]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 1:
            raise ValueError(f"{self.name} expects args=(X,), got {len(args)} argument(s)")
        X = np.asarray(args[0], dtype=np.float32)
        if X.ndim != 2 or X.shape[1] != self.num_coefs:
            raise IndexError(f"expected X of shape (N, {self.num_coefs}), got {X.shape}")
        y = _observed_value(constraints, "y").astype(np.float32)
        N = X.shape[0]
        if y.shape != (N,):
            raise IndexError(f"expected y of length {N}, got shape {y.shape}")
        staged = np.empty((N, self.num_coefs + 1), dtype=np.float32)
        staged[:, : self.num_coefs] = X
        staged[:, self.num_coefs] = y
        P = self.num_coefs + (1 if self.intercept else 0)
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_GLM_BERNOULLI_LOGIT, num_params=P, num_obs=N, num_coefs=self.num_coefs,
            has_intercept=1 if self.intercept else 0, num_groups=0,
            intercept_mu=self.intercept_mu, intercept_sigma=self.intercept_sigma,
            coef_mu=self.coef_mu, coef_sigma=self.coef_sigma, mu_loc=0.0, mu_scale=1.0, tau_scale=1.0)
        empty = np.zeros(0, dtype=np.int32)
        return Lowered(plan, np.ascontiguousarray(staged.reshape(-1)), empty, empty, P)

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        P = self.num_params(args, constraints)
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, P))
        out = rng.normal(self.coef_mu, self.coef_sigma, size=(num_chains, P))
        if self.intercept:
            out[:, 0] = rng.normal(self.intercept_mu, self.intercept_sigma, size=num_chains)
        return out


@dataclass
class HierarchicalNormalNoncentered(TeaModelSpec):
    """``mu ~ normal(mu_loc, mu_scale)``, ``tau ~ halfcauchy(tau_scale)``,
    ``theta ~ iid(normal(mu, tau), J; reparam=:noncentered)``,
    ``y[j][i] ~ normal(theta[j], sigma[j])``.

    Unconstrained parameters: [mu, log(tau), z_1 .. z_J]; the constrained
    vector is [mu, tau, theta_1 .. theta_J] with theta_j = mu + tau z_j
    (docs/noncentered-reparam.md:22-36).
    args = (sigma, group_sizes); constraints = {"y": y} with y the
    concatenated observations, group after group.
    """

    num_groups: int
    mu_loc: float = 0.0
    mu_scale: float = 5.0
    tau_scale: float = 2.5
    name: str = "hierarchical_normal_noncentered"

    def parameter_names(self, args=(), constraints=None):
        return ["mu", "tau"] + [f"theta[{j + 1}]" for j in range(self.num_groups)]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 2:
            raise ValueError(f"{self.name} expects args=(sigma, group_sizes), got {len(args)} argument(s)")
        sigma = np.asarray(args[0], dtype=np.float32)
        sizes = np.asarray(args[1], dtype=np.int64)
        J = self.num_groups
        if sigma.shape != (J,) or sizes.shape != (J,):
            raise IndexError(f"expected sigma and group_sizes of length {J}, got {sigma.shape} and {sizes.shape}")
        if np.any(sizes < 0):
            raise ValueError("group sizes must be >= 0")
        y = _observed_value(constraints, "y").astype(np.float32)
        N = int(sizes.sum())
        if y.shape != (N,):
            raise IndexError(f"expected {N} observations (sum of group sizes), got shape {y.shape}")
        starts = np.zeros(J, dtype=np.int32)
        starts[1:] = np.cumsum(sizes)[:-1]
        observed = np.concatenate([y, sigma]).astype(np.float32)
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_HIER_NORMAL_NONCENTERED, num_params=J + 2, num_obs=N, num_coefs=0,
            has_intercept=0, num_groups=J, intercept_mu=0.0, intercept_sigma=1.0, coef_mu=0.0, coef_sigma=1.0,
            mu_loc=self.mu_loc, mu_scale=self.mu_scale, tau_scale=self.tau_scale)
        return Lowered(plan, observed, sizes.astype(np.int32), starts, J + 2)

    def constrain(self, unconstrained, args=(), constraints=None):
        u = np.asarray(unconstrained)
        out = np.empty_like(u)
        mu = u[..., 0]
        tau = np.exp(u[..., 1])
        out[..., 0] = mu
        out[..., 1] = tau
        out[..., 2:] = mu[..., None] + tau[..., None] * u[..., 2:]
        return out

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        P = self.num_groups + 2
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, P))
        out = np.empty((num_chains, P))
        out[:, 0] = rng.normal(self.mu_loc, self.mu_scale, size=num_chains)
        tau = np.abs(self.tau_scale * rng.standard_cauchy(size=num_chains))
        out[:, 1] = np.log(np.maximum(tau, 1e-30))
        out[:, 2:] = rng.normal(0.0, 1.0, size=(num_chains, self.num_groups))
        return out


@dataclass
class NormalLocationScale(TeaModelSpec):
    """``mu ~ normal(mu_loc, mu_scale)``, ``s ~ gamma(shape, rate)``,
    ``y[i] ~ normal(mu, s)`` for i = 1..n -- the reference's device-lowerable
    gaussian model (bench/crossppl/julia/models.jl:112-119,
    test/uncertaintea/core/device_lowering_parity.jl:12-19: ``mu ~ normal(0, 1)``,
    ``s ~ gamma(2, 1)``).

    Unconstrained parameters: [mu, log(s)]; constrained: [mu, s].
    args = (n,); constraints = {"y": y} with n observations.
    """

    mu_loc: float = 0.0
    mu_scale: float = 1.0
    shape: float = 2.0
    rate: float = 1.0
    name: str = "normal_location_scale"

    def parameter_names(self, args=(), constraints=None):
        return ["mu", "s"]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 1:
            raise ValueError(f"{self.name} expects args=(n,), got {len(args)} argument(s)")
        n = int(args[0])
        if n < 0:
            raise ValueError("n must be >= 0")
        y = _observed_value(constraints, "y").astype(np.float32).reshape(-1)
        if y.shape != (n,):
            raise IndexError(f"expected {n} observations, got shape {y.shape}")
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_NORMAL_LOCATION_SCALE, num_params=2, num_obs=n, num_coefs=0, has_intercept=0,
            num_groups=0, intercept_mu=0.0, intercept_sigma=1.0, coef_mu=0.0, coef_sigma=1.0,
            mu_loc=self.mu_loc, mu_scale=self.mu_scale, tau_scale=1.0, scale_shape=self.shape,
            scale_rate=self.rate)
        empty = np.zeros(0, dtype=np.int32)
        return Lowered(plan, np.ascontiguousarray(y), empty, empty, 2)

    def constrain(self, unconstrained, args=(), constraints=None):
        u = np.asarray(unconstrained)
        out = np.array(u, dtype=np.float64, copy=True)
        out[..., 1] = np.exp(u[..., 1])
        return out

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, 2))
        out = np.empty((num_chains, 2))
        out[:, 0] = rng.normal(self.mu_loc, self.mu_scale, size=num_chains)
        out[:, 1] = np.log(np.maximum(rng.gamma(self.shape, 1.0 / self.rate, size=num_chains), 1e-30))
        return out


@dataclass
class NormalKnownScale(TeaModelSpec):
    """``mu ~ normal(mu_loc, mu_scale)``, ``y[i] ~ normal(mu, sigma)`` for i = 1..n
    with sigma known -- the reference's conjugate gaussian gate model
    (test/uncertaintea/core/device_persistent_nuts.jl:33-38, device_chees.jl:26-32:
    ``mu ~ normal(0, 1)``, ``{:y} ~ normal(mu, 1)`` observed at y = 0.3, posterior
    normal(0.15, sqrt(0.5))).

    Unconstrained parameter: [mu] (identity transform).
    args = (n,); constraints = {"y": y} with n observations.
    """

    mu_loc: float = 0.0
    mu_scale: float = 1.0
    sigma: float = 1.0
    name: str = "normal_known_scale"

    def parameter_names(self, args=(), constraints=None):
        return ["mu"]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 1:
            raise ValueError(f"{self.name} expects args=(n,), got {len(args)} argument(s)")
        n = int(args[0])
        if n < 0:
            raise ValueError("n must be >= 0")
        y = _observed_value(constraints, "y").astype(np.float32).reshape(-1)
        if y.shape != (n,):
            raise IndexError(f"expected {n} observations, got shape {y.shape}")
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_NORMAL_KNOWN_SCALE, num_params=1, num_obs=n, num_coefs=0, has_intercept=0,
            num_groups=0, intercept_mu=0.0, intercept_sigma=1.0, coef_mu=0.0, coef_sigma=1.0,
            mu_loc=self.mu_loc, mu_scale=self.mu_scale, tau_scale=1.0, obs_scale=self.sigma)
        empty = np.zeros(0, dtype=np.int32)
        return Lowered(plan, np.ascontiguousarray(y), empty, empty, 1)

    def constrain(self, unconstrained, args=(), constraints=None):
        return np.array(unconstrained, dtype=np.float64, copy=True)

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, 1))
        return rng.normal(self.mu_loc, self.mu_scale, size=(num_chains, 1))


@dataclass
class BernoulliBeta(TeaModelSpec):
    """``p ~ beta(alpha, beta)``, ``z[i] ~ bernoulli(p)`` for i = 1..n -- the
    reference's device-lowerable bernoulli model
    (test/uncertaintea/core/device_lowering_parity.jl:30-37: ``p ~ beta(2, 3)``).

    Unconstrained parameter: [logit(p)]; constrained: [p].
    args = (n,); constraints = {"z": z} with z in {0, 1}.
    """

    alpha: float = 2.0
    beta: float = 3.0
    name: str = "bernoulli_beta"

    def parameter_names(self, args=(), constraints=None):
        return ["p"]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 1:
            raise ValueError(f"{self.name} expects args=(n,), got {len(args)} argument(s)")
        n = int(args[0])
        if n < 0:
            raise ValueError("n must be >= 0")
        z = _observed_value(constraints, "z").astype(np.float32).reshape(-1)
        if z.shape != (n,):
            raise IndexError(f"expected {n} observations, got shape {z.shape}")
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_BERNOULLI_BETA, num_params=1, num_obs=n, num_coefs=0, has_intercept=0,
            num_groups=0, intercept_mu=0.0, intercept_sigma=1.0, coef_mu=0.0, coef_sigma=1.0, mu_loc=0.0,
            mu_scale=1.0, tau_scale=1.0, scale_shape=1.0, scale_rate=1.0, prob_alpha=self.alpha,
            prob_beta=self.beta)
        empty = np.zeros(0, dtype=np.int32)
        return Lowered(plan, np.ascontiguousarray(z), empty, empty, 1)

    def constrain(self, unconstrained, args=(), constraints=None):
        u = np.asarray(unconstrained, dtype=np.float64)
        return 1.0 / (1.0 + np.exp(-u))

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, 1))
        p = np.clip(rng.beta(self.alpha, self.beta, size=(num_chains, 1)), 1e-12, 1 - 1e-12)
        return np.log(p) - np.log1p(-p)


@dataclass
class LognormalGammaNormal(TeaModelSpec):
    """``a ~ lognormal(mu, sigma)``, ``b ~ gamma(shape, rate)``, ``scale = exp(a)``,
    ``y[i] ~ normal(b, scale)`` -- the reference's device-lowerable lognormal/gamma
    model (test/uncertaintea/core/device_lowering_parity.jl:21-28:
    ``a ~ lognormal(0, 1)``, ``b ~ gamma(3, 2)``).

    Unconstrained parameters: [log(a), log(b)]; constrained: [a, b].
    args = (n,); constraints = {"y": y}.
    """

    mu: float = 0.0
    sigma: float = 1.0
    shape: float = 3.0
    rate: float = 2.0
    name: str = "lognormal_gamma_normal"

    def parameter_names(self, args=(), constraints=None):
        return ["a", "b"]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 1:
            raise ValueError(f"{self.name} expects args=(n,), got {len(args)} argument(s)")
        n = int(args[0])
        if n < 0:
            raise ValueError("n must be >= 0")
        y = _observed_value(constraints, "y").astype(np.float32).reshape(-1)
        if y.shape != (n,):
            raise IndexError(f"expected {n} observations, got shape {y.shape}")
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_LOGNORMAL_GAMMA_NORMAL, num_params=2, num_obs=n, num_coefs=0, has_intercept=0,
            num_groups=0, intercept_mu=0.0, intercept_sigma=1.0, coef_mu=0.0, coef_sigma=1.0,
            mu_loc=self.mu, mu_scale=self.sigma, tau_scale=1.0, scale_shape=self.shape, scale_rate=self.rate)
        empty = np.zeros(0, dtype=np.int32)
        return Lowered(plan, np.ascontiguousarray(y), empty, empty, 2)

    def constrain(self, unconstrained, args=(), constraints=None):
        return np.exp(np.asarray(unconstrained, dtype=np.float64))

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, 2))
        out = np.empty((num_chains, 2))
        out[:, 0] = rng.normal(self.mu, self.sigma, size=num_chains)
        out[:, 1] = np.log(np.maximum(rng.gamma(self.shape, 1.0 / self.rate, size=num_chains), 1e-30))
        return out


@dataclass
class StudentTHeavyTail(TeaModelSpec):
    """``loc ~ studentt(nu_prior, mu, sigma)``, ``s ~ inversegamma(shape, scale)``,
    ``w ~ weibull(k, lambda)``, ``y[i] ~ studentt(nu_obs, loc, s + w)`` -- the
    reference's device-lowerable heavy-tail model
    (test/uncertaintea/core/device_lowering_parity.jl:51-60: studentt(4, 0, 1),
    inversegamma(3, 2), weibull(2, 1.5), studentt(5, loc, s + w)).

    Unconstrained parameters: [loc, log(s), log(w)]; constrained: [loc, s, w].
    args = (n,); constraints = {"y": y}.
    """

    nu_prior: float = 4.0
    mu: float = 0.0
    sigma: float = 1.0
    ig_shape: float = 3.0
    ig_scale: float = 2.0
    wb_shape: float = 2.0
    wb_scale: float = 1.5
    nu_obs: float = 5.0
    name: str = "studentt_heavy_tail"

    def parameter_names(self, args=(), constraints=None):
        return ["loc", "s", "w"]

    def lower(self, args=(), constraints=None) -> Lowered:
        if len(args) != 1:
            raise ValueError(f"{self.name} expects args=(n,), got {len(args)} argument(s)")
        n = int(args[0])
        if n < 0:
            raise ValueError("n must be >= 0")
        y = _observed_value(constraints, "y").astype(np.float32).reshape(-1)
        if y.shape != (n,):
            raise IndexError(f"expected {n} observations, got shape {y.shape}")
        plan = nat.PlanDesc(
            family=nat.UT_FAMILY_STUDENTT_HEAVY_TAIL, num_params=3, num_obs=n, num_coefs=0, has_intercept=0,
            num_groups=0, intercept_mu=0.0, intercept_sigma=1.0, coef_mu=0.0, coef_sigma=1.0, mu_loc=self.mu,
            mu_scale=self.sigma, tau_scale=1.0, scale_shape=self.ig_shape, scale_rate=self.ig_scale,
            prob_alpha=1.0, prob_beta=1.0, nu_prior=self.nu_prior, nu_obs=self.nu_obs, weibull_shape=self.wb_shape,
            weibull_scale=self.wb_scale)
        empty = np.zeros(0, dtype=np.int32)
        return Lowered(plan, np.ascontiguousarray(y), empty, empty, 3)

    def constrain(self, unconstrained, args=(), constraints=None):
        u = np.asarray(unconstrained, dtype=np.float64)
        out = u.copy()
        out[..., 1:] = np.exp(u[..., 1:])
        return out

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        if init_strategy == "uniform":
            return rng.uniform(-2.0, 2.0, size=(num_chains, 3))
        out = np.empty((num_chains, 3))
        out[:, 0] = self.mu + self.sigma * rng.standard_t(self.nu_prior, size=num_chains)
        out[:, 1] = np.log(self.ig_scale / np.maximum(rng.gamma(self.ig_shape, 1.0, size=num_chains), 1e-30))
        out[:, 2] = np.log(np.maximum(self.wb_scale * rng.weibull(self.wb_shape, size=num_chains), 1e-30))
        return out


# ---- synthetic workloads (seeded stand-ins for the benchmark data sets) -----

def logistic_regression_data(num_obs: int, num_coefs: int, seed: int, x_scale: float = 1.0):
    """X ~ N(0,1) * x_scale (N x D), beta_true ~ N(0,1), y ~ Bernoulli(logistic(X beta))."""
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((num_obs, num_coefs)) * x_scale).astype(np.float32)
    beta = rng.standard_normal(num_coefs)
    eta = X.astype(np.float64) @ beta
    y = (rng.uniform(size=num_obs) < 1.0 / (1.0 + np.exp(-eta))).astype(np.float32)
    return X, y, beta


def hierarchical_data(num_groups: int, group_sizes, seed: int, mu_loc=0.0, mu_scale=5.0, tau_scale=2.5,
                      sigma_range=(0.5, 2.0)):
    """sigma_j ~ U(sigma_range); y drawn from the prior predictive at `seed`."""
    rng = np.random.default_rng(seed)
    sizes = np.broadcast_to(np.asarray(group_sizes, dtype=np.int64), (num_groups,)).copy()
    sigma = rng.uniform(sigma_range[0], sigma_range[1], size=num_groups).astype(np.float32)
    mu = rng.normal(mu_loc, mu_scale)
    tau = abs(tau_scale * rng.standard_cauchy())
    theta = mu + tau * rng.standard_normal(num_groups)
    y = np.concatenate([rng.normal(theta[j], sigma[j], size=sizes[j]) for j in range(num_groups)]).astype(np.float32)
    return y, sigma, sizes, {"mu": mu, "tau": tau, "theta": theta}


def gauss_data(num_obs: int, seed: int, mu_loc=0.0, mu_scale=1.0, shape=2.0, rate=1.0):
    """mu ~ normal(mu_loc, mu_scale), s ~ gamma(shape, rate), y ~ normal(mu, s), seeded."""
    rng = np.random.default_rng(seed)
    mu = rng.normal(mu_loc, mu_scale)
    s = rng.gamma(shape, 1.0 / rate)
    y = rng.normal(mu, s, size=num_obs).astype(np.float32)
    return y, {"mu": mu, "s": s}
