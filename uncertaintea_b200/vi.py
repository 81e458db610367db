"""Mean-field ADVI on the device (the reference's device ADVI path).

``batched_advi`` mirrors the reference's ``batched_advi(...; backend)`` device
branch (src/inference/vi.jl:314-400 -> src/device/advi_kernels.jl:45-209): the
particles of every step are scored by the workspace's batched gradient kernel
and reduced on the device (``ut_advi_step``), the Adam ascent, gradient clip and
ELBO bookkeeping run on the host in float64 (vi.jl:179-227, guides.jl:23-57).
The device path supports the mean-field guide and the standard ELBO only, as the
reference's does.  Differences: the particle noise is drawn on the device from
the Philox stream (coordinate = particle, run_seed + iteration, stream 5,
parameter) instead of the host RNG, and an unsupported model raises from the
workspace before any step.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .device import DeviceBatchedWorkspace, _stream_handle, _torch


@dataclass
class ADVIResult:
    """Fitted mean-field Gaussian in unconstrained space (vi.jl:3-40)."""
    model: object
    args: tuple
    constraints: object
    location: np.ndarray
    log_scale: np.ndarray
    best_location: np.ndarray
    best_log_scale: np.ndarray
    elbo_history: np.ndarray
    gradient_norm_history: np.ndarray
    best_elbo: float
    num_particles: int
    learning_rate: float
    gradient_backend: str = "device"
    guide: str = "meanfield"


def _gaussian_entropy(log_scale) -> float:
    """Entropy of a diagonal Gaussian (guides.jl:51-57)."""
    ls = np.asarray(log_scale, dtype=np.float64)
    return 0.5 * ls.size * (1.0 + math.log(2.0 * math.pi)) + float(ls.sum())


def _clip_advi_gradients(location_gradient, log_scale_gradient, gradient_clip) -> float:
    """Joint L2 clip of both gradients in place; returns the norm used (vi.jl:179-203)."""
    norm = math.sqrt(float(np.dot(location_gradient, location_gradient) + np.dot(log_scale_gradient,
                                                                                log_scale_gradient)))
    if math.isfinite(gradient_clip) and norm > gradient_clip:
        f = gradient_clip / norm
        location_gradient *= f
        log_scale_gradient *= f
        return float(gradient_clip)
    return norm


def _adam_ascent_step(params, m1, m2, grad, iteration, lr, beta1, beta2, eps):
    """Adam ascent in place (vi.jl:205-227)."""
    c1 = 1.0 - beta1 ** iteration
    c2 = 1.0 - beta2 ** iteration
    m1 *= beta1
    m1 += (1.0 - beta1) * grad
    m2 *= beta2
    m2 += (1.0 - beta2) * grad * grad
    params += lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps)
    return params


def _resolve_scale_vector(name, scale, parameter_total):
    if np.isscalar(scale):
        return np.full(parameter_total, float(scale))
    v = np.asarray(scale, dtype=np.float64).reshape(-1)
    if v.size != parameter_total:
        raise IndexError(f"expected {name} to have length {parameter_total}, got {v.size}")
    return v.copy()


def batched_advi(model, args=(), constraints=None, *, num_iterations, num_particles=32, learning_rate=0.05,
                 initial_params=None, initial_log_scale=-1.0, guide="meanfield", lowrank_rank=1, num_flow_layers=4,
                 elbo="standard", iwae_samples=0, beta1=0.9, beta2=0.999, adam_epsilon=1e-8, gradient_clip=math.inf,
                 callback=None, callback_every=10, backend="cuda", precision=None, adtype="auto",
                 rng=None) -> ADVIResult:
    """Mean-field ADVI with ``num_particles`` particles per Adam step, run for
    ``num_iterations`` steps on the device (vi.jl:314; advi_kernels.jl:45).
    lowrank_rank and num_flow_layers belong to the reference's host-only
    :lowrank and :flow guides; like the reference's mean-field path, this one
    accepts and ignores them."""
    from .inference import _validate_adtype
    _validate_adtype("batched_advi", adtype, backend)
    if guide not in ("meanfield", "fullrank", "lowrank", "flow"):
        raise ValueError(f"batched_advi guide must be :meanfield, :fullrank, :lowrank, or :flow, got {guide}")
    if elbo not in ("standard", "iwae"):
        raise ValueError(f"batched_advi elbo must be :standard or :iwae, got {elbo}")
    if guide != "meanfield":
        raise ValueError(f"batched_advi guide={guide} is CPU-only; the device path supports :meanfield")
    if elbo != "standard":
        raise ValueError("batched_advi elbo=:iwae is CPU-only; the device path supports the standard ELBO")
    if num_iterations <= 0:
        raise ValueError("batched_advi requires num_iterations > 0")
    if num_particles <= 0:
        raise ValueError("batched_advi requires num_particles > 0")
    if not learning_rate > 0:
        raise ValueError("batched_advi requires learning_rate > 0")
    if not 0 <= beta1 < 1:
        raise ValueError("batched_advi requires 0 <= beta1 < 1")
    if not 0 <= beta2 < 1:
        raise ValueError("batched_advi requires 0 <= beta2 < 1")
    if not adam_epsilon > 0:
        raise ValueError("batched_advi requires adam_epsilon > 0")
    if not gradient_clip > 0:
        raise ValueError("batched_advi requires gradient_clip > 0")
    if precision not in (None, "float32", np.float32):
        raise ValueError(f"the B200 backend does not support {precision} arithmetic; request precision=Float32")
    torch = _torch()
    gen = rng if isinstance(rng, np.random.Generator) else np.random.default_rng(rng)
    run_seed = int(gen.integers(0, 2 ** 32))
    ws = DeviceBatchedWorkspace(model, num_particles, args=args, constraints=constraints)
    try:
        P, M = ws.parameter_count, num_particles
        if P < 1:
            raise ValueError("batched_advi requires at least one parameterized latent choice")
        if initial_params is None:
            location = np.asarray(model.initial_positions(gen, 1, args, constraints, "prior")[0], dtype=np.float64)
        else:
            location = np.asarray(initial_params, dtype=np.float64).reshape(-1).copy()
            if location.size != P:
                raise IndexError(f"expected initial_params to have length {P} in unconstrained space, "
                                 f"got {location.size}")
        log_scale = _resolve_scale_vector("initial_log_scale", initial_log_scale, P)
        dev = torch.device("cuda")
        f32 = torch.float32
        loc_d = torch.empty(P, dtype=f32, device=dev)
        scale_d = torch.empty(P, dtype=f32, device=dev)
        particles = torch.empty((M, P), dtype=f32, device=dev)
        values = torch.empty(M, dtype=f32, device=dev)
        grads = torch.empty((M, P), dtype=f32, device=dev)
        lg_d = torch.empty(P, dtype=f32, device=dev)
        sg_d = torch.empty(P, dtype=f32, device=dev)
        host = torch.empty(M + 2 * P, dtype=f32, pin_memory=True)
        m_loc, v_loc = np.zeros(P), np.zeros(P)
        m_ls, v_ls = np.zeros(P), np.zeros(P)
        elbo_history = np.empty(num_iterations)
        norm_history = np.empty(num_iterations)
        best_location, best_log_scale, best_elbo = location.copy(), log_scale.copy(), -math.inf
        lib = nat.load()
        for it in range(1, num_iterations + 1):
            loc_d.copy_(torch.from_numpy(location.astype(np.float32)))
            scale_d.copy_(torch.from_numpy(np.exp(log_scale).astype(np.float32)))
            nat.check(lib.ut_advi_step(ws.handle, nat.ptr(loc_d), nat.ptr(scale_d), (run_seed + it) & 0xFFFFFFFF,
                                       nat.ptr(particles), nat.ptr(values), nat.ptr(grads), nat.ptr(lg_d),
                                       nat.ptr(sg_d), _stream_handle()))
            host[:M].copy_(values)
            host[M:M + P].copy_(lg_d)
            host[M + P:].copy_(sg_d)
            torch.cuda.current_stream().synchronize()
            h = host.numpy().astype(np.float64)
            vals, loc_grad, scale_grad = h[:M], h[M:M + P].copy(), h[M + P:]
            if not (np.all(np.isfinite(vals)) and np.all(np.isfinite(loc_grad)) and np.all(np.isfinite(scale_grad))):
                raise ValueError("batched_advi encountered only non-finite unconstrained logjoint values or gradients")
            log_scale_grad = 1.0 + scale_grad
            norm_history[it - 1] = _clip_advi_gradients(loc_grad, log_scale_grad, gradient_clip)
            e = float(vals.mean()) + _gaussian_entropy(log_scale)
            elbo_history[it - 1] = e
            if e > best_elbo:
                best_elbo, best_location, best_log_scale = e, location.copy(), log_scale.copy()
            _adam_ascent_step(location, m_loc, v_loc, loc_grad, it, float(learning_rate), beta1, beta2, adam_epsilon)
            _adam_ascent_step(log_scale, m_ls, v_ls, log_scale_grad, it, float(learning_rate), beta1, beta2,
                              adam_epsilon)
            if callback is not None and (it % callback_every == 0 or it == num_iterations):
                callback("step", it, num_iterations, math.nan, 0)
        return ADVIResult(model, args, constraints, location, log_scale, best_location, best_log_scale,
                          elbo_history, norm_history, best_elbo, M, float(learning_rate))
    finally:
        ws.close()


def variational_mean(result: ADVIResult, space="constrained", use_best=True) -> np.ndarray:
    """Mean of the fitted Gaussian: the location (vi.jl:229-247)."""
    loc = result.best_location if use_best else result.location
    if space == "unconstrained":
        return loc.copy()
    if space == "constrained":
        return np.asarray(result.model.constrain(loc[None, :], result.args, result.constraints))[0]
    raise ValueError("variational space must be :constrained or :unconstrained")


def variational_samples(result: ADVIResult, *, num_samples, space="constrained", use_best=True,
                        rng=None) -> np.ndarray:
    """Draws from the fitted Gaussian, P x num_samples (vi.jl:249-290)."""
    if num_samples <= 0:
        raise ValueError("variational_samples requires num_samples > 0")
    gen = rng if isinstance(rng, np.random.Generator) else np.random.default_rng(rng)
    loc = result.best_location if use_best else result.location
    ls = result.best_log_scale if use_best else result.log_scale
    u = loc[:, None] + np.exp(ls)[:, None] * gen.standard_normal((loc.size, num_samples))
    if space == "unconstrained":
        return u
    if space == "constrained":
        return np.asarray(result.model.constrain(u.T, result.args, result.constraints)).T
    raise ValueError("variational space must be :constrained or :unconstrained")
