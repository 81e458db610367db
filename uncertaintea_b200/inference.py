"""``UncertainTea.Inference`` mirror: device-resident batched_hmc,
batched_nuts(tree_strategy="persistent") and batched_chees.

The per-iteration work (momentum draws, leapfrog trajectories, NUTS trees,
Metropolis accepts, ChEES cross-chain reductions, the pooled running-variance
update) runs on the GPU through the C ABI.  The host keeps the scalar warmup
state machine -- dual averaging, the windowed mass schedule, step-size
re-searches, the ChEES Adam on log T -- restated from the reference:

* dual averaging: src/inference/nuts/adaptation.jl:1-28
* warmup schedule / windows: adaptation.jl:43-136
* running-variance mass: adaptation.jl:138-223 (update itself on device)
* mass-adaptation weights: adaptation.jl:225-260
* WarmupDriver / PooledMassPerChainStepDriver: src/inference/warmup.jl:12-473
* reasonable step size searches: adaptation.jl:303-514
* ChEES: src/inference/api_batched_chees.jl:25-290

Randomness: the reference draws HMC momenta and accept uniforms on the host
(``randn``/``rand``) and its persistent NUTS kernel on device from Philox.
Here every draw comes from the device Philox stream with the persistent-NUTS
coordinate convention key=(chain, run_seed+iteration), counter=(stream, draw)
(src/device/persistent_nuts.jl:70-73, 700-704); HMC uses stream 0 for momenta
and stream 4 for the accept uniform.  ``rng`` only seeds the run.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .device import DeviceBatchedWorkspace, _check_precision, _resolve_device, _stream_handle

# data_types.jl:189-193
_RUNNING_VARIANCE_CLIP_START = 4
_RUNNING_VARIANCE_CLIP_SCALE_EARLY = 8.0
_RUNNING_VARIANCE_CLIP_SCALE_LATE = 5.0
_RUNNING_VARIANCE_REJECTION_WEIGHT_EARLY = 1.0
_RUNNING_VARIANCE_FLOOR = 1e-3
# api_batched_chees.jl:25-26
_CHEES_LOG_UPDATE_CLIP = 0.35
_CHEES_EPS = 1e-20


def _torch():
    import torch
    return torch


# ---------------------------------------------------------------------------
# warmup schedule (adaptation.jl:103-136)
# ---------------------------------------------------------------------------
@dataclass
class WarmupSchedule:
    initial_buffer: int
    slow_window_ends: list
    terminal_buffer: int


def _warmup_schedule(num_warmup: int) -> WarmupSchedule:
    if num_warmup < 0:
        raise ValueError("warmup schedule requires num_warmup >= 0")
    if num_warmup == 0:
        return WarmupSchedule(0, [], 0)
    if num_warmup < 20:
        initial_buffer = min(5, max(num_warmup - 1, 0))
        if initial_buffer == num_warmup:
            return WarmupSchedule(num_warmup, [], 0)
        return WarmupSchedule(initial_buffer, [num_warmup], 0)
    initial_buffer = min(max(5, num_warmup // 10), num_warmup)
    terminal_buffer = min(max(5, num_warmup // 10), max(num_warmup - initial_buffer, 0))
    slow_budget = num_warmup - initial_buffer - terminal_buffer
    if slow_budget <= 0:
        return WarmupSchedule(num_warmup, [], 0)
    ends = []
    next_size = min(25, slow_budget)
    start = initial_buffer + 1
    remaining = slow_budget
    while remaining > 0:
        size = remaining if remaining <= (3 * next_size) // 2 else next_size
        end = start + size - 1
        ends.append(end)
        remaining -= size
        start = end + 1
        next_size *= 2
    return WarmupSchedule(initial_buffer, ends, terminal_buffer)


def _warmup_window_length(schedule: WarmupSchedule, window_index: int) -> int:
    """1-based window index (adaptation.jl:43-48)."""
    start = schedule.initial_buffer + 1 if window_index == 1 else schedule.slow_window_ends[window_index - 2] + 1
    return schedule.slow_window_ends[window_index - 1] - start + 1


def _warmup_window_start(schedule: WarmupSchedule, window_index: int) -> int:
    """First iteration of a slow window, 1-based window index (adaptation.jl:50-54)."""
    return schedule.initial_buffer + 1 if window_index == 1 else schedule.slow_window_ends[window_index - 2] + 1


def _window_progress(count: int, window_length: int) -> float:  # adaptation.jl:56-65
    if window_length <= _RUNNING_VARIANCE_CLIP_START:
        return 1.0
    return min(max(count - _RUNNING_VARIANCE_CLIP_START, 0) / (window_length - _RUNNING_VARIANCE_CLIP_START), 1.0)


# ---------------------------------------------------------------------------
# dual averaging (adaptation.jl:1-28), vectorised over chains
# ---------------------------------------------------------------------------
class DualAveraging:
    gamma = 0.05
    t0 = 10.0
    kappa = 0.75

    def __init__(self, step_size, target_accept):
        step = np.asarray(step_size, dtype=np.float64)
        self.target_accept = float(target_accept)
        self.mu = np.log(10.0 * step)
        self.log_step_size = np.log(step)
        self.log_step_size_avg = np.log(step)
        self.hbar = np.zeros_like(step)
        self.iteration = 0

    def update(self, accept_prob):
        self.iteration += 1
        eta = 1.0 / (self.iteration + self.t0)
        self.hbar = (1.0 - eta) * self.hbar + eta * (self.target_accept - np.asarray(accept_prob, dtype=np.float64))
        self.log_step_size = self.mu - math.sqrt(self.iteration) / self.gamma * self.hbar
        eta_bar = self.iteration ** (-self.kappa)
        self.log_step_size_avg = eta_bar * self.log_step_size + (1.0 - eta_bar) * self.log_step_size_avg
        return np.exp(self.log_step_size)

    def final(self):
        return np.exp(self.log_step_size_avg)


class DeviceDualAveraging:
    """The DualAveraging state on the device (C x 5 or 5 doubles: mu, log step,
    log step average, hbar, iteration), made from a host DualAveraging and
    updated by ut_warmup_adapt without host copies."""

    def __init__(self, host: DualAveraging, device):
        torch = _torch()
        mu = np.atleast_1d(host.mu)
        cols = [mu, np.atleast_1d(host.log_step_size), np.atleast_1d(host.log_step_size_avg),
                np.atleast_1d(host.hbar), np.full(mu.shape, float(host.iteration))]
        self.per_chain = np.ndim(host.mu) > 0
        self.state = torch.from_numpy(np.ascontiguousarray(np.stack(cols, axis=1), dtype=np.float64)).to(device)


# ---------------------------------------------------------------------------
# running variance with the update on device (adaptation.jl:30-41, 138-223)
# ---------------------------------------------------------------------------
class DeviceRunningVariance:
    def __init__(self, lib, num_params: int, window_length: int, device):
        if window_length <= 0:
            raise ValueError("running variance state requires window_length > 0")
        torch = _torch()
        self.lib = lib
        self.P = num_params
        self.window_length = window_length
        self.state = torch.zeros(2 * num_params + 3, dtype=torch.float64, device=device)
        self.count = 0  # tracked on host: +1 per non-zero weight

    def progress(self) -> float:
        self.sync_count()
        return _window_progress(self.count, self.window_length)

    def clip_scale(self) -> float:
        self.sync_count()
        if self.count <= _RUNNING_VARIANCE_CLIP_START:
            return _RUNNING_VARIANCE_CLIP_SCALE_EARLY
        return _RUNNING_VARIANCE_CLIP_SCALE_EARLY + (
            _RUNNING_VARIANCE_CLIP_SCALE_LATE - _RUNNING_VARIANCE_CLIP_SCALE_EARLY) * self.progress()

    def update_device(self, positions, weights_device):
        """Welford update with device-resident weights (no host copy); the host
        count is then refreshed from the device state when it is needed."""
        nat.check(self.lib.ut_running_variance_update(nat.ptr(positions), nat.ptr(weights_device), self.P,
                                                      positions.shape[0], nat.ptr(self.state), self.window_length,
                                                      _stream_handle()))
        self.count = None

    def sync_count(self):
        if self.count is None:
            self.count = int(round(float(self.state[2 * self.P].item())))

    def update(self, positions, weights: np.ndarray):
        torch = _torch()
        w = np.asarray(weights, dtype=np.float64)
        if np.any(w < 0.0) or np.any(w > 1.0):
            raise ValueError("running variance weight must lie in [0, 1]")
        wd = torch.from_numpy(w).to(positions.device, non_blocking=False)
        nat.check(self.lib.ut_running_variance_update(nat.ptr(positions), nat.ptr(wd), self.P, positions.shape[0],
                                                      nat.ptr(self.state), self.window_length, _stream_handle()))
        self.sync_count()
        self.count += int(np.count_nonzero(w))
        self._wd = wd  # keep alive until the stream has consumed it

    def host_state(self):
        s = self.state.double().cpu().numpy()
        P = self.P
        return s[:P], s[P:2 * P], s[2 * P], s[2 * P + 1], s[2 * P + 2]

    def effective_count(self) -> float:
        _, _, _, ws, wss = self.host_state()
        return 0.0 if wss <= 0 else ws * ws / wss

    def inverse_mass(self, regularization: float) -> np.ndarray:  # adaptation.jl:211-223
        _, m2, _, ws, wss = self.host_state()
        ec = 0.0 if wss <= 0 else ws * ws / wss
        if ec < 2:
            return np.ones(self.P)
        denom = ws - wss / ws
        if denom <= 0:
            return np.ones(self.P)
        variance = m2 / denom
        shrink = ec / (ec + 5.0)
        return np.maximum(shrink * variance + (1.0 - shrink), regularization)


def _mass_adaptation_window_summary(schedule, window_index, variance, inverse_mass, updated) -> dict:
    """One slow window's record at its end (adaptation.jl:143-170): its span, the
    pooled samples, weight sum, effective count and mean weight of the running
    variance, the clip scale at its start and end, whether the mass was updated,
    and the mean / min / max of the diagonal mass (1 / inverse mass) it left."""
    _, _, _, ws, wss = variance.host_state()
    variance.sync_count()
    pooled = int(variance.count)
    mass = 1.0 / np.asarray(inverse_mass, dtype=np.float64)
    return {"window": window_index, "start": _warmup_window_start(schedule, window_index),
            "end": schedule.slow_window_ends[window_index - 1], "window_length": int(variance.window_length),
            "samples": pooled, "weight_sum": float(ws), "effective_count": 0.0 if wss <= 0 else float(ws * ws / wss),
            "mean_weight": 0.0 if pooled == 0 else float(ws) / pooled,
            "clip_scale_start": _RUNNING_VARIANCE_CLIP_SCALE_EARLY, "clip_scale_end": float(variance.clip_scale()),
            "updated": bool(updated), "mass_mean": float(mass.mean()), "mass_min": float(mass.min()),
            "mass_max": float(mass.max())}


def _mass_adaptation_weights(progress: float, accepted, accept_prob, divergent) -> np.ndarray:
    """adaptation.jl:225-260, vectorised."""
    ap = np.asarray(accept_prob, dtype=np.float64)
    acc = np.asarray(accepted, dtype=bool)
    div = np.asarray(divergent, dtype=bool)
    rej = _RUNNING_VARIANCE_REJECTION_WEIGHT_EARLY + (np.clip(ap, 0.0, 1.0)
                                                      - _RUNNING_VARIANCE_REJECTION_WEIGHT_EARLY) * progress
    w = np.where(np.isfinite(ap), rej, 0.0)
    w = np.where(acc, 1.0, w)
    return np.where(div, 0.0, w)


def _mean_batched_adaptation_probability(accept_prob, divergent) -> float:  # hmc_support.jl:635-652
    ap = np.asarray(accept_prob, dtype=np.float64)
    if ap.size == 0:
        return 0.0
    return float(np.sum(np.where(np.asarray(divergent, dtype=bool), 0.0, ap)) / ap.size)


# ---------------------------------------------------------------------------
# warmup drivers (warmup.jl:12-473)
# ---------------------------------------------------------------------------
class WarmupDriver:
    def __init__(self, lib, num_params, num_warmup, initial_step_size, target_accept, *, adapt_step_size,
                 adapt_mass_matrix, mass_matrix_regularization, mass_matrix_min_samples, device,
                 initial_inverse_mass=None):
        self.lib = lib
        self.device = device
        self.schedule = _warmup_schedule(num_warmup)
        self.step_size = float(initial_step_size)
        self.target_accept = float(target_accept)
        self.dual = DualAveraging(self.step_size, self.target_accept)
        first_len = (_RUNNING_VARIANCE_CLIP_START + 16) if not self.schedule.slow_window_ends \
            else _warmup_window_length(self.schedule, 1)
        self.variance = DeviceRunningVariance(lib, num_params, first_len, device)
        self.inverse_mass_matrix = np.ones(num_params) if initial_inverse_mass is None \
            else np.asarray(initial_inverse_mass, dtype=np.float64).copy()
        self.mass_window_index = 1
        self.mass_adaptation_windows = []
        self.num_params = num_params
        self.num_warmup = num_warmup
        self.adapt_step_size = adapt_step_size
        self.adapt_mass_matrix = adapt_mass_matrix
        self.regularization = float(mass_matrix_regularization)
        self.min_samples = int(mass_matrix_min_samples)

    def window_ends_now(self, iteration: int) -> bool:
        s = self.schedule
        return (self.adapt_mass_matrix and self.mass_window_index <= len(s.slow_window_ends)
                and iteration > s.initial_buffer and iteration == s.slow_window_ends[self.mass_window_index - 1])

    def in_mass_window(self, iteration: int) -> bool:
        s = self.schedule
        return (self.adapt_mass_matrix and self.mass_window_index <= len(s.slow_window_ends)
                and iteration > s.initial_buffer)

    def end_window(self):
        """A slow window's end (warmup.jl:262-326): the new inverse mass when the
        window pooled enough samples, the window's record, the next window's
        running variance."""
        s = self.schedule
        updated = False
        if self.variance.effective_count() >= self.min_samples:
            self.inverse_mass_matrix = self.variance.inverse_mass(self.regularization)
            updated = True
        self.mass_adaptation_windows.append(_mass_adaptation_window_summary(
            s, self.mass_window_index, self.variance, self.inverse_mass_matrix, updated))
        self.mass_window_index += 1
        if self.mass_window_index <= len(s.slow_window_ends):
            self.variance = DeviceRunningVariance(
                self.lib, self.num_params, _warmup_window_length(s, self.mass_window_index), self.device)
        else:
            self.variance = DeviceRunningVariance(self.lib, self.num_params,
                                                  _RUNNING_VARIANCE_CLIP_START + 16, self.device)

    def warmup_update(self, iteration, accept_statistic, positions, mass_weights, refind):
        if self.adapt_step_size:
            self.step_size = float(self.dual.update(accept_statistic))
        s = self.schedule
        if self.in_mass_window(iteration):
            self.variance.update(positions, mass_weights)
            if iteration == s.slow_window_ends[self.mass_window_index - 1]:
                self.end_window()
                if self.adapt_step_size and iteration < self.num_warmup and refind is not None:
                    self.step_size = float(refind(self.step_size, self.inverse_mass_matrix))
                    self.dual = DualAveraging(self.step_size, self.target_accept)
        return self.step_size

    def warmup_finalize(self):
        if self.adapt_step_size:
            self.step_size = float(self.dual.final())
        if self.adapt_mass_matrix and self.variance.effective_count() >= self.min_samples:
            self.inverse_mass_matrix = self.variance.inverse_mass(self.regularization)
        return self.step_size


class PooledMassPerChainStepDriver:
    """Shared pooled diagonal mass + per-chain dual-averaged step (warmup.jl:362-473)."""

    def __init__(self, lib, num_params, num_warmup, initial_step_sizes, target_accept, *, adapt_step_size,
                 adapt_mass_matrix, mass_matrix_regularization, mass_matrix_min_samples, device,
                 initial_inverse_mass=None):
        steps = np.asarray(initial_step_sizes, dtype=np.float64)
        self.mass = WarmupDriver(lib, num_params, num_warmup, steps[0] if steps.size else 1.0, target_accept,
                                 adapt_step_size=False, adapt_mass_matrix=adapt_mass_matrix,
                                 mass_matrix_regularization=mass_matrix_regularization,
                                 mass_matrix_min_samples=mass_matrix_min_samples, device=device,
                                 initial_inverse_mass=initial_inverse_mass)
        self.step_sizes = steps.copy()
        self.target_accept = float(target_accept)
        self.dual = DualAveraging(self.step_sizes, self.target_accept)
        self.num_warmup = num_warmup
        self.adapt_step_size = adapt_step_size

    @property
    def inverse_mass_matrix(self):
        return self.mass.inverse_mass_matrix

    def warmup_update(self, iteration, accept_statistics, positions, mass_weights, refind):
        if self.adapt_step_size:
            self.step_sizes = self.dual.update(accept_statistics)
        window_now = self.mass.window_ends_now(iteration)
        self.mass.warmup_update(iteration, 0.0, positions, mass_weights, None)
        if window_now and self.adapt_step_size and iteration < self.num_warmup and refind is not None:
            self.step_sizes = np.asarray(refind(self.step_sizes, self.mass.inverse_mass_matrix), dtype=np.float64)
            self.dual = DualAveraging(self.step_sizes, self.target_accept)
        return self.step_sizes

    def warmup_finalize(self):
        if self.adapt_step_size:
            self.step_sizes = self.dual.final()
        self.mass.warmup_finalize()
        return self.step_sizes


def _device_warmup_iteration(run, driver, per_chain, iteration, num_warmup, accepted, refind, weights):
    """One warmup iteration's adaptation with the per-iteration work on the
    device: ut_warmup_adapt (running-variance weights + dual averaging, the new
    steps written into the sampler's step buffer) and the Welford update with
    device weights -- no host copies.  The host takes over at a mass-window end
    (new inverse mass, window record, step re-search and dual-averaging
    restart, warmup.jl:262-326 / 371-470) and at the end of warmup (final
    steps, final mass).  Same order of operations as the host drivers."""
    lib = run.lib
    mass = driver.mass if per_chain else driver
    adapt = driver.adapt_step_size
    if adapt and getattr(driver, "dual_device", None) is None:
        driver.dual_device = DeviceDualAveraging(driver.dual, run.device)
    in_window = mass.in_mass_window(iteration)
    var = mass.variance
    nat.check(lib.ut_warmup_adapt(
        nat.ptr(run.accept_prob), nat.ptr(accepted), nat.ptr(run.divergent), run.C, run.P, nat.ptr(var.state),
        var.window_length, nat.ptr(weights) if in_window else None,
        nat.ptr(driver.dual_device.state) if adapt else None, 1 if per_chain else 0, 1 if adapt else 0,
        float(driver.target_accept), nat.ptr(run.step), _stream_handle()))
    if in_window:
        var.update_device(run.position, weights)
        if iteration == mass.schedule.slow_window_ends[mass.mass_window_index - 1]:
            mass.end_window()
            steps = run.step.double().cpu().numpy()
            if adapt and iteration < num_warmup and refind is not None:
                steps = np.asarray(refind(steps if per_chain else float(steps[0]), mass.inverse_mass_matrix),
                                   dtype=np.float64)
                driver.dual = DualAveraging(steps if per_chain else float(steps), driver.target_accept)
                driver.dual_device = DeviceDualAveraging(driver.dual, run.device)
            if per_chain:
                driver.step_sizes = np.broadcast_to(steps, (run.C,)).copy()
            else:
                driver.step_size = float(np.ravel(steps)[0])
            run.set_mass_and_step(mass.inverse_mass_matrix, driver.step_sizes if per_chain else driver.step_size)
    if iteration == num_warmup:
        if adapt:
            nat.check(lib.ut_dual_averaging_final(nat.ptr(driver.dual_device.state), run.C, 1 if per_chain else 0,
                                                  nat.ptr(run.step), _stream_handle()))
        steps = run.step.double().cpu().numpy()
        if per_chain:
            driver.step_sizes = steps
        else:
            driver.step_size = float(steps[0])
        if mass.adapt_mass_matrix and mass.variance.effective_count() >= mass.min_samples:
            mass.inverse_mass_matrix = mass.variance.inverse_mass(mass.regularization)
        run.set_mass_and_step(mass.inverse_mass_matrix, driver.step_sizes if per_chain else driver.step_size)


# ---------------------------------------------------------------------------
# ChEES scalar machinery (api_batched_chees.jl:25-290)
# ---------------------------------------------------------------------------
def _halton_base2(index: int) -> float:
    if index < 1:
        raise ValueError(f"Halton index must be >= 1, got {index}")
    result, fraction, remaining = 0.0, 0.5, index
    while remaining > 0:
        result += fraction * (remaining & 1)
        remaining >>= 1
        fraction *= 0.5
    return result


def _chees_jitter_value(jitter_amount: float, iteration: int) -> float:
    return _halton_base2(iteration) * float(jitter_amount) + (1.0 - float(jitter_amount))


def _chees_leapfrog_steps_from_jitter(jitter_value: float, trajectory_length: float, step_size: float) -> int:
    raw = float(jitter_value) * float(trajectory_length) / float(step_size)
    nearest = round(raw)
    steps = int(nearest) if abs(raw - nearest) <= 1e-9 * max(1.0, abs(raw)) else math.ceil(raw)
    return max(1, steps)


def _chees_iteration_step_and_steps(step_size, trajectory_length, jitter_amount, iteration, num_warmup,
                                    fixed_leapfrog_steps=None):
    """The step size and leapfrog step count of ChEES iteration `iteration`
    (1-based).  The reference's rule jitters the step count
    (api_batched_chees.jl:51-56).  With a fixed step count the same Halton
    jitter scales the step size instead, from the first sampling iteration on."""
    jitter = _chees_jitter_value(jitter_amount, iteration)
    L = _chees_leapfrog_steps_from_jitter(jitter, trajectory_length, step_size)
    if fixed_leapfrog_steps is None:
        return float(step_size), L, jitter
    eps = step_size * jitter if iteration > num_warmup else step_size
    return float(eps), int(fixed_leapfrog_steps), jitter


def _chees_jittered_leapfrog_steps(trajectory_length, step_size, jitter_amount, iteration) -> int:
    return _chees_leapfrog_steps_from_jitter(_chees_jitter_value(jitter_amount, iteration), trajectory_length,
                                             step_size)


@dataclass
class ChEESAdamState:
    learning_rate: float
    beta1: float
    beta2: float
    epsilon: float
    m: float = 0.0
    v: float = 0.0
    t: int = 0

    def ascend(self, gradient: float) -> float:
        self.t += 1
        self.m = self.beta1 * self.m + (1.0 - self.beta1) * gradient
        self.v = self.beta2 * self.v + (1.0 - self.beta2) * gradient * gradient
        m_hat = self.m / (1.0 - self.beta1 ** self.t)
        v_hat = self.v / (1.0 - self.beta2 ** self.t)
        return self.learning_rate * m_hat / (math.sqrt(v_hat) + self.epsilon)


@dataclass
class ChEESTrajectoryState:
    trajectory_length: float
    log_trajectory_length_ma: float
    adam: ChEESAdamState
    step: int
    decay_rate: float
    max_leapfrog_steps: int


def _chees_apply_trajectory_gradient(traj: ChEESTrajectoryState, gradient_numerator: float,
                                     acceptance_denominator: float, jitter_value: float,
                                     step_size_for_clip: float) -> float:
    g = (jitter_value * traj.trajectory_length * gradient_numerator / acceptance_denominator
         if acceptance_denominator > 0.0 else 0.0)
    log_t = math.log(traj.trajectory_length)
    saved = (traj.adam.m, traj.adam.v, traj.adam.t)
    raw = traj.adam.ascend(g)
    update = min(max(raw, -_CHEES_LOG_UPDATE_CLIP), _CHEES_LOG_UPDATE_CLIP)
    log_new = log_t + update
    if not math.isfinite(log_new):
        log_new = log_t
        traj.adam.m, traj.adam.v, traj.adam.t = saved
    w = float(traj.step) ** (-traj.decay_rate)
    traj.log_trajectory_length_ma = (1.0 - w) * traj.log_trajectory_length_ma + w * log_new
    new_t = math.exp(traj.log_trajectory_length_ma)
    new_t = min(max(new_t, step_size_for_clip), traj.max_leapfrog_steps * step_size_for_clip)
    traj.trajectory_length = new_t
    traj.step += 1
    return new_t


def _chees_harmonic_mean_accept(accept_prob, divergent) -> float:
    ap = np.asarray(accept_prob, dtype=np.float64)
    div = np.asarray(divergent, dtype=bool)
    keep = ap[~div]
    if keep.size == 0:
        return 0.0
    with np.errstate(divide="ignore"):
        total = float(np.sum(1.0 / keep))
    hm = keep.size / total if total != 0 else math.inf
    return hm if math.isfinite(hm) else 0.0


# ---------------------------------------------------------------------------
# results
# ---------------------------------------------------------------------------
@dataclass
class HMCChains:
    """Draws and per-draw diagnostics of a batched run; arrays are (C, S, ...)."""
    sampler: str
    model: object
    args: tuple
    constraints: object
    unconstrained: np.ndarray
    constrained: np.ndarray
    logjoint: np.ndarray
    accept_prob: np.ndarray
    energy: np.ndarray
    energy_error: np.ndarray
    accepted: np.ndarray
    divergent: np.ndarray
    tree_depth: np.ndarray
    integration_steps: np.ndarray
    step_size: np.ndarray
    inverse_mass_matrix: np.ndarray
    mass_adaptation_windows: list
    warmup_seconds: float
    sampling_seconds: float
    trajectory_length: float = float("nan")
    gradient_evaluations: int = 0
    surrogate: object = None  # report of the learned gradient surrogate, when one drove the run
    max_tree_depth: int = 0   # NUTS: the depth limit (treedepth-saturation diagnostics); 0 otherwise

    @property
    def num_chains(self):
        return self.unconstrained.shape[0]

    @property
    def num_samples(self):
        return self.unconstrained.shape[1]

    def parameter_names(self):
        return self.model.parameter_names(self.args, self.constraints)


def posterior_array(chains: HMCChains, space: str = "constrained") -> np.ndarray:
    return chains.constrained if space == "constrained" else chains.unconstrained


# ---------------------------------------------------------------------------
# device runner shared by the three samplers
# ---------------------------------------------------------------------------
class _DeviceRun:
    def __init__(self, model, args, constraints, num_chains, backend, precision, rng, initial_params,
                 init_strategy, init_max_retries, sampler):
        _check_precision(precision)
        torch = _torch()
        self.torch = torch
        self.device = _resolve_device(backend)
        self.ws = DeviceBatchedWorkspace(model, num_chains, backend=self.device, precision=precision, args=args,
                                         constraints=constraints)
        self.lib = self.ws.lib
        self.model, self.args, self.constraints = model, args, constraints
        self.C = num_chains
        self.P = self.ws.parameter_count
        self.rng = rng if isinstance(rng, np.random.Generator) else np.random.default_rng(rng)
        self.run_seed = int(self.rng.integers(0, 2 ** 32))
        self.probe_counter = 0
        dev = self.device
        f32 = torch.float32
        self.position = torch.empty((self.C, self.P), dtype=f32, device=dev)
        self.gradient = torch.empty_like(self.position)
        self.logjoint = torch.empty(self.C, dtype=f32, device=dev)
        self.inverse_mass = torch.ones(self.P, dtype=f32, device=dev)
        self.step = torch.empty(self.C, dtype=f32, device=dev)
        self.accept_prob = torch.zeros(self.C, dtype=f32, device=dev)
        self.energy = torch.zeros(self.C, dtype=f32, device=dev)
        self.energy_error = torch.zeros(self.C, dtype=f32, device=dev)
        self.accepted = torch.zeros(self.C, dtype=torch.uint8, device=dev)
        self.divergent = torch.zeros(self.C, dtype=torch.uint8, device=dev)
        self.tree_depth = torch.zeros(self.C, dtype=torch.int32, device=dev)
        self.integration_steps = torch.zeros(self.C, dtype=torch.int32, device=dev)
        self._initialize(initial_params, init_strategy, init_max_retries, sampler)

    def coord(self, iteration: int) -> int:
        return (self.run_seed + iteration) & 0xFFFFFFFF

    def _initialize(self, initial_params, init_strategy, init_max_retries, sampler):
        torch = self.torch
        if init_strategy not in ("prior", "uniform"):
            raise ValueError(f"{sampler} init_strategy must be :prior or :uniform, got {init_strategy!r}")
        redrawable = initial_params is None
        if initial_params is None:
            pos = self.model.initial_positions(self.rng, self.C, self.args, self.constraints, init_strategy)
        else:
            ip = np.asarray(initial_params, dtype=np.float64)
            if ip.ndim == 1:
                if ip.shape[0] != self.P:
                    raise IndexError(f"expected {self.P} unconstrained initial parameters, got {ip.shape[0]}")
                pos = np.tile(ip, (self.C, 1))
            else:
                if ip.shape != (self.P, self.C):
                    raise IndexError(f"expected initial_params matrix of size ({self.P}, {self.C}), got {ip.shape}")
                pos = ip.T.copy()
        attempt = 0
        while True:
            self.position.copy_(torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float32)))
            self.ws.logjoint_gradient_device(self.position, self.logjoint, self.gradient)
            lj = self.logjoint.cpu().numpy()
            g = self.gradient.cpu().numpy()
            bad = np.where(~(np.isfinite(lj) & np.all(np.isfinite(g), axis=1)))[0]
            if bad.size == 0:
                break
            if not redrawable or attempt >= init_max_retries:
                retried = f" after {init_max_retries} re-draw(s)" if redrawable else ""
                raise ValueError(
                    f"initial {sampler} parameters produced a non-finite unconstrained logjoint or gradient in "
                    f"{bad.size} of {self.C} chain(s){retried}; try init_strategy=:uniform or supply finite "
                    "initial_params")
            attempt += 1
            fresh = self.model.initial_positions(self.rng, self.C, self.args, self.constraints, init_strategy)
            pos[bad] = fresh[bad]

    def set_mass_and_step(self, inverse_mass, step):
        torch = self.torch
        self.inverse_mass.copy_(torch.from_numpy(np.asarray(inverse_mass, dtype=np.float32)))
        st = np.array(np.broadcast_to(np.asarray(step, dtype=np.float32), (self.C,)))
        self.step.copy_(torch.from_numpy(st))

    def hmc_buffers(self, proposal=None, endpoint_momentum=None):
        return nat.HmcBuffers(
            nat.ptr(self.position), nat.ptr(self.gradient), nat.ptr(self.logjoint), nat.ptr(self.inverse_mass),
            nat.ptr(self.step), nat.ptr(self.accept_prob), nat.ptr(self.energy), nat.ptr(self.energy_error),
            nat.ptr(self.accepted), nat.ptr(self.divergent), nat.ptr(proposal), nat.ptr(endpoint_momentum))

    def hmc_iteration(self, L, iteration, thr, proposal=None, endpoint_momentum=None):
        buf = self.hmc_buffers(proposal, endpoint_momentum)
        nat.check(self.lib.ut_hmc_iteration(self.ws.handle, ctypes.byref(buf), int(L), self.coord(iteration),
                                            float(thr), _stream_handle()))

    def nuts_iteration(self, max_depth, iteration, thr, strategy="persistent"):
        buf = nat.NutsBuffers(
            nat.ptr(self.position), nat.ptr(self.gradient), nat.ptr(self.logjoint), nat.ptr(self.inverse_mass),
            nat.ptr(self.step), nat.ptr(self.accept_prob), nat.ptr(self.energy), nat.ptr(self.energy_error),
            nat.ptr(self.tree_depth), nat.ptr(self.integration_steps), nat.ptr(self.divergent),
            nat.ptr(self.moved if hasattr(self, "moved") else self.accepted))
        fn = self.lib.ut_lockstep_nuts_iteration if strategy == "masked" else self.lib.ut_persistent_nuts_iteration
        nat.check(fn(self.ws.handle, ctypes.byref(buf), int(max_depth), float(thr), self.coord(iteration),
                     _stream_handle()))

    def probe(self, trial_steps, inverse_mass, coord):
        """log accept ratio of one leapfrog step per chain (momentum fixed by `coord`)."""
        torch = self.torch
        im = torch.from_numpy(np.asarray(inverse_mass, dtype=np.float32)).to(self.device)
        ts = torch.from_numpy(np.array(np.broadcast_to(
            np.asarray(trial_steps, dtype=np.float32), (self.C,)))).to(self.device)
        out = torch.empty(self.C, dtype=torch.float32, device=self.device)
        nat.check(self.lib.ut_leapfrog_probe(self.ws.handle, nat.ptr(self.position), nat.ptr(self.gradient),
                                             nat.ptr(self.logjoint), nat.ptr(im), nat.ptr(ts), coord, nat.ptr(out),
                                             _stream_handle()))
        return out.double().cpu().numpy()

    def next_probe_coord(self) -> int:
        self.probe_counter += 1
        return (self.run_seed + 0x80000000 + self.probe_counter) & 0xFFFFFFFF

    # adaptation.jl:303-385 (shared step; one momentum draw for the whole search)
    def find_reasonable_step_size(self, step_size, inverse_mass, divergence_threshold):
        coord = self.next_probe_coord()
        step, lo, hi, target = float(step_size), 1e-8, 1e3, 0.5
        direction = 0.0
        for trial in range(21):
            lar = self.probe(step, inverse_mass, coord)
            ee = np.where(lar == -np.inf, np.inf, -lar)
            div = ~np.isfinite(ee) | (ee > divergence_threshold)
            ap = np.where(~np.isfinite(lar), 0.0, np.where(lar >= 0, 1.0, np.exp(np.minimum(lar, 0.0))))
            mean_ap = _mean_batched_adaptation_probability(ap, div)
            if trial == 0:
                direction = 1.0 if mean_ap > target else -1.0
            elif (direction > 0 and mean_ap <= target) or (direction < 0 and mean_ap >= target):
                break
            nxt = step * (2.0 ** direction)
            if nxt < lo or nxt > hi:
                break
            step = nxt
        return min(max(step, lo), hi)

    # adaptation.jl:438-514 (per-chain steps; one momentum draw per search)
    def find_reasonable_step_size_per_chain(self, step_size, inverse_mass):
        coord = self.next_probe_coord()
        lo, hi, log_target = 1e-8, 1e3, math.log(0.5)
        steps = np.broadcast_to(np.asarray(step_size, dtype=np.float64), (self.C,)).copy()
        done = np.zeros(self.C, dtype=bool)
        lar = self.probe(steps, inverse_mass, coord)
        directions = np.where(lar > log_target, 1.0, -1.0)
        for _ in range(20):
            trial = steps.copy()
            nxt = steps * (2.0 ** directions)
            out_of_range = (~done) & ((nxt < lo) | (nxt > hi))
            done |= out_of_range
            active = ~done
            if not np.any(active):
                break
            trial[active] = nxt[active]
            lar = self.probe(trial, inverse_mass, coord)
            steps[active] = trial[active]
            crossed = ((directions > 0) & (lar <= log_target)) | ((directions < 0) & (lar >= log_target))
            done |= active & crossed
        return np.clip(steps, lo, hi)


def _validate_init(name, init_strategy, init_max_retries):
    """api_batched_nuts.jl:68-71, api_batched_chees.jl:348-351: checked before any
    device work."""
    if init_strategy not in ("prior", "uniform"):
        shown = f":{init_strategy}" if isinstance(init_strategy, str) else repr(init_strategy)
        raise ValueError(f"{name} init_strategy must be :prior or :uniform, got {shown}")
    if init_max_retries < 0:
        raise ValueError(f"{name} init_max_retries must be >= 0, got {init_max_retries}")


def _validate_adtype(name, adtype, backend):
    """The reference's gradient-backend keyword (api_batched_nuts.jl:60-63,
    vi.jl:339-342): one of :auto, :forward, :reverse, and :reverse is host-only.
    Every path here is a device path with analytic gradients (the work of the
    reference's forward-mode duals), so :auto and :forward select it."""
    if adtype not in ("auto", "forward", "reverse"):
        raise ValueError(f"{name} adtype must be :auto, :forward, or :reverse, got {adtype!r}")
    if adtype == "reverse" and backend is not None:
        raise ValueError(f"{name} adtype=:reverse is a host-only path and cannot be combined with a device `backend`")


def _validate_common(num_chains, num_samples, num_warmup, step_size, target_accept, divergence_threshold,
                     mass_matrix_regularization, mass_matrix_min_samples):
    if num_chains < 1:
        raise ValueError(f"num_chains must be >= 1, got {num_chains}")
    if num_samples < 1:
        raise ValueError(f"num_samples must be >= 1, got {num_samples}")
    if num_warmup < 0:
        raise ValueError(f"num_warmup must be >= 0, got {num_warmup}")
    if not (step_size > 0 and math.isfinite(step_size)):
        raise ValueError(f"step_size must be finite and > 0, got {step_size}")
    if not (0 < target_accept < 1):
        raise ValueError(f"target_accept must be in (0, 1), got {target_accept}")
    if not divergence_threshold > 0:
        raise ValueError(f"divergence_threshold must be > 0, got {divergence_threshold}")
    if not mass_matrix_regularization > 0:
        raise ValueError(f"mass_matrix_regularization must be > 0, got {mass_matrix_regularization}")
    if mass_matrix_min_samples < 1:
        raise ValueError(f"mass_matrix_min_samples must be >= 1, got {mass_matrix_min_samples}")


class _DrawBuffer:
    """Per-iteration sampling outputs kept on device until the run ends."""

    def __init__(self, run: _DeviceRun, num_samples: int):
        torch = run.torch
        dev = run.device
        S, C, P = num_samples, run.C, run.P
        self.run = run
        self.pos = torch.empty((S, C, P), dtype=torch.float32, device=dev)
        self.lj = torch.empty((S, C), dtype=torch.float32, device=dev)
        self.ap = torch.empty((S, C), dtype=torch.float32, device=dev)
        self.en = torch.empty((S, C), dtype=torch.float32, device=dev)
        self.ee = torch.empty((S, C), dtype=torch.float32, device=dev)
        self.acc = torch.empty((S, C), dtype=torch.uint8, device=dev)
        self.div = torch.empty((S, C), dtype=torch.uint8, device=dev)
        self.td = torch.empty((S, C), dtype=torch.int32, device=dev)
        self.ist = torch.empty((S, C), dtype=torch.int32, device=dev)

    def record(self, s, accepted=None, tree_depth=None, integration_steps=None):
        r = self.run
        self.pos[s].copy_(r.position)
        self.lj[s].copy_(r.logjoint)
        self.ap[s].copy_(r.accept_prob)
        self.en[s].copy_(r.energy)
        self.ee[s].copy_(r.energy_error)
        self.acc[s].copy_(accepted if accepted is not None else r.accepted)
        self.div[s].copy_(r.divergent)
        if tree_depth is not None:
            self.td[s].copy_(tree_depth)
            self.ist[s].copy_(integration_steps)
        else:
            self.td[s].zero_()
            self.ist[s].fill_(integration_steps if isinstance(integration_steps, int) else 0)

    def host(self, name):
        t = getattr(self, name)
        return t.cpu().numpy().swapaxes(0, 1)


def _finish(sampler, run, draws, step_sizes, inverse_mass, windows, warm_s, samp_s, traj=float("nan"),
            grad_evals=0):
    unconstrained = draws.host("pos")
    constrained = run.model.constrain(unconstrained, run.args, run.constraints)
    return HMCChains(
        sampler=sampler, model=run.model, args=run.args, constraints=run.constraints,
        unconstrained=unconstrained, constrained=constrained, logjoint=draws.host("lj"),
        accept_prob=draws.host("ap"), energy=draws.host("en"), energy_error=draws.host("ee"),
        accepted=draws.host("acc").astype(bool), divergent=draws.host("div").astype(bool),
        tree_depth=draws.host("td"), integration_steps=draws.host("ist"),
        step_size=np.broadcast_to(np.asarray(step_sizes, dtype=np.float64), (run.C,)).copy(),
        inverse_mass_matrix=np.asarray(inverse_mass, dtype=np.float64).copy(), mass_adaptation_windows=windows,
        warmup_seconds=warm_s, sampling_seconds=samp_s, trajectory_length=traj, gradient_evaluations=grad_evals)


def _invoke_callback(callback, every, stage, it, total, step, divergences):
    if callback is not None and (it % every == 0 or it == total):
        callback(stage, it, total, step, divergences)


# ---------------------------------------------------------------------------
# batched_hmc (api_batched_hmc.jl:16-60; device loop hmc_kernels.jl:306-723)
# ---------------------------------------------------------------------------
def batched_hmc(model, args=(), constraints=None, *, num_chains, num_samples, num_warmup=0, step_size=0.1,
                num_leapfrog_steps=10, initial_params=None, target_accept=0.8, adapt_step_size=True,
                adapt_mass_matrix=True, per_chain_adaptation=None, find_reasonable_step_size=False,
                divergence_threshold=1000.0, mass_matrix_regularization=1e-3, mass_matrix_min_samples=10,
                callback=None, callback_every=10, backend="cuda", precision=None, rng=None,
                init_strategy="prior", init_max_retries=100, device_adaptation=True) -> HMCChains:
    """reference: batched_hmc (src/inference/api_batched_hmc.jl:16-300; device loop
    src/device/hmc_kernels.jl:306-723).  With device_adaptation (the default,
    when no callback is given) every warmup iteration's step-size and
    mass-window bookkeeping runs on the device (ut_warmup_adapt), so the host
    only synchronises at mass-window ends; device_adaptation=False runs the
    same arithmetic on the host from O(C) copies per iteration."""
    _validate_init("batched_hmc", init_strategy, init_max_retries)
    _validate_common(num_chains, num_samples, num_warmup, step_size, target_accept, divergence_threshold,
                     mass_matrix_regularization, mass_matrix_min_samples)
    if num_leapfrog_steps < 1:
        raise ValueError(f"num_leapfrog_steps must be >= 1, got {num_leapfrog_steps}")
    per_chain = True if per_chain_adaptation is None else bool(per_chain_adaptation)
    run = _DeviceRun(model, args, constraints, num_chains, backend, precision, rng, initial_params,
                     init_strategy, init_max_retries, "batched HMC")
    torch = run.torch
    P, C = run.P, run.C
    im0 = np.ones(P)
    search = find_reasonable_step_size or (num_warmup > 0 and adapt_step_size)
    if per_chain:
        steps0 = run.find_reasonable_step_size_per_chain(step_size, im0) if search else np.full(C, float(step_size))
        driver = PooledMassPerChainStepDriver(run.lib, P, num_warmup, steps0, target_accept,
                                              adapt_step_size=adapt_step_size, adapt_mass_matrix=adapt_mass_matrix,
                                              mass_matrix_regularization=mass_matrix_regularization,
                                              mass_matrix_min_samples=mass_matrix_min_samples, device=run.device)
        refind = lambda steps, im: run.find_reasonable_step_size_per_chain(steps, im)  # noqa: E731
    else:
        s0 = run.find_reasonable_step_size(step_size, im0, divergence_threshold) if search else float(step_size)
        driver = WarmupDriver(run.lib, P, num_warmup, s0, target_accept, adapt_step_size=adapt_step_size,
                              adapt_mass_matrix=adapt_mass_matrix,
                              mass_matrix_regularization=mass_matrix_regularization,
                              mass_matrix_min_samples=mass_matrix_min_samples, device=run.device)
        refind = lambda s, im: run.find_reasonable_step_size(s, im, divergence_threshold)  # noqa: E731

    draws = _DrawBuffer(run, num_samples)
    total = num_warmup + num_samples
    divergences = 0
    on_device = device_adaptation and callback is None
    div_count = torch.zeros((), dtype=torch.int64, device=run.device)
    weights = torch.empty(C, dtype=torch.float64, device=run.device)
    run.set_mass_and_step(driver.inverse_mass_matrix, driver.step_sizes if per_chain else driver.step_size)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_sample = None
    for it in range(1, total + 1):
        steps = driver.step_sizes if per_chain else driver.step_size
        if not on_device:
            run.set_mass_and_step(driver.inverse_mass_matrix, steps)
        if it == num_warmup + 1:
            torch.cuda.synchronize()
            t_sample = time.perf_counter()
        run.hmc_iteration(num_leapfrog_steps, it, divergence_threshold)
        if it <= num_warmup and on_device:
            div_count += run.divergent.sum()
            _device_warmup_iteration(run, driver, per_chain, it, num_warmup, run.accepted, refind, weights)
            if it == num_warmup:
                divergences = int(div_count.item())
        elif it <= num_warmup:
            ap = run.accept_prob.double().cpu().numpy()
            acc = run.accepted.cpu().numpy().astype(bool)
            div = run.divergent.cpu().numpy().astype(bool)
            divergences += int(div.sum())
            var = driver.mass.variance if per_chain else driver.variance
            weights = _mass_adaptation_weights(var.progress(), acc, ap, div)
            if per_chain:
                stats = np.where(div, 0.0, ap)
                driver.warmup_update(it, stats, run.position, weights, refind)
            else:
                driver.warmup_update(it, _mean_batched_adaptation_probability(ap, div), run.position, weights,
                                     refind)
            if it == num_warmup:
                driver.warmup_finalize()
            _invoke_callback(callback, callback_every, "warmup", it, num_warmup, float(np.mean(steps)), divergences)
        else:
            draws.record(it - num_warmup - 1, integration_steps=num_leapfrog_steps)
            _invoke_callback(callback, callback_every, "sample", it - num_warmup, num_samples, float(np.mean(steps)),
                             divergences)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    if t_sample is None:
        t_sample = t0
    steps = driver.step_sizes if per_chain else driver.step_size
    windows = driver.mass.mass_adaptation_windows if per_chain else driver.mass_adaptation_windows
    out = _finish("hmc", run, draws, steps, driver.inverse_mass_matrix, windows, t_sample - t0, t1 - t_sample,
                  grad_evals=total * num_leapfrog_steps * C)
    out.integration_steps[:] = num_leapfrog_steps
    run.ws.close()
    return out


# ---------------------------------------------------------------------------
# batched_nuts, persistent tree (api_batched_nuts.jl:22-480, 761-961;
# device iteration persistent_nuts.jl:678-761)
# ---------------------------------------------------------------------------
def batched_nuts(model, args=(), constraints=None, *, num_chains, num_samples, num_warmup=0, step_size=0.1,
                 max_tree_depth=10, initial_params=None, init_strategy="prior", init_max_retries=100,
                 target_accept=0.8, adapt_step_size=True, adapt_mass_matrix=True, per_chain_adaptation=None,
                 find_reasonable_step_size=False, divergence_threshold=1000.0, mass_matrix_regularization=1e-3,
                 mass_matrix_min_samples=10, callback=None, callback_every=10, tree_strategy="persistent",
                 backend="cuda", precision=None, persistent_gradient="auto", device_sync_per_leaf=False,
                 adtype="auto", rng=None, device_adaptation=True) -> HMCChains:
    """Batched multinomial NUTS on the device (api_batched_nuts.jl:22-51).

    With device_adaptation (the default, when no callback is given) every
    warmup iteration's dual averaging and mass-window weights run on the device
    (ut_warmup_adapt): warmup copies nothing to the host between mass-window
    ends.  device_adaptation=False runs the same arithmetic on the host.

    tree_strategy "persistent" runs a whole iteration per chain in one launch;
    "masked" grows every chain's tree in lockstep, one leaf per batched
    gradient evaluation.  device_sync_per_leaf is accepted for the reference's
    masked-path debugging switch (a host synchronisation after every leaf); it
    changes no result, and the lockstep driver here reads the live-chain count
    every 16 leaves either way."""
    _validate_adtype("batched_nuts", adtype, backend)
    _validate_init("batched_nuts", init_strategy, init_max_retries)
    if tree_strategy not in ("hybrid", "masked", "persistent"):
        raise ValueError(f"batched_nuts tree_strategy must be :hybrid, :masked, or :persistent, got {tree_strategy!r}")
    if tree_strategy == "hybrid":  # api_batched_nuts.jl:99-102
        raise ValueError("batched_nuts device backend requires tree_strategy=:masked or :persistent, got :hybrid")
    if persistent_gradient not in ("auto", "scalar", "wide"):
        raise ValueError("batched_nuts persistent_gradient must be :auto, :scalar, or :wide")
    if max_tree_depth < 1:
        raise ValueError(f"max_tree_depth must be >= 1, got {max_tree_depth}")
    _validate_common(num_chains, num_samples, num_warmup, step_size, target_accept, divergence_threshold,
                     mass_matrix_regularization, mass_matrix_min_samples)
    per_chain = True if per_chain_adaptation is None else bool(per_chain_adaptation)
    run = _DeviceRun(model, args, constraints, num_chains, backend, precision, rng, initial_params,
                     init_strategy, init_max_retries, "batched NUTS")
    torch = run.torch
    run.moved = torch.zeros(run.C, dtype=torch.uint8, device=run.device)
    P, C = run.P, run.C
    im0 = np.ones(P)
    search = find_reasonable_step_size or (num_warmup > 0 and adapt_step_size)
    if per_chain:
        steps0 = run.find_reasonable_step_size_per_chain(step_size, im0) if search else np.full(C, float(step_size))
        driver = PooledMassPerChainStepDriver(run.lib, P, num_warmup, steps0, target_accept,
                                              adapt_step_size=adapt_step_size, adapt_mass_matrix=adapt_mass_matrix,
                                              mass_matrix_regularization=mass_matrix_regularization,
                                              mass_matrix_min_samples=mass_matrix_min_samples, device=run.device)
        refind = lambda steps, im: run.find_reasonable_step_size_per_chain(steps, im)  # noqa: E731
    else:
        s0 = run.find_reasonable_step_size(step_size, im0, divergence_threshold) if search else float(step_size)
        driver = WarmupDriver(run.lib, P, num_warmup, s0, target_accept, adapt_step_size=adapt_step_size,
                              adapt_mass_matrix=adapt_mass_matrix,
                              mass_matrix_regularization=mass_matrix_regularization,
                              mass_matrix_min_samples=mass_matrix_min_samples, device=run.device)
        refind = lambda s, im: run.find_reasonable_step_size(s, im, divergence_threshold)  # noqa: E731

    draws = _DrawBuffer(run, num_samples)
    total = num_warmup + num_samples
    divergences = 0
    grad_evals = torch.zeros((), dtype=torch.int64, device=run.device)
    on_device = device_adaptation and callback is None
    div_count = torch.zeros((), dtype=torch.int64, device=run.device)
    weights = torch.empty(C, dtype=torch.float64, device=run.device)
    run.set_mass_and_step(driver.inverse_mass_matrix, driver.step_sizes if per_chain else driver.step_size)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_sample = None
    for it in range(1, total + 1):
        steps = driver.step_sizes if per_chain else driver.step_size
        if not on_device:
            run.set_mass_and_step(driver.inverse_mass_matrix, steps)
        if it == num_warmup + 1:
            torch.cuda.synchronize()
            t_sample = time.perf_counter()
        run.nuts_iteration(max_tree_depth, it, divergence_threshold, tree_strategy)
        grad_evals += run.integration_steps.sum()
        if it <= num_warmup and on_device:
            div_count += run.divergent.sum()
            # NUTS has no accept flag: its weights are the rejection weights of the accept statistic
            _device_warmup_iteration(run, driver, per_chain, it, num_warmup, None, refind, weights)
            if it == num_warmup:
                divergences = int(div_count.item())
        elif it <= num_warmup:
            ap = run.accept_prob.double().cpu().numpy()
            div = run.divergent.cpu().numpy().astype(bool)
            divergences += int(div.sum())
            var = driver.mass.variance if per_chain else driver.variance
            weights = _mass_adaptation_weights(var.progress(), np.zeros(C, dtype=bool), ap, div)
            if per_chain:
                driver.warmup_update(it, np.where(div, 0.0, ap), run.position, weights, refind)
            else:
                driver.warmup_update(it, _mean_batched_adaptation_probability(ap, div), run.position, weights,
                                     refind)
            if it == num_warmup:
                driver.warmup_finalize()
            _invoke_callback(callback, callback_every, "warmup", it, num_warmup, float(np.mean(steps)), divergences)
        else:
            draws.record(it - num_warmup - 1, accepted=run.moved, tree_depth=run.tree_depth,
                         integration_steps=run.integration_steps)
            _invoke_callback(callback, callback_every, "sample", it - num_warmup, num_samples, float(np.mean(steps)),
                             divergences)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    if t_sample is None:
        t_sample = t0
    steps = driver.step_sizes if per_chain else driver.step_size
    windows = driver.mass.mass_adaptation_windows if per_chain else driver.mass_adaptation_windows
    out = _finish("nuts", run, draws, steps, driver.inverse_mass_matrix, windows, t_sample - t0, t1 - t_sample,
                  grad_evals=int(grad_evals.item()))
    out.max_tree_depth = int(max_tree_depth)
    run.ws.close()
    return out


# ---------------------------------------------------------------------------
# batched_chees (api_batched_chees.jl:314-746; device loop chees_kernels.jl:108-627)
# ---------------------------------------------------------------------------
def batched_chees(model, args=(), constraints=None, *, num_chains, num_samples, num_warmup=0, step_size=0.1,
                  num_leapfrog_steps=10, jitter_amount=1.0, adapt_trajectory_length=True, max_leapfrog_steps=1000,
                  trajectory_decay_rate=0.5, trajectory_learning_rate=0.5, trajectory_adam_beta1=0.0,
                  trajectory_adam_beta2=0.95, trajectory_adam_epsilon=1e-8, initial_params=None,
                  init_strategy="prior", init_max_retries=100, target_accept=0.651, adapt_step_size=True,
                  adapt_mass_matrix=True, find_reasonable_step_size=False, divergence_threshold=1000.0,
                  mass_matrix_regularization=1e-3, mass_matrix_min_samples=10, callback=None, callback_every=10,
                  backend="cuda", precision=None, rng=None, trajectory_velocity="reference", fixed_leapfrog_steps=None,
                  _trajectory_trace=None, _surrogate=None) -> HMCChains:
    """ChEES-HMC (api_batched_chees.jl:314-347).

    trajectory_velocity selects the endpoint velocity of the trajectory-length
    gradient.  "reference" (default) is the reference's estimator: the endpoint
    momentum after the reversible leapfrog's final negation
    (chees_kernels.jl:392-396, integrator.jl:146-220) under an Adam ascent on
    log T (api_batched_chees.jl:150-157), which makes its sign that of
    -dChEES/dlog T.  "forward" uses the velocity the trajectory ends with
    (the criterion's own derivative), so the ascent maximises ChEES as the
    reference documents; it is the same reduction with the numerator negated.

    fixed_leapfrog_steps (an addition; default None = the reference's rule)
    makes every iteration run exactly that many leapfrog steps, with no
    trajectory-length adaptation: a fixed trajectory budget, as the learned-
    surrogate comparison at 16 steps uses.  The Halton jitter, which the
    reference's rule applies to the step count, then applies to the step size
    of each sampling iteration (eps * j_i, j_i in [1 - jitter_amount, 1)): the
    gradient budget stays fixed, and a direction whose oscillation period
    divides the trajectory length no longer returns to its start every
    iteration (that resonance took one direction's ESS down 30x between runs
    whose adapted step sizes differed by 8 %).  jitter_amount=0 turns it off.
    """
    if fixed_leapfrog_steps is not None:
        if int(fixed_leapfrog_steps) < 1:
            raise ValueError(f"fixed_leapfrog_steps must be >= 1, got {fixed_leapfrog_steps}")
        adapt_trajectory_length = False
    _validate_init("batched_chees", init_strategy, init_max_retries)
    if trajectory_velocity not in ("reference", "forward"):
        raise ValueError(f"batched_chees trajectory_velocity must be 'reference' or 'forward', got {trajectory_velocity!r}")
    if not 0.0 <= jitter_amount <= 1.0:
        raise ValueError(f"batched_chees jitter_amount must be in [0, 1], got {jitter_amount}")
    if max_leapfrog_steps < 1:
        raise ValueError(f"batched_chees max_leapfrog_steps must be >= 1, got {max_leapfrog_steps}")
    if not 0.0 < trajectory_decay_rate <= 1.0:
        raise ValueError(f"batched_chees trajectory_decay_rate must be in (0, 1], got {trajectory_decay_rate}")
    if not trajectory_learning_rate > 0.0:
        raise ValueError(f"batched_chees trajectory_learning_rate must be > 0, got {trajectory_learning_rate}")
    if not 0.0 <= trajectory_adam_beta1 < 1.0:
        raise ValueError(f"batched_chees trajectory_adam_beta1 must be in [0, 1), got {trajectory_adam_beta1}")
    if not 0.0 <= trajectory_adam_beta2 < 1.0:
        raise ValueError(f"batched_chees trajectory_adam_beta2 must be in [0, 1), got {trajectory_adam_beta2}")
    if not trajectory_adam_epsilon > 0.0:
        raise ValueError(f"batched_chees trajectory_adam_epsilon must be > 0, got {trajectory_adam_epsilon}")
    if num_leapfrog_steps < 1:
        raise ValueError(f"num_leapfrog_steps must be >= 1, got {num_leapfrog_steps}")
    _validate_common(num_chains, num_samples, num_warmup, step_size, target_accept, divergence_threshold,
                     mass_matrix_regularization, mass_matrix_min_samples)
    run = _DeviceRun(model, args, constraints, num_chains, backend, precision, rng, initial_params,
                     init_strategy, init_max_retries, "batched ChEES")
    torch = run.torch
    P, C = run.P, run.C
    im0 = np.ones(P)
    s0 = float(step_size)
    if find_reasonable_step_size or (num_warmup > 0 and adapt_step_size):
        s0 = run.find_reasonable_step_size(s0, im0, divergence_threshold)
    driver = WarmupDriver(run.lib, P, num_warmup, s0, target_accept, adapt_step_size=adapt_step_size,
                          adapt_mass_matrix=adapt_mass_matrix, mass_matrix_regularization=mass_matrix_regularization,
                          mass_matrix_min_samples=mass_matrix_min_samples, device=run.device)
    refind = lambda s, im: run.find_reasonable_step_size(s, im, divergence_threshold)  # noqa: E731
    t_init = num_leapfrog_steps * s0
    traj = ChEESTrajectoryState(t_init, math.log(t_init),
                                ChEESAdamState(trajectory_learning_rate, trajectory_adam_beta1, trajectory_adam_beta2,
                                               trajectory_adam_epsilon), 1, float(trajectory_decay_rate),
                                max_leapfrog_steps)
    adapt_traj = num_warmup > 0 and adapt_trajectory_length
    initials = torch.empty_like(run.position) if adapt_traj else None
    proposal = torch.empty_like(run.position) if adapt_traj else None
    momentum = torch.empty_like(run.position) if adapt_traj else None
    out2 = (ctypes.c_double * 2)()
    draws = _DrawBuffer(run, num_samples)
    total = num_warmup + num_samples
    divergences = 0
    grad_evals = 0
    if _surrogate is not None:
        _surrogate.setup(run, num_warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_sample = None
    for it in range(1, total + 1):
        eps, L, jitter = _chees_iteration_step_and_steps(driver.step_size, traj.trajectory_length, jitter_amount,
                                                         it, num_warmup, fixed_leapfrog_steps)
        run.set_mass_and_step(driver.inverse_mass_matrix, eps)
        if it == num_warmup + 1:
            torch.cuda.synchronize()
            t_sample = time.perf_counter()
        warm = it <= num_warmup
        if warm and adapt_trajectory_length:
            initials.copy_(run.position)
        if _surrogate is not None:
            L = _surrogate.cap_steps(L)
            grad_evals += _surrogate.iteration(run, L, it, divergence_threshold, warm,
                                               proposal if (warm and adapt_traj) else None,
                                               momentum if (warm and adapt_traj) else None)
        else:
            run.hmc_iteration(L, it, divergence_threshold, proposal if (warm and adapt_traj) else None,
                              momentum if (warm and adapt_traj) else None)
            grad_evals += L * C
        if warm:
            ap = run.accept_prob.double().cpu().numpy()
            acc = run.accepted.cpu().numpy().astype(bool)
            div = run.divergent.cpu().numpy().astype(bool)
            divergences += int(div.sum())
            num = den = 0.0
            if adapt_trajectory_length:
                nat.check(run.lib.ut_chees_reduce(run.ws.handle, nat.ptr(initials), nat.ptr(proposal),
                                                  nat.ptr(momentum), nat.ptr(run.accept_prob),
                                                  nat.ptr(run.divergent), nat.ptr(run.inverse_mass), out2,
                                                  _stream_handle()))
                num, den = out2[0], out2[1]
                if trajectory_velocity == "forward":
                    num = -num
            weights = _mass_adaptation_weights(driver.variance.progress(), acc, ap, div)
            driver.warmup_update(it, _chees_harmonic_mean_accept(ap, div), run.position, weights, refind)
            if adapt_trajectory_length:
                _chees_apply_trajectory_gradient(traj, num, den, jitter, driver.step_size)
                if _trajectory_trace is not None:
                    _trajectory_trace.append(traj.trajectory_length)
            if _surrogate is not None:
                _surrogate.after_warmup_iteration(run, it)
            if it == num_warmup:
                driver.warmup_finalize()
                if _surrogate is not None:
                    # Philox coordinates past the run's own iterations
                    steps_fn = _chees_leapfrog_steps_from_jitter if fixed_leapfrog_steps is None else \
                        (lambda _j, _t, _e: int(fixed_leapfrog_steps))
                    _surrogate.end_warmup(run, driver, traj, lambda i: _chees_jitter_value(jitter_amount, i),
                                          steps_fn, divergence_threshold, total + 1)
            _invoke_callback(callback, callback_every, "warmup", it, num_warmup, driver.step_size, divergences)
        else:
            draws.record(it - num_warmup - 1, integration_steps=L)
            draws.ist[it - num_warmup - 1].fill_(L)
            _invoke_callback(callback, callback_every, "sample", it - num_warmup, num_samples, driver.step_size,
                             divergences)
    if _surrogate is not None:
        _surrogate.finish(run)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    if t_sample is None:
        t_sample = t0
    out = _finish("chees", run, draws, driver.step_size, driver.inverse_mass_matrix, driver.mass_adaptation_windows,
                  t_sample - t0, t1 - t_sample, traj=traj.trajectory_length, grad_evals=grad_evals)
    run.ws.close()
    return out
