"""Learned gradient surrogate for ChEES-HMC (no counterpart in the reference).

An MLP  P -> 256 -> 256 -> P  (SiLU) is trained by the library's own forward,
backward and Adam kernels (``uncertaintea_b200/csrc/ut_mlp.cuh``) on
(unconstrained position, exact logjoint gradient) pairs that the exact ChEES
warmup produces.  It then drives the leapfrog kicks of the sampling
trajectories while the Metropolis accept uses the exact device logjoint: the
leapfrog map of any position-only force field is volume-preserving and
reversible, so the chains keep the exact posterior as their target whatever
the surrogate's error.  Exact gradients remain the fallback when the accept
rate drops, and the measure of the surrogate's error.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .device import _stream_handle

HIDDEN = 256
MAX_PARAMS = 128


def _torch():
    import torch
    return torch


def weight_layout(num_params: int) -> dict:
    """Slices of the flat weight array: W1 (256, Pp), b1 (256,), W2 (256, 256),
    b2 (256,), W3 (Pp, 256), b3 (Pp,), with Pp = num_params rounded up to 16
    (entries at index >= num_params are zero)."""
    pp = (num_params + 15) // 16 * 16
    out, off = {}, 0
    for name, shape in (("W1", (HIDDEN, pp)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
                        ("W3", (pp, HIDDEN)), ("b3", (pp,))):
        n = int(np.prod(shape))
        out[name] = (slice(off, off + n), shape)
        off += n
    out["total"] = off
    out["padded_params"] = pp
    return out


def _dev_f32(t, shape, name):
    torch = _torch()
    if not (torch.is_tensor(t) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError(f"{name} must be a contiguous float32 CUDA tensor")
    if tuple(t.shape) != tuple(shape):
        raise IndexError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t


class GradientSurrogate:
    """The surrogate network on the current CUDA device (weights, Adam state,
    normalisation), driven through the library's C ABI."""

    def __init__(self, num_params: int, seed: int = 0):
        if not 1 <= num_params <= MAX_PARAMS:
            raise ValueError(f"the gradient surrogate supports 1..{MAX_PARAMS} parameters, got {num_params}")
        self.lib = nat.load()
        self.P = int(num_params)
        h = ctypes.c_void_p()
        nat.check(self.lib.ut_surrogate_create(self.P, int(seed) & 0xFFFFFFFF, ctypes.byref(h)))
        self.handle = h
        n = ctypes.c_int64()
        nat.check(self.lib.ut_surrogate_num_weights(self.handle, ctypes.byref(n)))
        self.num_weights = int(n.value)

    # ---- weights and normalisation (host copies) ----
    def get_weights(self) -> np.ndarray:
        w = np.empty(self.num_weights, dtype=np.float32)
        nat.check(self.lib.ut_surrogate_get_weights(self.handle, w.ctypes.data, w.size))
        return w

    def set_weights(self, weights) -> None:
        w = np.ascontiguousarray(weights, dtype=np.float32)
        nat.check(self.lib.ut_surrogate_set_weights(self.handle, w.ctypes.data, w.size))

    def get_normalization(self) -> np.ndarray:
        """(4, P): in_mean, in_scale, out_mean, out_scale."""
        out = np.empty(4 * self.P, dtype=np.float32)
        nat.check(self.lib.ut_surrogate_get_normalization(self.handle, out.ctypes.data))
        return out.reshape(4, self.P)

    def set_normalization(self, norm) -> None:
        a = np.ascontiguousarray(np.asarray(norm, dtype=np.float32).reshape(-1))
        if a.size != 4 * self.P:
            raise IndexError(f"normalisation needs 4 x {self.P} entries, got {a.size}")
        nat.check(self.lib.ut_surrogate_set_normalization(self.handle, a.ctypes.data))

    def fit_normalization(self, theta, grad) -> None:
        n = theta.shape[0]
        _dev_f32(theta, (n, self.P), "theta")
        _dev_f32(grad, (n, self.P), "grad")
        nat.check(self.lib.ut_surrogate_fit_normalization(self.handle, nat.ptr(theta), nat.ptr(grad), n,
                                                          _stream_handle()))

    # ---- training ----
    def train(self, theta, grad, *, steps: int, batch: int = 4096, learning_rate: float = 2e-3,
              final_learning_rate: float = 1e-4, seed: int = 0, index=None):
        """Adam steps on the pairs (theta, grad) (device tensors, n x P);
        returns the per-step batch losses as a device tensor."""
        torch = _torch()
        n = theta.shape[0]
        _dev_f32(theta, (n, self.P), "theta")
        _dev_f32(grad, (n, self.P), "grad")
        if index is not None and (not index.is_cuda or index.dtype != torch.int32 or index.numel() != steps * batch):
            raise ValueError("index must be an int32 CUDA tensor of steps * batch entries")
        losses = torch.empty(steps, dtype=torch.float32, device=theta.device)
        nat.check(self.lib.ut_surrogate_train(self.handle, nat.ptr(theta), nat.ptr(grad), n, nat.ptr(index),
                                              int(batch), int(steps), float(learning_rate),
                                              float(final_learning_rate), int(seed) & 0xFFFFFFFF, nat.ptr(losses),
                                              _stream_handle()))
        return losses

    def loss_gradient(self, theta, grad, index):
        """(loss, weight gradient) of one batch of pair rows, no update."""
        torch = _torch()
        n = theta.shape[0]
        _dev_f32(theta, (n, self.P), "theta")
        _dev_f32(grad, (n, self.P), "grad")
        if not (index.is_cuda and index.dtype == torch.int32):
            raise ValueError("index must be an int32 CUDA tensor")
        wg = torch.empty(self.num_weights, dtype=torch.float32, device=theta.device)
        loss = torch.empty(1, dtype=torch.float32, device=theta.device)
        nat.check(self.lib.ut_surrogate_loss_gradient(self.handle, nat.ptr(theta), nat.ptr(grad), n, nat.ptr(index),
                                                      index.numel(), nat.ptr(wg), nat.ptr(loss), _stream_handle()))
        return loss, wg

    def gradient(self, theta, out=None):
        """Surrogate gradient at the rows of theta (n x P device tensor)."""
        n = theta.shape[0]
        _dev_f32(theta, (n, self.P), "theta")
        if out is None:
            out = _torch().empty_like(theta)
        nat.check(self.lib.ut_surrogate_gradient(self.handle, nat.ptr(theta), n, nat.ptr(out), _stream_handle()))
        return out

    def relative_error(self, theta, grad) -> float:
        """||surrogate - grad||_F / ||grad - mean(grad)||_F over the rows: 0 is
        exact, 1 is no better than the mean gradient."""
        torch = _torch()
        est = self.gradient(theta)
        num = torch.linalg.norm((est - grad).double())
        den = torch.linalg.norm((grad - grad.mean(dim=0, keepdim=True)).double())
        return float(num / den)

    def check(self) -> None:
        nat.check(self.lib.ut_surrogate_check(self.handle, _stream_handle()))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            nat.check(self.lib.ut_surrogate_destroy(self.handle))
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class SurrogateReport:
    """What the surrogate did in a run."""
    num_pairs: int = 0
    train_steps: int = 0
    train_seconds: float = 0.0
    final_loss: float = float("nan")
    relative_error_after_training: float = float("nan")
    relative_error_checks: list = field(default_factory=list)
    surrogate_iterations: int = 0
    exact_iterations_after_warmup: int = 0
    fallback_at: int | str | None = None  # sampling iteration, "training" or "readapt"
    readapted_step_size: float = float("nan")


class SurrogateChEESController:
    """Hooks the surrogate into batched_chees.

    Warmup: exact iterations; the (position, exact gradient) pairs of the
    last iterations (at most the last 60% of warmup, so the initial transient
    is left out) are copied into a device pair buffer, ``num_pairs`` rows at
    most.  End of warmup: normalisation, Adam over the pairs
    (max(``min_train_steps``, ``train_epochs`` passes) steps of ``batch``
    rows), then ``readapt_iterations`` surrogate iterations that
    re-tune the step size by dual averaging (the surrogate's energy error
    differs from the exact one).  Sampling: surrogate iterations; when the
    mean accept probability over the last ``fallback_window`` iterations falls
    below ``fallback_accept``, the exact gradient is recomputed and every
    later iteration is exact.  Every ``error_check_every`` sampling iterations
    the surrogate is compared with the exact gradient at the current
    positions (one extra exact gradient evaluation).  A surrogate whose
    relative error after training is not below ``max_relative_error`` is not
    used, and neither is one whose step-size re-tuning fails (accept rate
    below ``fallback_accept`` over ``fallback_window`` iterations, or the step
    shrinking 64-fold): the run then continues with exact gradients."""

    def __init__(self, *, num_pairs=2 ** 20, train_epochs=8, min_train_steps=10000, batch=4096, learning_rate=2e-3,
                 final_learning_rate=1e-5, readapt_iterations=100, fallback_accept=0.2, fallback_window=20,
                 error_check_every=0, seed=0, surrogate=None, train=True, max_relative_error=0.5):
        self.num_pairs = int(num_pairs)
        self.train_epochs = float(train_epochs)
        self.min_train_steps = int(min_train_steps)
        self.batch = int(batch)
        self.learning_rate = float(learning_rate)
        self.final_learning_rate = float(final_learning_rate)
        self.readapt_iterations = int(readapt_iterations)
        self.fallback_accept = float(fallback_accept)
        self.fallback_window = int(fallback_window)
        self.error_check_every = int(error_check_every)
        self.seed = int(seed)
        self.surrogate = surrogate
        self.do_train = bool(train)
        self.report = SurrogateReport()
        self.pairs_theta = None
        self.pairs_grad = None
        self.filled = 0
        self.record_from = None
        self.active = False
        self.fallen_back = False
        self.recent_accept = []
        self.max_steps = 1000
        self.max_relative_error = float(max_relative_error)

    # ---- warmup ----
    def setup(self, run, num_warmup):
        torch = run.torch
        if self.surrogate is None:
            self.surrogate = GradientSurrogate(run.P, seed=self.seed)
        elif self.surrogate.P != run.P:
            raise IndexError(f"surrogate has {self.surrogate.P} parameters, the model {run.P}")
        if self.do_train:
            iters = max(1, min(math.ceil(0.6 * num_warmup), math.ceil(self.num_pairs / run.C)))
            self.num_pairs = min(self.num_pairs, iters * run.C)
            self.record_from = num_warmup - iters + 1
            self.pairs_theta = torch.empty((self.num_pairs, run.P), dtype=torch.float32, device=run.device)
            self.pairs_grad = torch.empty_like(self.pairs_theta)

    def after_warmup_iteration(self, run, it):
        if self.pairs_theta is None or it < self.record_from or self.filled >= self.num_pairs:
            return
        take = min(run.C, self.num_pairs - self.filled)
        self.pairs_theta[self.filled:self.filled + take].copy_(run.position[:take])
        self.pairs_grad[self.filled:self.filled + take].copy_(run.gradient[:take])
        self.filled += take

    def end_warmup(self, run, driver, traj, jitter_fn, steps_fn, thr, first_iteration):
        """Train, then re-tune the step size on surrogate trajectories; returns
        the number of iterations (Philox coordinates) it used."""
        torch = run.torch
        rep = self.report
        if self.do_train and self.filled > 1:
            theta = self.pairs_theta[:self.filled]
            grad = self.pairs_grad[:self.filled]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            self.surrogate.fit_normalization(theta, grad)
            steps = max(self.min_train_steps, int(round(self.train_epochs * self.filled / self.batch)))
            losses = self.surrogate.train(theta, grad, steps=steps, batch=self.batch,
                                          learning_rate=self.learning_rate,
                                          final_learning_rate=self.final_learning_rate, seed=self.seed)
            torch.cuda.synchronize()
            rep.train_seconds = time.perf_counter() - t0
            rep.num_pairs = self.filled
            rep.train_steps = steps
            rep.final_loss = float(losses[-min(steps, 32):].mean())
            self.pairs_theta = self.pairs_grad = None  # release the pair buffer
        rep.relative_error_after_training = self.surrogate.relative_error(run.position, run.gradient)
        self.max_steps = int(traj.max_leapfrog_steps)
        if not rep.relative_error_after_training < self.max_relative_error:
            self._fall_back(run, "training")  # too inaccurate to drive trajectories
            return 0
        self.active = True
        # step-size re-tuning on surrogate dynamics (trajectory length fixed);
        # given up (exact gradients from then on) when the surrogate's accept
        # rate stays below fallback_accept or the step collapses
        from .inference import DualAveraging, _chees_harmonic_mean_accept
        dual = DualAveraging(driver.step_size, driver.target_accept)
        eps0 = eps = driver.step_size
        accepts = []
        for k in range(self.readapt_iterations):
            it = first_iteration + k
            run.set_mass_and_step(driver.inverse_mass_matrix, eps)
            L = self.cap_steps(steps_fn(jitter_fn(it), traj.trajectory_length, eps))
            self._surrogate_iteration(run, L, it, thr)
            ap = run.accept_prob.double().cpu().numpy()
            div = run.divergent.cpu().numpy().astype(bool)
            accepts.append(float(ap.mean()))
            eps = float(dual.update(_chees_harmonic_mean_accept(ap, div)))
            window = accepts[-self.fallback_window:]
            if (len(window) == self.fallback_window and np.mean(window) < self.fallback_accept) or eps < eps0 / 64:
                self._fall_back(run, "readapt")
                return k + 1
        if self.readapt_iterations > 0:
            driver.step_size = float(dual.final())
        rep.readapted_step_size = driver.step_size
        return self.readapt_iterations

    def cap_steps(self, L: int) -> int:
        """Leapfrog steps of a surrogate trajectory, at most max_leapfrog_steps."""
        return int(min(L, self.max_steps)) if self.active and not self.fallen_back else int(L)

    def _fall_back(self, run, where):
        self.fallen_back = True
        self.report.fallback_at = where
        # exact state for the exact iterations that follow
        run.ws.logjoint_gradient_device(run.position, run.logjoint, run.gradient)

    # ---- iterations ----
    def _surrogate_iteration(self, run, L, it, thr, proposal=None, momentum=None):
        buf = run.hmc_buffers(proposal, momentum)
        nat.check(run.lib.ut_surrogate_hmc_iteration(run.ws.handle, self.surrogate.handle, ctypes.byref(buf),
                                                     int(L), run.coord(it), float(thr), _stream_handle()))

    def iteration(self, run, L, it, thr, warm, proposal=None, momentum=None):
        """One iteration; returns the exact gradient evaluations it cost
        (a logjoint-only evaluation counts as one)."""
        if warm or not self.active or self.fallen_back:
            run.hmc_iteration(L, it, thr, proposal, momentum)
            if not warm:
                self.report.exact_iterations_after_warmup += 1
            return L * run.C
        self._surrogate_iteration(run, L, it, thr, proposal, momentum)
        self.report.surrogate_iterations += 1
        cost = run.C
        self.recent_accept.append(float(run.accept_prob.mean()))
        if len(self.recent_accept) > self.fallback_window:
            self.recent_accept.pop(0)
        if self.error_check_every > 0 and self.report.surrogate_iterations % self.error_check_every == 0:
            run.ws.logjoint_gradient_device(run.position, run.logjoint, run.gradient)
            self.report.relative_error_checks.append(self.surrogate.relative_error(run.position, run.gradient))
            cost += run.C
        if (len(self.recent_accept) == self.fallback_window
                and float(np.mean(self.recent_accept)) < self.fallback_accept):
            self._fall_back(run, it)
            cost += run.C
        return cost

    def finish(self, run):
        if self.active and not self.fallen_back:
            # leave the exact gradient at the final positions in the state
            run.ws.logjoint_gradient_device(run.position, run.logjoint, run.gradient)


def batched_chees_surrogate(model, args=(), constraints=None, *, num_chains, num_samples, num_warmup=500,
                            num_pairs=2 ** 20, train_epochs=8, min_train_steps=10000, train_batch=4096,
                            learning_rate=2e-3,
                            final_learning_rate=1e-5, readapt_iterations=100, fallback_accept=0.2,
                            fallback_window=20, error_check_every=0, max_relative_error=0.5, surrogate=None,
                            surrogate_seed=0, **kwargs):
    """batched_chees whose sampling trajectories are driven by a learned
    gradient surrogate (exact logjoint in the accept).  Extra keyword
    arguments are those of batched_chees.  The returned chains carry a
    ``surrogate`` report (pairs, training time and loss, relative error,
    fallback)."""
    from .inference import batched_chees
    if num_warmup < 1 and surrogate is None:
        raise ValueError("the surrogate is trained on warmup pairs: num_warmup must be >= 1 "
                         "(or pass a trained surrogate)")
    ctl = SurrogateChEESController(num_pairs=num_pairs, train_epochs=train_epochs,
                                   min_train_steps=min_train_steps, batch=train_batch,
                                   learning_rate=learning_rate, final_learning_rate=final_learning_rate,
                                   readapt_iterations=readapt_iterations, fallback_accept=fallback_accept,
                                   fallback_window=fallback_window, error_check_every=error_check_every,
                                   seed=surrogate_seed, surrogate=surrogate, train=surrogate is None,
                                   max_relative_error=max_relative_error)
    chains = batched_chees(model, args, constraints, num_chains=num_chains, num_samples=num_samples,
                           num_warmup=num_warmup, _surrogate=ctl, **kwargs)
    chains.surrogate = ctl.report
    return chains
