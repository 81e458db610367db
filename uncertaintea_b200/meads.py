"""MEADS on the device: a tuning-free generalized-HMC ensemble sampler.

``batched_meads`` mirrors the reference's ``batched_meads``
(src/inference/api_batched_meads.jl:170-547; Hoffman & Sountsov, AISTATS 2022),
which runs on the host only.  Here every piece of an iteration runs on the
device (``ut_meads_iteration``): the per-fold ensemble statistics of the
neighbour fold (mean, std, trace-ratio eigenvalue estimates of the whitened
states and gradients), the step size, damping and slice drift, the partial
momentum refresh, one leapfrog step through the workspace's batched gradient
and the persistent-slice accept.  The host only launches and records draws.
There is no warmup adaptation phase; ``num_warmup`` draws are discarded.
Differences: the momentum refresh noise and the initial momentum / slice come
from the device Philox stream (streams 0 and 4), not the host RNG; the
returned inverse mass is the variance of the final ensemble (the reference
returns each chain's fold variance).
"""
from __future__ import annotations

import time

from . import _native as nat
from .device import _stream_handle
from .inference import _DeviceRun, _DrawBuffer, _finish, _invoke_callback


def batched_meads(model, args=(), constraints=None, *, num_chains, num_samples, num_warmup=0, num_folds=4,
                  initial_params=None, init_strategy="prior", init_max_retries=100, divergence_threshold=1000.0,
                  callback=None, callback_every=10, backend="cuda", precision=None, rng=None, _adapt_trace=None):
    """MEADS draws for ``num_chains`` chains (api_batched_meads.jl:170)."""
    if init_strategy not in ("prior", "uniform"):
        raise ValueError(f"batched_meads init_strategy must be :prior or :uniform, got {init_strategy!r}")
    if init_max_retries < 0:
        raise ValueError(f"batched_meads init_max_retries must be >= 0, got {init_max_retries}")
    if num_folds < 2:
        raise ValueError(f"batched_meads num_folds must be >= 2, got {num_folds}")
    if num_chains < 2 * num_folds:
        raise ValueError("batched_meads needs num_chains >= 2 * num_folds (each fold's ensemble statistics need "
                         f">= 2 members); got num_chains={num_chains}, num_folds={num_folds}")
    if num_samples <= 0:
        raise ValueError(f"batched_meads num_samples must be > 0, got {num_samples}")
    if num_warmup < 0:
        raise ValueError(f"batched_meads num_warmup must be >= 0, got {num_warmup}")
    run = _DeviceRun(model, args, constraints, num_chains, backend, precision, rng, initial_params, init_strategy,
                     init_max_retries, "batched MEADS")
    torch = run.torch
    C, K = run.C, int(num_folds)
    momentum = torch.empty_like(run.position)
    slice_u = torch.empty(C, dtype=torch.float32, device=run.device)
    steps = torch.zeros(C, dtype=torch.int32, device=run.device)
    fold = torch.zeros((K, 4), dtype=torch.float32, device=run.device)
    buf = nat.MeadsBuffers(*[nat.ptr(t) for t in (run.position, run.gradient, run.logjoint, momentum, slice_u,
                                                   run.accept_prob, run.energy, run.energy_error, run.accepted,
                                                   run.divergent, steps, fold)])
    lib = run.lib
    nat.check(lib.ut_meads_init(run.ws.handle, buf, run.coord(0), _stream_handle()))
    draws = _DrawBuffer(run, num_samples)
    total = num_warmup + num_samples
    divergences = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_sample = t0 if num_warmup == 0 else None
    for it in range(1, total + 1):
        if it == num_warmup + 1 and t_sample is None:
            torch.cuda.synchronize()
            t_sample = time.perf_counter()
        nat.check(lib.ut_meads_iteration(run.ws.handle, buf, K, it, float(divergence_threshold), run.coord(it),
                                         _stream_handle()))
        if _adapt_trace is not None:
            fp = fold.cpu().numpy()
            _adapt_trace.append({"step": float(fp[:, 0].mean()), "damping": float(fp[:, 1].mean())})
        if callback is not None:
            divergences += int(run.divergent.sum().item())
        if it <= num_warmup:
            _invoke_callback(callback, callback_every, "warmup", it, num_warmup, float("nan"), divergences)
            continue
        s = it - num_warmup - 1
        draws.record(s, integration_steps=0)
        draws.ist[s].copy_(steps)
        _invoke_callback(callback, callback_every, "sample", s + 1, num_samples, float("nan"), divergences)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    fp = fold.cpu().numpy()
    inverse_mass = run.position.double().var(dim=0).cpu().numpy()
    grad_evals = int(draws.ist.sum().item())
    out = _finish("meads", run, draws, float(fp[:, 0].mean()), inverse_mass, [], t_sample - t0, t1 - t_sample,
                  grad_evals=grad_evals)
    run.ws.close()
    return out
