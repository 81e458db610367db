"""Uneven batching (no counterpart in the reference): many independent
non-centred hierarchical normal models, each with its own groups, group
sizes, priors and chain count, sampled together by batched persistent NUTS on
one GPU.

Per iteration the library launches one persistent-NUTS kernel per
parameter-slot class (the classes run concurrently), then the warmup
adaptation of the reference's default batched NUTS (a dual-averaged step per
chain after a reasonable-step search, a pooled windowed diagonal mass per
model) or draw recording, all on the device, replayed from a captured CUDA
graph.  Chains per CTA and shared-memory staging of each
class's model data come from the library's autotuner, which times every
candidate on the same iteration.  The host only checks convergence at
checkpoints: per-model split R-hat on the device, from which the time each
model needs to reach R-hat < 1.01 is read.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .device import _stream_handle
from .inference import _warmup_schedule

NUM_CLASSES = 8
ACT_WELFORD, ACT_WINDOW_END, ACT_FINAL = 1, 2, 4


def _torch():
    import torch
    return torch


class _CudaArray:
    """A raw device buffer described by __cuda_array_interface__ (for a
    zero-copy torch view; valid while the batch owns the buffer)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(int(s) for s in shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 2, "strides": None}


def _device_view(ptr, shape, typestr):
    torch = _torch()
    if not ptr:
        raise RuntimeError("buffer not allocated")
    return torch.as_tensor(_CudaArray(ptr, shape, typestr), device="cuda")


def warmup_actions(num_warmup: int) -> np.ndarray:
    """Per warmup iteration (0-based) the adaptation actions of the windowed
    schedule (adaptation.jl:1-133, the same schedule the single-model samplers
    use): bit 0 = add the positions to the mass window, bit 1 = the window
    ends and sets the inverse mass, bit 2 = final step size."""
    acts = np.zeros(max(num_warmup, 0), dtype=np.uint8)
    if num_warmup <= 0:
        return acts
    s = _warmup_schedule(num_warmup)
    ends = list(s.slow_window_ends)
    for i in range(1, num_warmup + 1):
        a = 0
        if ends and s.initial_buffer < i <= ends[-1]:
            a |= ACT_WELFORD
        if i in ends:
            a |= ACT_WINDOW_END
        if i == num_warmup:
            a |= ACT_FINAL
        acts[i - 1] = a
    return acts


def split_ess(draws):
    """Bulk split ESS per parameter of draws (S, C, P) -- a torch tensor on any
    device -- with the reference's estimator (diagnostics.jl:550-583: chains
    split in halves, FFT autocovariances, Geyer's paired sums truncated at the
    first non-positive pair and made monotone), vectorised over parameters."""
    torch = _torch()
    x = draws.double()
    S, C, P = x.shape
    h = S // 2
    if h < 2:
        return torch.full((P,), float("nan"), dtype=torch.float64, device=x.device)
    split = torch.cat([x[:h], x[h:2 * h]], dim=1).permute(1, 0, 2)  # (2C, h, P)
    M = 2 * C
    means = split.mean(dim=1)
    W = split.var(dim=1, unbiased=True).mean(dim=0)
    B = h * means.var(dim=0, unbiased=True) if M > 1 else torch.zeros_like(W)
    var_plus = (h - 1) / h * W + B / h
    total = float(M * h)
    xc = split - means[:, None, :]
    n = 1 << int(math.ceil(math.log2(2 * h)))
    f = torch.fft.rfft(xc, n=n, dim=1)
    acov = torch.fft.irfft(f * f.conj(), n=n, dim=1)[:, :h] / h
    mean_acov = acov.mean(dim=0)  # (h, P)
    rho = 1.0 - (W[None, :] - mean_acov) / var_plus[None, :]
    rho[0] = 1.0
    rho = torch.clamp(rho, max=1.0)
    if h % 2:
        rho = torch.cat([rho, torch.zeros_like(rho[:1])], dim=0)
    pairs = rho[0::2] + rho[1::2]
    valid = torch.cumprod((pairs > 0).to(torch.int8), dim=0).bool()
    mono = torch.cummin(torch.where(valid, pairs, torch.full_like(pairs, float("inf"))), dim=0).values
    tau = torch.clamp(-1.0 + 2.0 * torch.where(valid, mono, torch.zeros_like(mono)).sum(dim=0), min=1.0)
    ess = torch.clamp(total / tau, max=total)
    ess = torch.where(var_plus <= 0, torch.zeros_like(ess), ess)
    return torch.where((W == 0) & (var_plus == 0), torch.full_like(ess, float("nan")), ess)


def _split_rhat_cols(split):
    """Split R-hat per column of (M, h, P) split chains (diagnostics.jl:514-540)."""
    torch = _torch()
    M, h, _ = split.shape
    means = split.mean(dim=1)
    W = split.var(dim=1, unbiased=True).mean(dim=0)
    B = h * means.var(dim=0, unbiased=True)
    var_plus = (h - 1) / h * W + B / h
    r = torch.sqrt(torch.clamp(var_plus / W, min=1.0))
    r = torch.where(W == 0, torch.where(var_plus == 0, torch.full_like(r, float("nan")),
                                        torch.full_like(r, float("inf"))), r)
    return r


def _rank_normal_cols(split):
    """Rank-normalise every column of (M, h, P) over its M*h values:
    (rank - 3/8) / (n + 1/4) through the normal quantile, ranks 1..n with ties
    in the reference's order, a stable sort over draw-major, split-chain-minor
    values (diagnostics.jl:589-600 on the column-major (2C, S/2) matrix)."""
    torch = _torch()
    M, h, P = split.shape
    flat = split.permute(1, 0, 2).reshape(h * M, P)
    n = M * h
    order = torch.argsort(flat, dim=0, stable=True)
    ranks = torch.empty_like(flat)
    ranks.scatter_(0, order, torch.arange(1, n + 1, dtype=flat.dtype, device=flat.device)[:, None].expand(n, P))
    z = torch.special.ndtri((ranks - 0.375) / (n + 0.25))
    return z.reshape(h, M, P).permute(1, 0, 2)


def split_rhat(draws):
    """Plain split R-hat per parameter of draws (S, C, P) -- a torch tensor on
    any device (diagnostics.jl:514-540 on each parameter's split chains)."""
    torch = _torch()
    x = draws.double()
    S, C, P = x.shape
    h = S // 2
    if h < 2:
        return torch.full((P,), float("nan"), dtype=torch.float64, device=x.device)
    split = torch.stack([x[:h], x[h:2 * h]], dim=2).reshape(h, 2 * C, P).permute(1, 0, 2)
    return _split_rhat_cols(split)


def rank_split_rhat(draws):
    """Rank-normalised split R-hat per parameter of draws (S, C, P) -- a torch
    tensor on any device: max of the bulk R-hat of the rank-normalised split
    chains and the tail R-hat of the rank-normalised |x - median|
    (diagnostics.jl:602-612, the sampler gate's estimator)."""
    torch = _torch()
    x = draws.double()
    S, C, P = x.shape
    h = S // 2
    if h < 2:
        return torch.full((P,), float("nan"), dtype=torch.float64, device=x.device)
    # (2C, h, P): chain c's first half is split chain 2c, its second half 2c + 1
    split = torch.stack([x[:h], x[h:2 * h]], dim=2).reshape(h, 2 * C, P).permute(1, 0, 2)
    bulk = _split_rhat_cols(_rank_normal_cols(split))
    srt = torch.sort(split.reshape(-1, P), dim=0).values
    n = srt.shape[0]
    med = 0.5 * (srt[(n - 1) // 2] + srt[n // 2])  # the 0.5 quantile with linear interpolation
    tail = _split_rhat_cols(_rank_normal_cols(torch.abs(split - med)))
    return torch.maximum(bulk, tail)


class MultiModelBatch:
    """A batch of (model, args, constraints) hierarchical models on the current
    CUDA device (library-owned state, see ut_multi_* in include/ut_b200.h)."""

    def __init__(self, models, chains, max_tree_depth: int = 10):
        self.lib = nat.load()
        self.models = list(models)
        M = len(self.models)
        if M < 1:
            raise ValueError("a batch needs at least one model")
        chains = np.broadcast_to(np.asarray(chains, dtype=np.int32), (M,)).copy()
        self.chains = chains
        lowered = [m.lower(a, c) for (m, a, c) in self.models]
        self.lowered = lowered
        self.P = np.array([lw.num_params for lw in lowered], dtype=np.int64)
        plans = (nat.PlanDesc * M)(*[lw.plan for lw in lowered])
        obs = np.ascontiguousarray(np.concatenate([lw.observed.reshape(-1) for lw in lowered]), dtype=np.float32)
        offs = np.zeros(M + 1, dtype=np.int64)
        offs[1:] = np.cumsum([lw.observed.size for lw in lowered])
        trips = np.ascontiguousarray(np.concatenate([lw.trip_counts for lw in lowered]), dtype=np.int32)
        starts = np.ascontiguousarray(np.concatenate([lw.loop_starts for lw in lowered]), dtype=np.int32)
        h = ctypes.c_void_p()
        nat.check(self.lib.ut_multi_create(M, plans, obs.ctypes.data, offs.ctypes.data, trips.ctypes.data,
                                           starts.ctypes.data, chains.ctypes.data, int(max_tree_depth),
                                           ctypes.byref(h)))
        self.handle = h
        self.M = M
        self.max_tree_depth = int(max_tree_depth)
        self.state_offsets = np.zeros(M + 1, dtype=np.int64)
        self.chain_offsets = np.zeros(M + 1, dtype=np.int64)
        self.param_offsets = np.zeros(M + 1, dtype=np.int64)
        nat.check(self.lib.ut_multi_layout(self.handle, self.state_offsets.ctypes.data,
                                           self.chain_offsets.ctypes.data, self.param_offsets.ctypes.data))

    # ---- configuration ----
    def class_info(self) -> dict:
        k = np.zeros(NUM_CLASSES, np.int32)
        nm = np.zeros(NUM_CLASSES, np.int32)
        nc = np.zeros(NUM_CLASSES, np.int64)
        w = np.zeros(NUM_CLASSES, np.int32)
        st = np.zeros(NUM_CLASSES, np.int32)
        nat.check(self.lib.ut_multi_class_info(self.handle, k.ctypes.data, nm.ctypes.data, nc.ctypes.data,
                                               w.ctypes.data, st.ctypes.data))
        return {"slots": k, "models": nm, "chains": nc, "chains_per_block": w, "stage_limit_bytes": st}

    def configure(self, klass: int, chains_per_block: int, stage_limit_bytes: int) -> None:
        nat.check(self.lib.ut_multi_configure(self.handle, int(klass), int(chains_per_block), int(stage_limit_bytes)))

    def autotune(self, trials: int = 2) -> np.ndarray:
        """Per class (8) x candidate ((chains per CTA 1, 2, 4) x (staging off, on))
        mean NUTS-launch milliseconds; the fastest candidate is kept."""
        out = np.zeros(NUM_CLASSES * 6, dtype=np.float32)
        nat.check(self.lib.ut_multi_autotune(self.handle, int(trials), out.ctypes.data, _stream_handle()))
        return out.reshape(NUM_CLASSES, 3, 2)

    # ---- state ----
    def set_positions(self, positions) -> None:
        torch = _torch()
        t = positions if torch.is_tensor(positions) else torch.from_numpy(np.ascontiguousarray(positions,
                                                                                                dtype=np.float32))
        t = t.to(device="cuda", dtype=torch.float32).contiguous().reshape(-1)
        if t.numel() != int(self.state_offsets[-1]):
            raise IndexError(f"expected {int(self.state_offsets[-1])} position values, got {t.numel()}")
        nat.check(self.lib.ut_multi_set_positions(self.handle, nat.ptr(t), _stream_handle()))
        _torch().cuda.current_stream().synchronize()

    def begin(self, num_warmup, num_samples, seed, target_accept=0.8, initial_step=0.1, divergence_threshold=1000.0,
              draws_capacity=None) -> None:
        acts = warmup_actions(num_warmup)
        cap = num_samples if draws_capacity is None else int(draws_capacity)
        nat.check(self.lib.ut_multi_begin(self.handle, int(num_warmup), int(num_samples), int(seed) & 0xFFFFFFFF,
                                          float(target_accept), float(initial_step), float(divergence_threshold),
                                          acts.ctypes.data if acts.size else None, cap))

    def run(self, num_iterations: int, use_graph: bool = True) -> None:
        nat.check(self.lib.ut_multi_run(self.handle, int(num_iterations), int(bool(use_graph)), _stream_handle()))

    def set_stopped(self, stopped) -> None:
        """Per-model stop flags (nonzero = the model's chains no longer move)."""
        flags = np.ascontiguousarray(np.asarray(stopped, dtype=np.uint8))
        nat.check(self.lib.ut_multi_set_stopped(self.handle, nat.ptr(flags), _stream_handle()))

    def split_rhat(self, num_draws: int) -> np.ndarray:
        torch = _torch()
        out = torch.empty(self.M, dtype=torch.float32, device="cuda")
        nat.check(self.lib.ut_multi_split_rhat(self.handle, int(num_draws), nat.ptr(out), _stream_handle()))
        return out.cpu().numpy()

    def view(self) -> dict:
        """Zero-copy torch views of the batch's device buffers (valid until the
        next begin / close)."""
        v = nat.MultiView()
        nat.check(self.lib.ut_multi_buffers(self.handle, ctypes.byref(v)))
        sf, tc, pf, cap = v.state_floats, v.total_chains, v.param_floats, v.draws_capacity
        out = {"position": _device_view(v.position, (sf,), "<f4"),
               "gradient": _device_view(v.gradient, (sf,), "<f4"),
               "logjoint": _device_view(v.logjoint, (tc,), "<f4"),
               "step": _device_view(v.step, (tc,), "<f4"),
               "inverse_mass": _device_view(v.inverse_mass, (pf,), "<f4"),
               "accept_prob": _device_view(v.accept_prob, (tc,), "<f4"),
               "tree_depth": _device_view(v.tree_depth, (tc,), "<i4"),
               "integration_steps": _device_view(v.integration_steps, (tc,), "<i4"),
               "divergent": _device_view(v.divergent, (tc,), "|u1"),
               "iteration": _device_view(v.iteration, (1,), "<i4")}
        if cap > 0:
            out["draws"] = _device_view(v.draws, (cap, sf), "<f4")
            out["draw_accept"] = _device_view(v.draw_accept, (cap, tc), "<f4")
            out["draw_tree_depth"] = _device_view(v.draw_tree_depth, (cap, tc), "<i4")
            out["draw_divergent"] = _device_view(v.draw_divergent, (cap, tc), "|u1")
        return out

    def model_draws(self, m: int, num_draws=None):
        """Model m's recorded draws as a device tensor (S, C_m, P_m) (a view)."""
        d = self.view()["draws"]
        S = d.shape[0] if num_draws is None else int(num_draws)
        a, b = int(self.state_offsets[m]), int(self.state_offsets[m + 1])
        return d[:S, a:b].reshape(S, int(self.chains[m]), int(self.P[m]))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            nat.check(self.lib.ut_multi_destroy(self.handle))
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class MultiChains:
    """Result of batched_nuts_multi: per-model arrays (length num_models) and
    the batch's aggregate figures."""
    batch: MultiModelBatch
    num_params: np.ndarray
    num_chains: np.ndarray
    min_ess: np.ndarray
    max_rhat: np.ndarray
    time_to_rhat: np.ndarray          # seconds from the start of the run (warmup included); inf if never
    sampling_time_to_rhat: np.ndarray  # seconds from the start of sampling
    warmup_seconds: float
    sampling_seconds: float            # device time of the sampling iterations (checkpoints excluded)
    autotune_ms: np.ndarray | None = None
    draws_per_model: np.ndarray | None = None  # the draws that are each model's own (per-model stopping)
    classes: dict = field(default_factory=dict)
    divergences: int = 0
    mean_tree_depth: float = float("nan")

    @property
    def aggregate_ess_per_second(self) -> float:
        return float(np.nansum(self.min_ess) / self.sampling_seconds)

    def time_to_rhat_quantiles(self, qs=(0.5, 0.99), from_sampling=False) -> list:
        """Quantiles over models of the time to R-hat < target (an observed
        value, no interpolation; inf when that share of models never got there)."""
        t = self.sampling_time_to_rhat if from_sampling else self.time_to_rhat
        return [float(np.quantile(t, q, method="inverted_cdf")) for q in qs]

    @property
    def converged_fraction(self) -> float:
        return float(np.mean(np.isfinite(self.time_to_rhat)))

    def draws(self, m: int) -> np.ndarray:
        """Model m's draws on the host as (C, S, P) (the single-model samplers' layout)."""
        return self.batch.model_draws(m).permute(1, 0, 2).cpu().numpy()


def batched_nuts_multi(models, *, chains_per_model=64, num_warmup=1000, num_samples=1000, max_tree_depth=10,
                       target_accept=0.8, initial_step_size=0.1, divergence_threshold=1000.0, rng=None,
                       init_strategy="prior", autotune=True, autotune_after=None, autotune_trials=2,
                       rhat_check_every=50, rhat_target=1.01, use_graph=True, callback=None,
                       stop_converged=False) -> MultiChains:
    """Batched persistent NUTS over many hierarchical models at once.

    models: list of (HierarchicalNormalNoncentered, args, constraints).  Warmup
    adapts every model's step size and diagonal mass on the device; the
    autotuner runs after ``autotune_after`` warmup iterations (default: a
    fifth of the warmup), when the trees look like the stationary ones.
    Every ``rhat_check_every`` sampling iterations the per-model split R-hat of
    the draws so far is computed on the device; a model below ``rhat_target``
    there is confirmed with the rank-normalised split R-hat (the gate's
    estimator), and its time-to-R-hat is the first checkpoint where that max
    over its parameters is below the target.  Reported R-hats are rank-normalised.

    stop_converged: a model that reaches the target stops there (its chains no
    longer move, ut_multi_set_stopped) and the run continues for the others up
    to ``num_samples`` draws (the cap), or until every model has stopped; each
    model's R-hat and ESS are then over its own draws."""
    torch = _torch()
    if num_warmup < 0 or num_samples < 4:
        raise ValueError("need num_warmup >= 0 and num_samples >= 4")
    if rhat_check_every < 1:
        raise ValueError("rhat_check_every must be >= 1")
    rng = rng if isinstance(rng, np.random.Generator) else np.random.default_rng(rng)
    batch = MultiModelBatch(models, chains_per_model, max_tree_depth)
    M = batch.M
    init = np.empty(int(batch.state_offsets[-1]), dtype=np.float32)
    for m, (model, args, cons) in enumerate(batch.models):
        q = model.initial_positions(rng, int(batch.chains[m]), args, cons, init_strategy)
        init[batch.state_offsets[m]:batch.state_offsets[m + 1]] = np.asarray(q, dtype=np.float32).reshape(-1)
    batch.set_positions(init)
    seed = int(rng.integers(0, 2 ** 32))
    batch.begin(num_warmup, num_samples, seed, target_accept, initial_step_size, divergence_threshold)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    timings = None
    done = 0
    if autotune and num_warmup > 0:
        first = max(1, num_warmup // 5) if autotune_after is None else int(autotune_after)
        first = min(first, num_warmup)
        batch.run(first, use_graph)
        done = first
        timings = batch.autotune(autotune_trials)
    batch.run(num_warmup - done, use_graph)
    torch.cuda.synchronize()
    t_warm = time.perf_counter() - t0
    if autotune and num_warmup == 0:
        timings = batch.autotune(autotune_trials)
    ttr = np.full(M, np.inf)
    sttr = np.full(M, np.inf)
    stopped = np.zeros(M, dtype=np.uint8)
    own = np.full(M, num_samples, dtype=np.int64)   # draws that are the model's own
    samp_ms = 0.0
    t_samp0 = time.perf_counter()
    s = 0
    while s < num_samples:
        k = min(rhat_check_every, num_samples - s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.run(k, use_graph)
        e1.record(stream)
        s += k
        if s >= 4:
            r = batch.split_rhat(s)  # synchronises
            hit = (r < rhat_target) & ~np.isfinite(sttr) & (stopped == 0)
            for m in np.flatnonzero(hit):  # confirm with the gate's rank-normalised R-hat
                hit[m] = float(torch.nan_to_num(rank_split_rhat(batch.model_draws(int(m), s)),
                                                nan=float("inf")).max()) < rhat_target
            now = time.perf_counter()
            sttr[hit] = now - t_samp0
            ttr[hit] = now - t0
            if stop_converged and hit.any():
                stopped[hit] = 1
                own[hit] = s
                batch.set_stopped(stopped)
        torch.cuda.synchronize()
        samp_ms += e0.elapsed_time(e1)
        if callback is not None:
            callback("sample", s, num_samples)
        if stop_converged and stopped.all():
            break
    own = np.minimum(own, s)
    final_rhat = np.empty(M)  # rank-normalised, each model over its own draws
    ess = np.empty(M)
    for m in range(M):
        d = batch.model_draws(m, int(own[m]))
        final_rhat[m] = float(torch.nan_to_num(rank_split_rhat(d), nan=float("inf")).max())
        ess[m] = float(torch.nan_to_num(split_ess(d), nan=float("inf")).min())
    v = batch.view()
    div, depth_sum, depth_n = 0, 0.0, 0
    for m in range(M):  # each model's own draws (a stopped model's later rows repeat its last state)
        a, b = int(batch.chain_offsets[m]), int(batch.chain_offsets[m + 1])
        n = int(own[m])
        div += int(v["draw_divergent"][:n, a:b].sum())
        depth_sum += float(v["draw_tree_depth"][:n, a:b].double().sum())
        depth_n += n * (b - a)
    return MultiChains(batch=batch, num_params=batch.P.copy(), num_chains=batch.chains.copy(), min_ess=ess,
                       max_rhat=final_rhat, time_to_rhat=ttr, sampling_time_to_rhat=sttr, warmup_seconds=t_warm,
                       sampling_seconds=samp_ms / 1000.0, autotune_ms=timings, classes=batch.class_info(),
                       divergences=div, mean_tree_depth=depth_sum / max(depth_n, 1), draws_per_model=own)
