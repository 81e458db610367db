"""``UncertainTea.Diagnostics`` mirror: split R-hat, rank-normalised R-hat and
bulk ESS (src/inference/diagnostics.jl:461-650), plus the min-ESS/s metric
(docs/benchmarks.md:57, sampling time only).

Autocovariances are computed with an FFT; they are the same biased estimates
(sum over the overlap divided by S) as the reference's direct sums
(diagnostics.jl:541-548), so the truncated paired estimator is unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.special import ndtri

try:  # multi-threaded FFTs when scipy provides them
    import scipy.fft as _fft
    _FFT_KW = {"workers": -1}
except ImportError:  # pragma: no cover
    _fft = np.fft
    _FFT_KW = {}


def _split_chain_draws(draws: np.ndarray) -> np.ndarray:
    """(C, S) -> (2C, S//2): first and second half of every chain (diagnostics.jl:500-511)."""
    C, S = draws.shape
    h = S // 2
    out = np.empty((2 * C, h), dtype=np.float64)
    out[0::2] = draws[:, :h]
    out[1::2] = draws[:, h:2 * h]
    return out


def _chain_stats(draws: np.ndarray):
    """diagnostics.jl:514-527."""
    M, S = draws.shape
    means = draws.mean(axis=1)
    variances = draws.var(axis=1, ddof=1) if S > 1 else np.zeros(M)
    W = variances.mean()
    B = S * means.var(ddof=1) if (S > 1 and M > 1) else 0.0
    var_plus = ((S - 1) / S) * W + B / S
    return means, variances, W, B, var_plus


def _split_rhat_of(split: np.ndarray) -> float:
    _, _, W, _, var_plus = _chain_stats(split)
    if W == 0:
        return float("nan") if var_plus == 0 else float("inf")
    return float(np.sqrt(max(var_plus / W, 1.0)))


def _split_ess_of(split: np.ndarray) -> float:
    """diagnostics.jl:550-583 (paired, monotone-truncated autocorrelation sum)."""
    M, S = split.shape
    means, _, W, _, var_plus = _chain_stats(split)
    total = M * S
    if W == 0 and var_plus == 0:
        return float("nan")
    if var_plus <= 0:
        return 0.0
    x = split - means[:, None]
    n = 1 << int(np.ceil(np.log2(2 * S)))
    f = _fft.rfft(x, n=n, axis=1, **_FFT_KW)
    acov = _fft.irfft((f * np.conj(f)).real, n=n, axis=1, **_FFT_KW)[:, :S] / S
    mean_acov = acov.mean(axis=0)
    rho = 1.0 - (W - mean_acov) / var_plus
    rho[0] = 1.0
    rho = np.minimum(rho, 1.0)
    pair_sums = []
    for start in range(0, S, 2):
        s = rho[start] + (rho[start + 1] if start + 1 <= S - 1 else 0.0)
        if not s > 0:
            break
        pair_sums.append(s)
    ps = np.minimum.accumulate(np.asarray(pair_sums)) if pair_sums else np.zeros(0)
    tau = max(-1.0 + 2.0 * ps.sum(), 1.0)
    return float(min(total, total / tau))


def _rank_normal(draws: np.ndarray) -> np.ndarray:
    """diagnostics.jl:589-600: (r - 3/8) / (S + 1/4) through the normal quantile.
    Ties take ranks in the reference's order: a stable sort of the (2C, S/2)
    split matrix flattened column-major (draw-major, split chain minor)."""
    flat = draws.reshape(-1, order="F")
    S = flat.size
    order = np.argsort(flat, kind="stable")
    ranks = np.empty(S, dtype=np.float64)
    ranks[order] = np.arange(1, S + 1)
    return ndtri((ranks - 0.375) / (S + 0.25)).reshape(draws.shape, order="F")


def _draws(chains, space):
    """(C, S, P) draws of one space (diagnostics.jl:332-340)."""
    if space == "constrained":
        arr = chains.constrained
    elif space == "unconstrained":
        arr = chains.unconstrained
    else:
        raise ValueError("diagnostic space must be :constrained or :unconstrained")
    return np.asarray(arr)


def _validated_draws(chains, space):
    """diagnostics.jl:384-402: at least one chain and 4 draws per chain (one
    chain still gives two split halves)."""
    d = _draws(chains, space)
    if d.ndim != 3 or d.shape[0] < 1:
        raise ValueError("chain diagnostics require at least 1 chain")
    if d.shape[1] < 4:
        raise ValueError("chain diagnostics require at least 4 samples per chain")
    return d


def rhat(chains, space: str = "constrained", method: str = "split") -> np.ndarray:
    if method not in ("split", "rank"):
        raise ValueError(f"rhat method must be :split or :rank, got {method!r}")
    d = _validated_draws(chains, space)
    out = np.empty(d.shape[2])
    for p in range(d.shape[2]):
        split = _split_chain_draws(d[:, :, p].astype(np.float64))
        if method == "split":
            out[p] = _split_rhat_of(split)
        else:
            bulk = _split_rhat_of(_rank_normal(split))
            med = np.quantile(split.reshape(-1), 0.5)
            folded = _split_rhat_of(_rank_normal(np.abs(split - med)))
            out[p] = max(bulk, folded)
    return out


def ess(chains, space: str = "constrained") -> np.ndarray:
    d = _validated_draws(chains, space)
    out = np.empty(d.shape[2])
    for p in range(d.shape[2]):
        out[p] = _split_ess_of(_split_chain_draws(d[:, :, p].astype(np.float64)))
    return out


def min_ess_per_second(chains, space: str = "constrained") -> float:
    """min over parameters of bulk ESS / sampling seconds (warmup excluded)."""
    return float(np.nanmin(ess(chains, space)) / max(chains.sampling_seconds, 1e-12))


def _quantile_sorted(sorted_values: np.ndarray, probability: float) -> float:
    """diagnostics.jl:486-497: linear interpolation at position 1 + (n - 1) p."""
    n = sorted_values.size
    if n == 0:
        raise ValueError("quantile requires at least one value")
    if n == 1:
        return float(sorted_values[0])
    position = (n - 1) * probability
    lower, upper = int(np.floor(position)), int(np.ceil(position))
    if lower == upper:
        return float(sorted_values[lower])
    weight = position - lower
    return float((1 - weight) * sorted_values[lower] + weight * sorted_values[upper])


def _indicator_split_ess(split: np.ndarray, threshold: float) -> float:
    """Split ESS of I(x <= threshold); NaN when the indicator is constant
    (summaries.jl:16-21)."""
    indicator = split <= threshold
    if indicator.all() or not indicator.any():
        return float("nan")
    return _split_ess_of(indicator.astype(np.float64))


def _nan_min(a: float, b: float) -> float:
    """Julia's min: NaN when either argument is NaN."""
    return float("nan") if (np.isnan(a) or np.isnan(b)) else min(a, b)


EBFMI_WARNING_THRESHOLD = 0.3  # warnings.jl:27


@dataclass
class SamplerWarnings:
    """SamplerWarnings (data_types.jl:147): per-chain divergence counts, E-BFMI and
    treedepth-saturation counts, and the parameters with low ESS / high R-hat."""
    num_divergent: np.ndarray
    ebfmi: np.ndarray
    treedepth_hits: np.ndarray
    low_ess_parameters: list
    high_rhat_parameters: list
    ebfmi_threshold: float = EBFMI_WARNING_THRESHOLD


def _ebfmi(energies: np.ndarray) -> float:
    """warnings.jl:7-18: sum of squared successive energy differences / sum of
    squared deviations from the mean energy; NaN with fewer than 2 draws or
    constant energy."""
    e = np.asarray(energies, dtype=np.float64)
    if e.size < 2:
        return float("nan")
    den = float(np.sum((e - e.mean()) ** 2))
    if den == 0:
        return float("nan")
    return float(np.sum(np.diff(e) ** 2) / den)


def check_diagnostics(chains, space: str = "constrained", rhat_threshold: float = 1.01, ess_threshold: float = 100.0,
                      ebfmi_threshold: float = EBFMI_WARNING_THRESHOLD) -> SamplerWarnings:
    """``check_diagnostics(chains; space, rhat_threshold, ess_threshold,
    ebfmi_threshold)`` (warnings.jl:20-24, 38-77): divergences, E-BFMI and treedepth
    saturation per chain; parameters whose R-hat exceeds the threshold (or is not
    finite) and whose ESS is below the threshold (or not finite), checked when
    there are at least 4 draws per chain."""
    divergent = np.asarray(chains.divergent).astype(bool)
    energy = np.asarray(chains.energy, dtype=np.float64)
    num_divergent = divergent.sum(axis=1).astype(np.int64)
    ebfmi = np.array([_ebfmi(energy[c]) for c in range(energy.shape[0])])
    depth_limit = int(getattr(chains, "max_tree_depth", 0) or 0)
    if depth_limit > 0:
        treedepth_hits = (np.asarray(chains.tree_depth) == depth_limit).sum(axis=1).astype(np.int64)
    else:
        treedepth_hits = np.zeros(divergent.shape[0], dtype=np.int64)
    low_ess, high_rhat = [], []
    d = _draws(chains, space)
    if d.shape[0] >= 1 and d.shape[1] >= 4:
        rh, es = rhat(chains, space), ess(chains, space)
        names = chains.parameter_names() if hasattr(chains, "parameter_names") else [str(i) for i in range(d.shape[2])]
        for p, name in enumerate(names):
            if not np.isfinite(rh[p]) or rh[p] > rhat_threshold:
                high_rhat.append(name)
            if not np.isfinite(es[p]) or es[p] < ess_threshold:
                low_ess.append(name)
    return SamplerWarnings(num_divergent, ebfmi, treedepth_hits, low_ess, high_rhat, float(ebfmi_threshold))


def has_warnings(warnings: SamplerWarnings) -> bool:
    """warnings.jl:79-86."""
    return bool(np.any(warnings.num_divergent > 0)
                or np.any(np.isfinite(warnings.ebfmi) & (warnings.ebfmi < warnings.ebfmi_threshold))
                or np.any(warnings.treedepth_hits > 0) or warnings.low_ess_parameters
                or warnings.high_rhat_parameters)


class Summary(dict):
    """The result of ``summarize``: a dict (space, quantiles, diagnostics,
    parameters, warnings) whose text form is a per-parameter table followed by
    the run diagnostics and, when there are any, the sampler warnings."""

    def __str__(self):
        qs = self["quantiles"]
        head = ["parameter", "mean", "sd", "mcse"] + [f"q{100 * q:g}" for q in qs] + ["rhat", "ess_bulk", "ess_tail"]
        rows = []
        for p in self["parameters"]:
            rows.append([str(p["parameter"])] + [f"{v:.4g}" for v in (p["mean"], p["sd"], p["mcse_mean"])]
                        + [f"{v:.4g}" for v in p["quantiles"]]
                        + [f"{p['rhat']:.4f}", f"{p['ess_bulk']:.1f}", f"{p['ess_tail']:.1f}"])
        widths = [max(len(h), *(len(r[i]) for r in rows)) if rows else len(h) for i, h in enumerate(head)]
        fmt = lambda cells: "  ".join(c.rjust(w) for c, w in zip(cells, widths))  # noqa: E731
        d = self["diagnostics"]
        lines = [f"summary ({self['space']} space)", fmt(head)] + [fmt(r) for r in rows]
        lines.append(f"acceptance rate {d['acceptance_rate']:.4f}, divergence rate {d['divergence_rate']:.4f}, "
                     f"mean step size {d['mean_step_size']:.4g}")
        w = self.get("warnings")
        if w is not None and has_warnings(w):
            lines.append("warnings:")
            if int(np.sum(w.num_divergent)) > 0:
                lines.append(f"  divergences: {int(np.sum(w.num_divergent))} total {list(map(int, w.num_divergent))}")
            low = np.isfinite(w.ebfmi) & (w.ebfmi < w.ebfmi_threshold)
            if np.any(low):
                lines.append(f"  low E-BFMI (< {w.ebfmi_threshold}): {np.round(w.ebfmi, 3).tolist()}")
            if int(np.sum(w.treedepth_hits)) > 0:
                lines.append(f"  treedepth saturation: {int(np.sum(w.treedepth_hits))} total")
            if w.low_ess_parameters:
                lines.append(f"  low ESS parameters: {w.low_ess_parameters}")
            if w.high_rhat_parameters:
                lines.append(f"  high Rhat parameters: {w.high_rhat_parameters}")
        return "\n".join(lines)


def _mass_adaptation_diagnostics(windows, num_chains):
    """Per slow window, the reference's summary over chains (diagnostics.jl:411-448).
    The mass here is pooled, so every chain shares one record per window: chains
    = num_chains, updated chains = num_chains or 0, and min = mean = max."""
    out = []
    for w in windows or []:
        if "weight_sum" not in w:
            continue
        out.append({"window_index": w["window"], "iteration_start": w["start"], "iteration_end": w["end"],
                    "window_length": w["window_length"], "chains": num_chains,
                    "updated_chains": num_chains if w["updated"] else 0, "mean_pooled_samples": float(w["samples"]),
                    "mean_weight_sum": w["weight_sum"], "mean_effective_count": w["effective_count"],
                    "min_effective_count": w["effective_count"], "max_effective_count": w["effective_count"],
                    "mean_weight": w["mean_weight"], "mean_clip_scale_end": w["clip_scale_end"],
                    "mass_mean": w["mass_mean"], "mass_min": w["mass_min"], "mass_max": w["mass_max"]})
    return sorted(out, key=lambda r: (r["window_index"], r["iteration_start"], r["iteration_end"]))


def summarize(chains, space: str = "constrained", quantiles=(0.05, 0.5, 0.95), per_chain: bool = False):
    """``summarize(chains; space, quantiles, per_chain)`` (diagnostics.jl:662-712,
    summaries.jl:1-76): per parameter the pooled mean and sample SD, the requested
    quantiles, split R-hat, bulk ESS, the MCSE of the mean (sd / sqrt(ess)), the
    tail ESS (the smaller split ESS of the indicators at the pooled 5% / 95%
    quantiles), the MCSE of each quantile (half the spread of the order
    statistics at q -+ sqrt(q (1 - q) / ess_q)), and with per_chain the per-chain
    means and SDs; plus the run's acceptance and divergence rates and the
    per-chain step sizes."""
    quantiles = list(quantiles)
    if not quantiles:
        raise ValueError("summary quantiles must be non-empty")
    probs = [float(q) for q in quantiles]
    if not all(0.0 <= q <= 1.0 for q in probs):
        raise ValueError("summary quantiles must lie in [0, 1]")
    d = _validated_draws(chains, space)
    C, S, P = d.shape
    names = chains.parameter_names() if hasattr(chains, "parameter_names") else [str(i) for i in range(P)]
    rh, es = rhat(chains, space), ess(chains, space)
    rows = []
    for p in range(P):
        x = d[:, :, p].astype(np.float64)
        pooled = x.reshape(-1)                       # chain after chain (diagnostics.jl:474-484)
        sorted_draws = np.sort(pooled)
        mean = float(pooled.mean())
        sd = float(np.sqrt(max(pooled.var(ddof=1), 0.0))) if pooled.size > 1 else 0.0
        ess_bulk = float(es[p])
        qvals = [_quantile_sorted(sorted_draws, q) for q in probs]
        split = _split_chain_draws(x)
        mcse_mean = sd * np.sqrt(1.0 / ess_bulk) if (np.isfinite(ess_bulk) and ess_bulk > 0) else float("nan")
        q05, q95 = _quantile_sorted(sorted_draws, 0.05), _quantile_sorted(sorted_draws, 0.95)
        ess_tail = _nan_min(_indicator_split_ess(split, q05), _indicator_split_ess(split, q95))
        mcse_q = []
        for q, theta in zip(probs, qvals):
            ess_q = _indicator_split_ess(split, theta)
            if not (np.isfinite(ess_q) and ess_q > 0):
                mcse_q.append(float("nan"))
                continue
            spread = np.sqrt(q * (1 - q) / ess_q)
            lo = _quantile_sorted(sorted_draws, min(max(q - spread, 0.0), 1.0))
            hi = _quantile_sorted(sorted_draws, min(max(q + spread, 0.0), 1.0))
            mcse_q.append((hi - lo) / 2)
        row = {"index": p, "parameter": names[p], "mean": mean, "sd": sd, "quantiles": qvals,
               "rhat": float(rh[p]), "ess": ess_bulk, "ess_bulk": ess_bulk, "mcse_mean": float(mcse_mean),
               "ess_tail": ess_tail, "mcse_quantiles": mcse_q, "per_chain_means": None, "per_chain_sds": None}
        if per_chain:
            row["per_chain_means"] = x.mean(axis=1)
            row["per_chain_sds"] = x.std(axis=1, ddof=1) if S > 1 else np.zeros(C)
        rows.append(row)
    accept = np.asarray(chains.accept_prob, dtype=np.float64)
    divergent = np.asarray(chains.divergent)
    steps = np.broadcast_to(np.asarray(chains.step_size, dtype=np.float64), (C,)).copy()
    diagnostics = {"acceptance_rate": float(accept.mean()) if accept.size else 0.0,
                   "divergence_rate": float(np.count_nonzero(divergent) / divergent.size) if divergent.size else 0.0,
                   "step_sizes": steps, "mean_step_size": float(steps.mean()) if steps.size else 0.0,
                   "mass_adaptation": _mass_adaptation_diagnostics(getattr(chains, "mass_adaptation_windows", None),
                                                                   C)}
    return Summary(space=space, quantiles=probs, diagnostics=diagnostics, parameters=rows,
                   warnings=check_diagnostics(chains, space), acceptance_rate=diagnostics["acceptance_rate"],
                   divergence_rate=diagnostics["divergence_rate"])
