"""``UncertainTea.Diagnostics`` mirror: split R-hat, rank-normalised R-hat and
bulk ESS (src/inference/diagnostics.jl:461-650), plus the min-ESS/s metric
(docs/benchmarks.md:57, sampling time only).

Autocovariances are computed with an FFT; they are the same biased estimates
(sum over the overlap divided by S) as the reference's direct sums
(diagnostics.jl:541-548), so the truncated paired estimator is unchanged.
"""
from __future__ import annotations

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
    """diagnostics.jl:589-600: (r - 3/8) / (S + 1/4) through the normal quantile."""
    flat = draws.reshape(-1)
    S = flat.size
    order = np.argsort(flat, kind="stable")
    ranks = np.empty(S, dtype=np.float64)
    ranks[order] = np.arange(1, S + 1)
    return ndtri((ranks - 0.375) / (S + 0.25)).reshape(draws.shape)


def _draws(chains, space):
    arr = chains.constrained if space == "constrained" else chains.unconstrained
    return np.asarray(arr)


def rhat(chains, space: str = "constrained", method: str = "split") -> np.ndarray:
    if method not in ("split", "rank"):
        raise ValueError(f"rhat method must be :split or :rank, got {method!r}")
    d = _draws(chains, space)
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
    d = _draws(chains, space)
    out = np.empty(d.shape[2])
    for p in range(d.shape[2]):
        out[p] = _split_ess_of(_split_chain_draws(d[:, :, p].astype(np.float64)))
    return out


def min_ess_per_second(chains, space: str = "constrained") -> float:
    """min over parameters of bulk ESS / sampling seconds (warmup excluded)."""
    return float(np.nanmin(ess(chains, space)) / max(chains.sampling_seconds, 1e-12))


def summarize(chains, space: str = "constrained", quantiles=(0.05, 0.5, 0.95)):
    d = _draws(chains, space)
    names = chains.parameter_names() if hasattr(chains, "parameter_names") else [str(i) for i in range(d.shape[2])]
    rh, es = rhat(chains, space), ess(chains, space)
    rows = []
    for p in range(d.shape[2]):
        flat = d[:, :, p].reshape(-1).astype(np.float64)
        rows.append({"parameter": names[p], "mean": float(flat.mean()), "sd": float(flat.std(ddof=1)),
                     "quantiles": [float(np.quantile(flat, q)) for q in quantiles], "rhat": float(rh[p]),
                     "ess": float(es[p])})
    return {"parameters": rows, "acceptance_rate": float(np.mean(chains.accept_prob)),
            "divergence_rate": float(np.mean(chains.divergent))}
