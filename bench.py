"""Benchmark of the batched density hot path on the B200.

Default workload (the headline): one batched logjoint + gradient evaluation
of the large dense logistic regression -- X is 100000 x 100 ~ N(0,1)/sqrt(100),
y ~ Bernoulli(logistic(X beta_true)), prior normal(0,1) -- over 4096 chains.
A step is one evaluation of all 4096 chains; the metric is chain-gradient
evaluations per second.  Data are seeded synthetic stand-ins (no data set is
shipped).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

At N=1 the line also carries `hbm_sweep`: the same design at 1, 4, 8 and 16
chains, where an evaluation is bound by reading X from HBM (achieved GB/s
against the measured HBM bandwidth), `samplers`: the 1000x10 GLM HMC, the
hierarchical (J=64) persistent-NUTS, and the 100000x100 GLM masked-NUTS and MEADS runs (min ESS/s, R-hat, gradient
evaluations/s; skipped with --no-samplers), `surrogate_chees`: the
learned-gradient-surrogate workload on the same model (min ESS/s of
surrogate-driven ChEES-HMC vs plain ChEES-HMC and vs the plain masked NUTS run,
all at R-hat < 1.01; skipped with --no-surrogate), and
`uneven_batch`: 512 hierarchical models of uneven sizes in one batched
persistent-NUTS run (aggregate ESS/s, per-model time to R-hat < 1.01;
skipped with --no-uneven).

Multi-GPU: the path does not shard (every chain's gradient needs all of X),
so N GPUs run N independent replicas (weak scaling) and `value` is the
aggregate over all ranks divided by the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_OBS, N_COEF, N_CHAINS = 100_000, 100, 4096
FLOP_FP32 = 4.0 * N_OBS * N_COEF * N_CHAINS            # two N x D x C contractions (x, +)
METRIC = "grad evals/s"
UNIT = "chain-gradient evaluations/s"
WORKLOAD = ("logistic regression: batched logjoint+gradient, N=100000 obs, D=100, "
            "4096 chains, FP32 (3xTF32 tensor-core contraction when available)")


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    def __init__(self, index=0):
        self.samples = []
        self.proc = None
        self.index = index

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _max_over_ranks(x, dist=None, device="cuda"):
    """Max of x over all ranks (the slowest replica's clock); x itself at N = 1."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _replica_value(units_per_rank, world, seconds_max):
    """Whole-job throughput of `world` independent replicas: all ranks' units over
    the max-over-ranks time."""
    return world * units_per_rank / seconds_max


def _data():
    from uncertaintea_b200.models import BernoulliLogitGLM, logistic_regression_data
    X, y, _ = logistic_regression_data(N_OBS, N_COEF, seed=3, x_scale=1.0 / np.sqrt(N_COEF))
    model = BernoulliLogitGLM(N_COEF, coef_mu=0.0, coef_sigma=1.0)
    params = np.random.default_rng(1).standard_normal((N_CHAINS, N_COEF)).astype(np.float32)
    return model, X, y, params


def cpu_reference_rate(model, X, y, params, budget_s=12.0, threads=0):
    """Chain-gradient evaluations/s of the CPU restatement of the reference's
    batched path (chain-parallel, all host threads), on a bounded sample."""
    import oracle
    om = oracle.OracleModel(model.lower((X,), {"y": y}))
    cores = oracle.max_threads() if threads == 0 else threads
    chunk = max(8, cores * 4)
    done, t0 = 0, time.perf_counter()
    while True:
        om.logjoint_gradient_f32(params[done % N_CHAINS: done % N_CHAINS + chunk], threads=threads)
        done += chunk
        el = time.perf_counter() - t0
        if el >= budget_s or done >= 64 * chunk:
            break
    return done / el, cores, f"{done} chain-gradients of the full N=100000 x D=100 model in {el:.1f} s"


def _emit(name, result, t0=None):
    """One sub-result of the run as its own JSON line (before the headline
    line), with the wall seconds the section took since t0."""
    if result is not None:
        took = {"section_s": round(time.perf_counter() - t0, 1)} if t0 is not None else {}
        print(json.dumps({"sub": name, **result, **took}), flush=True)


def _profiled_traffic():
    """DRAM bytes (read + write) of one tensor-core launch on this workload, from
    the committed ncu summary (its `traffic_bytes_per_launch:` line), or None."""
    path = os.path.join(ROOT, "profiles", "tc_glm_kernel_config3.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for ln in f:
            if ln.strip().startswith("traffic_bytes_per_launch:"):
                return float(ln.split(":", 1)[1].strip().split()[0])
    return None


# Gradient tolerance of the FP64 check, elementwise:
#   |g - g64| <= GRAD_RTOL * |g64| + GRAD_ATOL_MAG * m,
# m = the sum of the magnitudes of the terms g adds up (oracle gradient_magnitude).
GRAD_RTOL = 1e-5
GRAD_ATOL_MAG = 1e-6


def fp64_error(model, X, y, params, totals, grads):
    """The measured error of one timed evaluation (all 4096 chains) against
    the FP64 oracle: max relative logjoint error; max elementwise relative
    gradient error over components whose magnitude does not cancel (|g64| at
    least 1% of the sum of the magnitudes of its terms); and the max of the
    elementwise error over its tolerance (<= 1 passes)."""
    import oracle
    om = oracle.OracleModel(model.lower((X,), {"y": y}))
    t0 = time.perf_counter()
    q64 = params.astype(np.float64)
    t64, g64 = om.logjoint_gradient_f64(q64)
    mag = om.gradient_magnitude_f64(q64)
    err = np.abs(grads.astype(np.float64) - g64)
    keep = np.abs(g64) >= 1e-2 * mag
    return {"chains": int(params.shape[0]),
            "logjoint_max_rel_err": float(np.max(np.abs(totals.astype(np.float64) - t64) / np.abs(t64))),
            "gradient_max_rel_err": float(np.max(err[keep] / np.abs(g64[keep]))),
            "gradient_components_checked_relative": float(keep.mean()),
            "gradient_max_err_over_bound": float(np.max(err / (GRAD_RTOL * np.abs(g64) + GRAD_ATOL_MAG * mag))),
            "gradient_max_norm_rel_err": float(np.max(np.max(err, 1) / np.max(np.abs(g64), 1))),
            "tolerance": f"|g - g64| <= {GRAD_RTOL:g} |g64| + {GRAD_ATOL_MAG:g} * sum_i |term_i|",
            "oracle_s": time.perf_counter() - t0}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's batched GLM
    logjoint + gradient (chain-parallel over every host thread).  Each step is
    one full evaluation of the same 4096-chain batch; warm-up steps are
    untimed, every timed step is timed by itself."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    import oracle
    model, X, y, params = _data()
    om = oracle.OracleModel(model.lower((X,), {"y": y}))
    cores = oracle.max_threads()
    step_s = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        om.logjoint_gradient_f32(params)
        if i >= args.warmup:
            step_s.append(time.perf_counter() - t0)
    total_s = float(sum(step_s))
    value = N_CHAINS * args.steps / total_s
    sample = (f"every step: all {N_CHAINS} chain-gradients of the full N=100000 x D=100 model "
              f"(C++ restatement of the reference's CPU batched path; Julia is not runnable here)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": N_CHAINS, "n_obs": N_OBS, "n_coefs": N_COEF,
                       "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    model, X, y, params = _data()
    ws = DeviceBatchedWorkspace(model, N_CHAINS, args=(X,), constraints={"y": y})
    qd = torch.from_numpy(params).cuda()
    totals = torch.empty(N_CHAINS, device="cuda")
    grads = torch.empty_like(qd)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step():
        ws.logjoint_gradient_device(qd, totals, grads)

    for _ in range(max(args.warmup, 3)):
        flush.fill_(1.0)
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s, e in evs:
        flush.fill_(1.0)  # evict X / params from L2 between steps
        s.record(stream)
        step()
        e.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in evs]
    total_ms = float(sum(step_ms))
    t_max = _max_over_ranks(total_ms, dist)
    clk = clocks.stop()
    value = _replica_value(N_CHAINS * args.steps, world, t_max / 1000.0)

    # end to end through the public host-array API: pinned host params in,
    # host totals + gradients out, every step.
    pinned = torch.from_numpy(params).pin_memory()   # (C, P) chain-major, page-locked
    pt = pinned.numpy().T                              # P x C reference-layout view of it
    for _ in range(2):
        ws.logjoint_gradient(pt)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps = max(10, args.steps)
    for _ in range(e2e_steps):
        vals, g = ws.logjoint_gradient(pt)
    e2e_s = _max_over_ranks(time.perf_counter() - t0, dist)
    e2e_value = _replica_value(N_CHAINS * e2e_steps, world, e2e_s)

    hbm, bf16, peak_kind = _peaks()
    tc = bool(getattr(ws, "tensor_core_path", lambda: False)())
    work = (3.0 if tc else 1.0) * FLOP_FP32 / 1e12   # 3xTF32: three TF32 products per FP32 product
    peak = bf16 / 2.0                                  # dense TF32 = half of dense bf16
    avg_s = (total_ms / args.steps) / 1000.0
    achieved = work / avg_s
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": _profiled_traffic() if tc else None, "peak_source": f"{peak_kind} bf16/2 (dense TF32)",
            "note": ("3xTF32 TF32-FLOPs; traffic = ncu DRAM read+write bytes of one launch "
                     "(profiles/tc_glm_kernel_config3.md)" if tc
                     else "FP32 CUDA-core FLOPs (no tensor-core path active)")}
    cpu = fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, sample = cpu_reference_rate(model, X, y, params, budget_s=args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
        fp64 = fp64_error(model, X, y, params, totals.cpu().numpy(), grads.cpu().numpy())
    launches = int(ws.launches_per_gradient()) * args.steps if hasattr(ws, "launches_per_gradient") else 2 * args.steps
    ws.close()
    if rank == 0:
        # every sub-result is its own short line, printed when it is done; the
        # headline line comes last
        _emit("fp64_error", fp64)
        if world == 1:
            for name, fn in (("hbm_sweep", hbm_sweep), ("hbm_sweep_large", hbm_sweep_large),
                             ("hbm_trajectory", hbm_trajectory)):
                t0 = time.perf_counter()
                _emit(name, fn(), t0)
            samplers = None
            if not args.no_samplers:
                samplers = {}
                for name, fn in (("glm1000x10_hmc", sampler_glm_hmc), ("hier64x20_nuts", sampler_hier_nuts),
                                 ("glm100000x100_nuts", glm_large_nuts), ("glm100000x100_meads", glm_large_meads)):
                    t0 = time.perf_counter()
                    samplers[name] = fn()
                    _emit("samplers." + name, samplers[name], t0)
            if not args.no_surrogate:
                t0 = time.perf_counter()
                sur = surrogate_comparison()
                if samplers is not None:
                    # the metric's own comparison: surrogate-driven trajectories vs plain NUTS on the same model
                    nuts = samplers["glm100000x100_nuts"]
                    sur["plain_nuts"] = {k: nuts[k] for k in ("min_ess_per_s", "min_ess", "max_rank_rhat", "sampling_s")}
                    for v in ("fixed16", "adapted_reference", "adapted_forward"):
                        sur[v]["ratio_vs_plain_nuts"] = sur[v]["surrogate"]["min_ess_per_s"] / nuts["min_ess_per_s"]
                _emit("surrogate_chees", sur, t0)
            if not args.no_uneven:
                t0 = time.perf_counter()
                _emit("uneven_batch", uneven_batch(), t0)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "global_batch": N_CHAINS * world, "n_obs": N_OBS,
                           "n_coefs": N_COEF, "parallelism": f"replicas{world}",
                           "l2": "flushed between timed steps (256 MB write)"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N_CHAINS * N_COEF * 4,
                        "d2h_bytes_per_step": N_CHAINS * (N_COEF + 1) * 4},
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches}
        if fp64 is not None:
            line["fp64_error"] = {k: fp64[k] for k in ("logjoint_max_rel_err", "gradient_max_rel_err",
                                                       "gradient_max_err_over_bound")}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def hbm_sweep_large(num_obs=1_000_000, chain_counts=(1, 4, 16), steps=10, warmup=3):
    """The few-chain streaming evaluation on a design larger than L2 (N =
    1000000 x 100, 400 MB): every evaluation streams X from HBM, and one launch
    is long enough (~60 us at the copy bandwidth) that the launch ramp and the
    fused fold's tail no longer dominate, so this is the kernel's own HBM
    roofline.  Back-to-back evaluations, one event pair per evaluation."""
    import torch
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    from uncertaintea_b200.models import BernoulliLogitGLM, logistic_regression_data
    X, y, _ = logistic_regression_data(num_obs, N_COEF, seed=4, x_scale=1.0 / np.sqrt(N_COEF))
    model = BernoulliLogitGLM(N_COEF)
    hbm, _, kind = _peaks()
    params = np.random.default_rng(1).standard_normal((16, N_COEF)).astype(np.float32)
    stream = torch.cuda.current_stream()
    rows = []
    for C in chain_counts:
        ws = DeviceBatchedWorkspace(model, C, args=(X,), constraints={"y": y})
        qd = torch.from_numpy(params[:C].copy()).cuda()
        totals, grads = torch.empty(C, device="cuda"), torch.empty_like(qd)
        row = {"chains": C, "n_obs": num_obs, "kernel_path": ws.kernel_path()}
        for name, grad in (("logjoint_gradient", True), ("logjoint", False)):
            def step():
                if grad:
                    ws.logjoint_gradient_device(qd, totals, grads)
                else:
                    ws.logjoint_device(qd, totals)
            for _ in range(max(warmup, 3)):
                step()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            for a, b in evs:
                a.record(stream)
                step()
                b.record(stream)
            torch.cuda.synchronize()
            ms = float(np.median([a.elapsed_time(b) for a, b in evs]))
            nbytes = num_obs * N_COEF * 4 + num_obs * 4 + (2 if grad else 1) * C * N_COEF * 4 + C * 4
            gbs = nbytes / (ms / 1000.0) / 1e9
            row[name] = {"ms": ms, "bytes": nbytes, "GB/s": gbs, "frac": gbs / hbm}
        ws.check()
        ws.close()
        rows.append(row)
    return {"metric": "few-chain logjoint(+gradient) HBM roofline, design larger than L2",
            "peak_GB/s": hbm, "peak_source": f"{kind} HBM copy bandwidth",
            "l2": "X (400 MB) > L2 (126 MB): every evaluation reads X from HBM", "rows": rows}


def hbm_trajectory(designs=((100_000, "config-3 design, 40 MB: steps 2..L read X from L2"),
                            (1_000_000, "400 MB design > L2: every step reads X from HBM")),
                   chain_counts=(1, 4), L=8, reps=10, warmup=3):
    """Whole HMC trajectories of L leapfrog steps on the streaming path: the L
    gradient evaluations and the kicks and drifts between them in one
    cooperative launch (bracketed by the momentum and accept kernels), against
    one launch per step (UT_DISABLE_STREAM_TRAJECTORY=1, the same values bit for
    bit).  Achieved GB/s = L x the algorithmic bytes of one evaluation (X and y)
    / the iteration's device time; L2 flushed (256 MB write) before every timed
    iteration, so each trajectory's first read of X comes from HBM."""
    import ctypes
    import torch
    from uncertaintea_b200 import _native as nat
    from uncertaintea_b200.device import DeviceBatchedWorkspace, _stream_handle
    from uncertaintea_b200.models import BernoulliLogitGLM, logistic_regression_data
    hbm, _, kind = _peaks()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    lib = nat.load()
    out = []
    for num_obs, note in designs:
        X, y, _ = logistic_regression_data(num_obs, N_COEF, seed=4, x_scale=1.0 / np.sqrt(N_COEF))
        model = BernoulliLogitGLM(N_COEF)
        nbytes = num_obs * N_COEF * 4 + num_obs * 4
        for C in chain_counts:
            ws = DeviceBatchedWorkspace(model, C, args=(X,), constraints={"y": y})
            q0 = torch.from_numpy((0.05 * np.random.default_rng(2).standard_normal((C, N_COEF))).astype(np.float32)).cuda()
            f = lambda dt=torch.float32: torch.zeros(C, dtype=dt, device="cuda")  # noqa: E731
            outs = [f(), f(), f(), f(torch.uint8), f(torch.uint8)]
            im = torch.ones(N_COEF, device="cuda")
            stp = torch.full((C,), 1e-3, device="cuda")
            row = {"chains": C, "n_obs": num_obs, "L": L, "kernel_path": ws.kernel_path(), "note": note}
            for name, env in (("one_launch", None), ("launch_per_step", "1")):
                if env:
                    os.environ["UT_DISABLE_STREAM_TRAJECTORY"] = env
                else:
                    os.environ.pop("UT_DISABLE_STREAM_TRAJECTORY", None)
                qd = q0.clone()
                t, g = ws.logjoint_gradient_device(qd)
                buf = nat.HmcBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(im), nat.ptr(stp),
                                     *[nat.ptr(o) for o in outs], None, None)
                times = []
                for it in range(warmup + reps):
                    flush.fill_(1.0)
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    nat.check(lib.ut_hmc_iteration(ws.handle, ctypes.byref(buf), L, 1000 + it, 1000.0,
                                                   _stream_handle()))
                    b.record(stream)
                    torch.cuda.synchronize()
                    if it >= warmup:
                        times.append(a.elapsed_time(b))
                ms = float(np.median(times))
                gbs = L * nbytes / (ms / 1000.0) / 1e9
                row[name] = {"ms": ms, "us_per_step": 1000.0 * ms / L, "GB/s": gbs, "frac": gbs / hbm}
                ws.check()
            os.environ.pop("UT_DISABLE_STREAM_TRAJECTORY", None)
            ws.check()
            ws.close()
            out.append(row)
    return {"metric": "few-chain HMC trajectory (L leapfrog evaluations), achieved GB/s of L x (X + y)",
            "peak_GB/s": hbm, "peak_source": f"{kind} HBM copy bandwidth",
            "l2": "flushed (256 MB write) before every timed iteration", "rows": out}


def hbm_sweep(chain_counts=(1, 4, 8, 16), steps=20, warmup=5):
    """Few-chain logjoint + gradient on the same 100000 x 100 design, where one
    evaluation must read all of X from HBM: achieved bytes per second against the
    measured HBM copy bandwidth.  Algorithmic bytes per evaluation = X (N*F*4) +
    y (N*4) + parameters in and gradients out (2*C*F*4) + values out (C*4).  L2 is
    flushed (256 MB write) before every timed evaluation; per-step CUDA events."""
    import torch
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    model, X, y, params = _data()
    hbm, _, kind = _peaks()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    out = []
    for C in chain_counts:
        ws = DeviceBatchedWorkspace(model, C, args=(X,), constraints={"y": y})
        qd = torch.from_numpy(params[:C].copy()).cuda()
        totals = torch.empty(C, device="cuda")
        grads = torch.empty_like(qd)
        row = {"chains": C, "kernel_path": ws.kernel_path()}
        for name, grad in (("logjoint_gradient", True), ("logjoint", False)):
            def step():
                if grad:
                    ws.logjoint_gradient_device(qd, totals, grads)
                else:
                    ws.logjoint_device(qd, totals)
            for _ in range(max(warmup, 3)):
                flush.fill_(1.0)
                step()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            for a, b in evs:
                flush.fill_(1.0)
                a.record(stream)
                step()
                b.record(stream)
            torch.cuda.synchronize()
            ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
            nbytes = N_OBS * N_COEF * 4 + N_OBS * 4 + (2 if grad else 1) * C * N_COEF * 4 + C * 4
            gbs = nbytes / (ms / 1000.0) / 1e9
            row[name] = {"ms": ms, "bytes": nbytes, "GB/s": gbs, "frac": gbs / hbm}
        # sustained: evaluations back to back over 6 workspaces holding their own
        # copies of X (240 MB > the 126 MB L2, visited cyclically, so every
        # evaluation reads its design from HBM), one event pair around them all
        extra = [DeviceBatchedWorkspace(model, C, args=(X,), constraints={"y": y}) for _ in range(5)]
        ring = [ws] + extra
        reps = 10 * len(ring)
        for _ in range(2):
            for w in ring:
                w.logjoint_gradient_device(qd, totals, grads)
        a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a_ev.record(stream)
        for r in range(reps):
            ring[r % len(ring)].logjoint_gradient_device(qd, totals, grads)
        b_ev.record(stream)
        torch.cuda.synchronize()
        ms = a_ev.elapsed_time(b_ev) / reps
        nbytes = N_OBS * N_COEF * 4 + N_OBS * 4 + 2 * C * N_COEF * 4 + C * 4
        row["sustained_logjoint_gradient"] = {"ms": ms, "GB/s": nbytes / (ms / 1000.0) / 1e9,
                                              "frac": nbytes / (ms / 1000.0) / 1e9 / hbm,
                                              "method": "back-to-back over 6 copies of X (240 MB > L2), no flush"}
        for w in extra:
            w.close()
        out.append(row)
        ws.close()
    # Yardsticks under the same flush + event method: a one-element fill (the
    # launch + event floor of a single timed launch) and torch's own sum over a
    # device copy of the same 40 MB design (a library read of the same bytes).
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    tiny = torch.empty(1, device="cuda")
    yard = {}
    for name, fn in (("launch_floor_one_element_fill", lambda: tiny.fill_(0.0)),
                     ("torch_sum_of_X", lambda: Xd.sum())):
        for _ in range(max(warmup, 3)):
            flush.fill_(1.0)
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in evs:
            flush.fill_(1.0)
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
        nbytes = 0 if name.startswith("launch") else N_OBS * N_COEF * 4
        yard[name] = {"ms": ms, "GB/s": nbytes / (ms / 1000.0) / 1e9, "frac": nbytes / (ms / 1000.0) / 1e9 / hbm}
    return {"metric": "few-chain logjoint(+gradient) HBM roofline", "peak_GB/s": hbm,
            "peak_source": f"{kind} HBM copy bandwidth", "l2": "flushed before every timed evaluation",
            "rows": out, "yardsticks": yard}


def _device_diagnostics(ch, S=None, chunk=None):
    """Rank-normalised split R-hat, plain split R-hat and bulk ESS per
    parameter of the first S draws of ch's unconstrained draws, computed on the
    device a few parameters at a time with the reference's estimators
    (uncertaintea_b200.multi: rank_split_rhat, split_rhat, split_ess; they
    agree with the host diagnostics to 1e-9).  The host estimators take
    minutes on 4096 chains x 1000 draws x 100 parameters."""
    import torch
    from uncertaintea_b200.multi import rank_split_rhat, split_ess, split_rhat
    d = ch.unconstrained                        # (C, S_total, P)
    C, S_tot, P = d.shape
    S = S_tot if S is None else S
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    if chunk is None:   # about 1.6 GB of float64 draws per chunk
        chunk = max(1, min(16, int(2e8 // (S * C))))
    r_rank, r_split, e = np.empty(P), np.empty(P), np.empty(P)
    for p0 in range(0, P, chunk):
        p1 = min(P, p0 + chunk)
        x = torch.from_numpy(np.ascontiguousarray(d[:, :S, p0:p1].transpose(1, 0, 2))).to(dev)   # (S, C, p)
        r_rank[p0:p1] = torch.nan_to_num(rank_split_rhat(x), nan=float("inf")).cpu().numpy()
        r_split[p0:p1] = torch.nan_to_num(split_rhat(x), nan=float("inf")).cpu().numpy()
        e[p0:p1] = torch.nan_to_num(split_ess(x), nan=float("inf")).cpu().numpy()
        del x
    return r_rank, r_split, e


def _chain_summary(ch, cfg, extra=None):
    """Min bulk ESS/s and both R-hats of a sampler run.  The gate is the
    reference's: rank-normalised split R-hat < 1.01 (diagnostics.jl:607-612,
    docs/benchmarks.md:8-13); the plain split R-hat is reported beside it."""
    r_rank, r_split, e = _device_diagnostics(ch)
    total_s = ch.warmup_seconds + ch.sampling_seconds
    out = {"min_ess_per_s": float(np.min(e) / ch.sampling_seconds), "min_ess": float(np.min(e)),
           "max_rank_rhat": float(np.max(r_rank)), "max_split_rhat": float(np.max(r_split)),
           "gate_rank_rhat_lt_1.01": bool(np.max(r_rank) < 1.01),
           "warmup_s": ch.warmup_seconds, "sampling_s": ch.sampling_seconds,
           "grad_evals_per_s": ch.gradient_evaluations / total_s, "mean_accept": float(ch.accept_prob.mean()),
           "config": cfg}
    out.update(extra or {})
    return out


def _gate_prefixes(ch, lengths):
    """The gate on the first S draws of every chain, for each S in lengths: max
    rank-normalised split R-hat and min bulk ESS over parameters (the
    reference's estimators, computed per parameter on the device:
    multi.rank_split_rhat / multi.split_ess), and min-ESS/s over the device
    time of those S sampling iterations (a sampling iteration's cost does not
    depend on its index, so that time is the run's times S / S_total)."""
    S_tot = ch.unconstrained.shape[1]
    rows = []
    for S in lengths:
        if S > S_tot:
            break
        r_rank, _, e = _device_diagnostics(ch, S)
        r_max, e_min = float(np.max(r_rank)), float(np.min(e))
        t = ch.sampling_seconds * S / S_tot
        rows.append({"draws": S, "max_rank_rhat": r_max, "min_ess": e_min, "min_ess_per_s": e_min / t,
                     "gate_rank_rhat_lt_1.01": bool(r_max < 1.01)})
    return rows


def _gated_summary(ch, cfg, lengths, extra=None):
    """The 1000-draw figures (as configured) and the gate over longer prefixes of
    the same run: `gate` is the shortest prefix whose rank R-hat is below 1.01
    (null when none is)."""
    rows = _gate_prefixes(ch, lengths)
    first = rows[0]
    passed = [r for r in rows if r["gate_rank_rhat_lt_1.01"]]
    total_s = ch.warmup_seconds + ch.sampling_seconds
    out = {"min_ess_per_s": first["min_ess_per_s"], "min_ess": first["min_ess"],
           "max_rank_rhat": first["max_rank_rhat"], "gate_rank_rhat_lt_1.01": first["gate_rank_rhat_lt_1.01"],
           "draws": first["draws"], "gate": passed[0] if passed else None, "prefixes": rows,
           "warmup_s": ch.warmup_seconds, "sampling_s_all_draws": ch.sampling_seconds,
           "grad_evals_per_s": ch.gradient_evaluations / total_s, "mean_accept": float(ch.accept_prob.mean()),
           "config": cfg}
    out.update(extra or {})
    return out


def sampler_glm_hmc(num_samples=16000):
    """Batched HMC on the 1000 x 10 logistic regression: 256 chains, 8 leapfrog
    steps, step 0.05 without step adaptation, 1000 warmup, seed 1.  The
    configured 1000 draws are the first 1000 of one run of num_samples; the
    gate is evaluated on longer prefixes of it."""
    from uncertaintea_b200 import BernoulliLogitGLM, batched_hmc, logistic_regression_data
    X, y, _ = logistic_regression_data(1000, 10, seed=1)
    ch = batched_hmc(BernoulliLogitGLM(10), (X,), {"y": y}, num_chains=256, num_samples=num_samples,
                     num_warmup=1000, step_size=0.05, num_leapfrog_steps=8, adapt_step_size=False, rng=1)
    return _gated_summary(ch, f"256 chains, L=8, step 0.05, 1000 warmup + 1000 draws (gate on up to "
                              f"{num_samples}), GLM 1000x10", [1000, 2000, 4000, 8000, 16000])


def sampler_hier_nuts(num_samples=8000):
    """Batched persistent NUTS on the non-centred hierarchical model with J = 64
    groups x 20 observations (sigma_j ~ U(0.5, 2), y from the prior at seed 7;
    4096 chains, max tree depth 10, 1000 warmup).  The configured 1000 draws are
    the first 1000 of one run of num_samples; the gate is evaluated on longer
    prefixes of it."""
    from uncertaintea_b200 import HierarchicalNormalNoncentered, batched_nuts, hierarchical_data
    yh, sig, sizes, _ = hierarchical_data(64, 20, 7)
    ch = batched_nuts(HierarchicalNormalNoncentered(64), (sig, sizes), {"y": yh}, num_chains=4096,
                      num_samples=num_samples, num_warmup=1000, max_tree_depth=10, rng=7)
    return _gated_summary(ch, f"4096 chains, depth 10, 1000 warmup + 1000 draws (gate on up to {num_samples}), "
                              "hierarchical J=64 x 20", [1000, 2000, 4000, 8000],
                          {"mean_tree_depth": float(ch.tree_depth.mean())})


def glm_large_nuts(num_chains=4096, num_warmup=200, num_samples=200):
    """Masked (lockstep) NUTS on the large logistic regression, 4096 chains, max
    tree depth 10: every leaf is one batched tensor-core gradient over the chains
    whose trees are still growing (compacted).  Fewer iterations than the small-model runs
    (200 + 200) keep the bench within minutes; the draws are still nearly
    independent (min ESS at the draw count)."""
    from uncertaintea_b200 import batched_nuts
    model, X, y, _ = _data()
    ch = batched_nuts(model, (X,), {"y": y}, num_chains=num_chains, num_samples=num_samples, num_warmup=num_warmup,
                      max_tree_depth=10, tree_strategy="masked", rng=1)
    return _chain_summary(ch, f"{num_chains} chains, masked NUTS depth 10, {num_warmup}+{num_samples}, GLM 100000x100",
                          {"ms_per_sampling_iteration": 1e3 * ch.sampling_seconds / num_samples,
                           "mean_tree_depth": float(ch.tree_depth.mean()), "max_tree_depth": int(ch.tree_depth.max()),
                           "mean_leapfrog_steps": float(ch.integration_steps.mean())})


def glm_large_meads(num_chains=4096, num_warmup=3000, num_samples=1000):
    """MEADS on the large logistic regression (4096 chains, 4 folds): one
    batched tensor-core gradient per iteration, every adaptation statistic on
    the device, no warmup adaptation phase.  Started from prior draws (a
    posterior ~15x narrower than the prior) the ensemble step size grows from
    3e-4 to ~0.5 over ~2500 iterations as the folds contract, so the first 3000
    draws are discarded."""
    from uncertaintea_b200 import batched_meads
    model, X, y, _ = _data()
    ch = batched_meads(model, (X,), {"y": y}, num_chains=num_chains, num_samples=num_samples,
                       num_warmup=num_warmup, rng=1)
    return _chain_summary(ch, f"{num_chains} chains, MEADS 4 folds, {num_warmup} discarded + {num_samples}, "
                          "GLM 100000x100", {"ms_per_iteration": 1e3 * ch.sampling_seconds / num_samples,
                                             "step_size": float(np.mean(ch.step_size))})


def _surrogate_pair(model, X, y, **kw):
    """Plain ChEES-HMC and surrogate-driven ChEES-HMC with the same settings:
    min ESS per sampling second (and per total second: warmup + surrogate
    training + sampling), rank R-hat, mean trajectory steps, the ratio, and
    the largest difference of posterior means in posterior SDs."""
    from uncertaintea_b200 import batched_chees, batched_chees_surrogate
    runs = {"plain": batched_chees(model, (X,), {"y": y}, **kw),
            "surrogate": batched_chees_surrogate(model, (X,), {"y": y}, **kw)}
    out = {}
    for name, ch in runs.items():
        r, _, e = _device_diagnostics(ch)
        total_s = ch.warmup_seconds + ch.sampling_seconds
        out[name] = {"min_ess_per_s": float(np.min(e) / ch.sampling_seconds), "min_ess": float(np.min(e)),
                     "min_ess_per_total_s": float(np.min(e) / total_s), "max_rank_rhat": float(np.max(r)),
                     "sampling_s": ch.sampling_seconds, "warmup_s": ch.warmup_seconds,
                     "mean_leapfrog_steps": float(ch.integration_steps.mean()),
                     "mean_accept": float(ch.accept_prob.mean()), "step_size": float(np.mean(ch.step_size))}
    rep = runs["surrogate"].surrogate
    out["surrogate"].update({"pairs": rep.num_pairs, "train_steps": rep.train_steps, "train_s": rep.train_seconds,
                             "relative_error": rep.relative_error_after_training, "fallback_at": rep.fallback_at})
    up = runs["plain"].unconstrained.reshape(-1, N_COEF)
    us = runs["surrogate"].unconstrained.reshape(-1, N_COEF)
    out["max_mean_diff_in_sd"] = float(np.max(np.abs(up.mean(0) - us.mean(0)) / up.std(0)))
    out["ratio"] = out["surrogate"]["min_ess_per_s"] / out["plain"]["min_ess_per_s"]
    out["ratio_including_warmup_and_training"] = (out["surrogate"]["min_ess_per_total_s"]
                                                  / out["plain"]["min_ess_per_total_s"])
    out["gate_rank_rhat_lt_1.01"] = bool(max(out["plain"]["max_rank_rhat"], out["surrogate"]["max_rank_rhat"]) < 1.01)
    return out


def surrogate_comparison(num_chains=4096, num_warmup=500, num_samples=500):
    """The learned-surrogate workload on the same model: ChEES-HMC with exact
    gradients vs ChEES-HMC whose trajectories the trained MLP drives (exact
    logjoint in the accept), same seeds and settings.  The surrogate is trained
    on 2^20 (theta, gradient) pairs of the last 256 warmup iterations.
    Variants:
      fixed16            -- 16 leapfrog steps every iteration (the trajectory
                            budget of the configuration), step size adapted,
                            then Halton-jittered per sampling iteration;
      adapted_reference  -- trajectory length adapted with the reference's
                            estimator (16 initial steps);
      adapted_forward    -- adapted with the forward endpoint velocity (an
                            ascent on the ChEES criterion).
    Min ESS over the 100 coefficients per second of sampling, and per second
    of warmup + training + sampling.  The fixed-16 pair samples twice as many
    iterations: at 16 steps of the adapted step size its draws are more
    autocorrelated, and 500 of them stop just short of rank R-hat < 1.01."""
    model, X, y, _ = _data()
    base = dict(num_chains=num_chains, num_samples=num_samples, num_warmup=num_warmup, rng=1)
    fixed = dict(base, num_samples=2 * num_samples)
    out = {"fixed16": _surrogate_pair(model, X, y, fixed_leapfrog_steps=16, **fixed),
           "adapted_reference": _surrogate_pair(model, X, y, num_leapfrog_steps=16, **base),
           "adapted_forward": _surrogate_pair(model, X, y, num_leapfrog_steps=16, trajectory_velocity="forward",
                                              **base)}
    out["metric"] = "min ESS/s (rank R-hat<1.01), surrogate ChEES-HMC vs plain ChEES-HMC"
    out["unit"] = "effective samples/s"
    out["config"] = (f"learned gradient surrogate on the 100000x100 logistic regression, {num_chains} chains, "
                     f"{num_warmup} warmup + {num_samples} sampling iterations ({2 * num_samples} for fixed16)")
    return out


def uneven_models(num_models=512, seed=5):
    """The uneven-batch workload: num_models independent non-centred
    hierarchical normal models with J ~ UniformInt[8, 512] groups and
    UniformInt[5, 100] observations per group, sigma_j ~ U(0.5, 2), y drawn
    from the prior predictive (seeded)."""
    from uncertaintea_b200.models import HierarchicalNormalNoncentered, hierarchical_data
    r = np.random.default_rng(seed)
    models = []
    for i in range(num_models):
        J = int(r.integers(8, 513))
        sizes = r.integers(5, 101, size=J)
        y, sig, sz, _ = hierarchical_data(J, sizes, 1000 + i)
        models.append((HierarchicalNormalNoncentered(J), (sig, sz), {"y": y}))
    return models


def uneven_batch(num_models=512, chains=64, num_warmup=500, num_samples=1000):
    """All models in one batched persistent-NUTS run (one launch per
    parameter-slot class per iteration, replayed from a CUDA graph, launch
    shapes from the autotuner): aggregate min-ESS per sampling second and the
    per-model time to R-hat < 1.01 (checked every 50 draws).  Per-model
    stopping: a model that reaches the target stops there and the rest run on,
    up to num_samples draws (the cap); ESS and R-hat are over each model's own
    draws."""
    from uncertaintea_b200.multi import batched_nuts_multi
    models = uneven_models(num_models)
    res = batched_nuts_multi(models, chains_per_model=chains, num_warmup=num_warmup, num_samples=num_samples,
                             rng=1, rhat_check_every=50, stop_converged=True)
    drawn = int(res.draws_per_model.max())
    fin = lambda v: v if np.isfinite(v) else None  # noqa: E731  (null: not reached within the run)
    p50, p99 = (fin(v) for v in res.time_to_rhat_quantiles())
    s50, s99 = (fin(v) for v in res.time_to_rhat_quantiles(from_sampling=True))
    cls = res.classes
    out = {"metric": "aggregate min-ESS/s; per-model time to R-hat<1.01 (p50/p99 over models)",
           "unit": "effective samples/s; s", "aggregate_ess_per_s": res.aggregate_ess_per_second,
           "time_to_rhat_p50_s": p50, "time_to_rhat_p99_s": p99,
           "sampling_time_to_rhat_p50_s": s50, "sampling_time_to_rhat_p99_s": s99,
           "time_to_rhat_note": "null = that share of models did not reach R-hat < 1.01 within the run",
           "converged_fraction": res.converged_fraction, "median_model_min_ess": float(np.median(res.min_ess)),
           "converged_models_time_to_rhat_p50_s": (float(np.median(res.time_to_rhat[np.isfinite(res.time_to_rhat)]))
                                                   if np.isfinite(res.time_to_rhat).any() else None),
           "final_rank_rhat_p50": float(np.median(res.max_rhat)),
           "final_rank_rhat_p99": float(np.quantile(res.max_rhat, 0.99)),
           "warmup_s": res.warmup_seconds, "sampling_s": res.sampling_seconds,
           "ms_per_iteration": 1000.0 * res.sampling_seconds / max(drawn, 1),
           "draws_cap": num_samples, "draws_run": drawn,
           "draws_per_model_p50": float(np.median(res.draws_per_model)),
           "mean_tree_depth": res.mean_tree_depth, "divergences": res.divergences,
           "total_obs": int(sum(int(m[1][1].sum()) for m in models)), "total_chains": int(res.num_chains.sum()),
           "classes": {"slots": cls["slots"].tolist(), "models": cls["models"].tolist(),
                       "chains_per_block": cls["chains_per_block"].tolist(),
                       "stage_limit_bytes": cls["stage_limit_bytes"].tolist()},
           "config": (f"uneven batch: {num_models} non-centred hierarchical models, J~U[8,512], obs/group~U[5,100], "
                      f"{chains} chains each, max tree depth 10, {num_warmup} warmup + up to {num_samples} draws, "
                      "per-model stopping at R-hat<1.01, CUDA graph replay, autotuned launch shapes")}
    res.batch.close()
    return out


def run_kernel_only(args):
    """Only the device evaluations (no L2 flush, no e2e, no CPU leg): the
    command the ncu summaries under profiles/ were captured with."""
    import torch
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    model, X, y, params = _data()
    ws = DeviceBatchedWorkspace(model, N_CHAINS, args=(X,), constraints={"y": y})
    qd = torch.from_numpy(params).cuda()
    for _ in range(args.warmup + args.steps):
        t, g = ws.logjoint_gradient_device(qd)
    torch.cuda.synchronize()
    ws.check()
    print(json.dumps({"kernel_path": ws.kernel_path(), "evaluations": args.warmup + args.steps}))
    ws.close()


def run_trajectory_only(args):
    """Only one-launch HMC trajectories (L = 8) of one chain on the 1000000 x 100
    design, args.steps of them: the command the trajectory kernel's ncu summary
    under profiles/ was captured with."""
    import ctypes
    import torch
    from uncertaintea_b200 import _native as nat
    from uncertaintea_b200.device import DeviceBatchedWorkspace, _stream_handle
    from uncertaintea_b200.models import BernoulliLogitGLM, logistic_regression_data
    X, y, _ = logistic_regression_data(1_000_000, N_COEF, seed=4, x_scale=1.0 / np.sqrt(N_COEF))
    ws = DeviceBatchedWorkspace(BernoulliLogitGLM(N_COEF), 1, args=(X,), constraints={"y": y})
    qd = torch.from_numpy((0.05 * np.random.default_rng(2).standard_normal((1, N_COEF))).astype(np.float32)).cuda()
    t, g = ws.logjoint_gradient_device(qd)
    im, st = torch.ones(N_COEF, device="cuda"), torch.full((1,), 1e-3, device="cuda")
    outs = [torch.zeros(1, device="cuda") for _ in range(3)] + [torch.zeros(1, dtype=torch.uint8, device="cuda")
                                                               for _ in range(2)]
    buf = nat.HmcBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(im), nat.ptr(st), *[nat.ptr(o) for o in outs],
                         None, None)
    for it in range(args.steps):
        nat.check(nat.load().ut_hmc_iteration(ws.handle, ctypes.byref(buf), 8, 100 + it, 1000.0, _stream_handle()))
    torch.cuda.synchronize()
    ws.check()
    print(json.dumps({"kernel_path": ws.kernel_path(), "trajectories": args.steps, "L": 8}))
    ws.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--kernel-only", action="store_true")
    ap.add_argument("--trajectory-only", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the learned-surrogate ChEES comparison (about a minute) in the output line")
    ap.add_argument("--no-samplers", action="store_true",
                    help="skip the small-model HMC and NUTS sampler runs in the output line")
    ap.add_argument("--no-uneven", action="store_true",
                    help="skip the uneven-batch run (512 hierarchical models, about two minutes)")
    args = ap.parse_args()
    if args.trajectory_only:
        run_trajectory_only(args)
        return
    if args.kernel_only:
        run_kernel_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
