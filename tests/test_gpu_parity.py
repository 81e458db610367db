"""GPU parity tests: the sm_100a kernels, called through the C ABI, against the
CPU oracle on the same seeded inputs.

Tolerances (stated per test):
* Philox blocks and uniforms: bit-exact.
* Box-Muller normals: |gpu - oracle| <= 2e-6 * max(1, |oracle|) (libm vs CUDA
  logf/cosf differ in the last bits, rng.jl:185-194).
* logjoint (FP32) vs the FP64 oracle: |lj - lj64| <= 1e-5 * |lj64|.
* gradient (FP32) vs the FP64 oracle, elementwise:
  |g - g64| <= 1e-5 |g64| + 1e-6 m, m = the sum of the magnitudes of the terms
  the component adds up (the scale of FP32 summation error, see GRAD_ATOL_MAG),
  and per chain max_p |g - g64| <= 1e-5 max_p |g64|.
* HMC / NUTS iterations vs the FP32 oracle under identical Philox streams:
  the same accept / tree decisions for >= 98% of chains, and states of the
  chains with identical decisions within rtol 1e-3, atol 1e-4.  An HMC accept
  decision that differs must be a near-tie: the chain's accept uniform lies
  between the two sides' accept probabilities.
"""
import ctypes

import numpy as np
import pytest

import oracle
from uncertaintea_b200 import _native as nat
from uncertaintea_b200.models import (BernoulliBeta, BernoulliLogitGLM, HierarchicalNormalNoncentered,
                                      LognormalGammaNormal, NormalKnownScale, NormalLocationScale, StudentTHeavyTail,
                                      gauss_data,
                                      hierarchical_data, logistic_regression_data)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ws(model, args, constraints, C):
    from uncertaintea_b200.device import DeviceBatchedWorkspace
    return DeviceBatchedWorkspace(model, C, args=args, constraints=constraints)


GRAD_RTOL = 1e-5
# Absolute part of the elementwise gradient tolerance, as a fraction of the
# gradient magnitude m: the sum of the magnitudes of the terms a component adds
# up (oracle gradient_magnitude_f64).  An FP32 sum errs by a multiple of the
# unit roundoff times m, not times the sum itself, so a component whose terms
# cancel (|g64| << m) cannot meet a purely relative bound in FP32 however it
# is summed.  1e-6 m is about 17 FP32 roundoffs of m; the largest error
# measured on any kernel path (warp, tiled, tensor core, streaming, live-chain
# re-split, all 4096 chains of the 100000 x 100 design) is 3.9e-7 m.
GRAD_ATOL_MAG = 1e-6


def _ref(om, q):
    """FP64 oracle logjoint, gradient and gradient magnitude of chain-major q."""
    q64 = np.asarray(q, dtype=np.float64)
    t64, g64 = om.logjoint_gradient_f64(q64)
    return t64, g64, om.gradient_magnitude_f64(q64)


def _grad_err(g, g64):
    """Per-chain norm-relative error: max_p |g - g64| / max_p |g64|."""
    scale = np.maximum(np.max(np.abs(g64), axis=1), 1e-30)
    return np.max(np.max(np.abs(g.astype(np.float64) - g64), axis=1) / scale)


def _grad_ok(g, g64, mag, norm=True):
    """Both gradient bounds: elementwise |g - g64| <= 1e-5 |g64| + 1e-6 m, and
    (norm=True) the per-chain norm bound max_p |g - g64| <= 1e-5 max_p |g64|."""
    g = np.asarray(g, dtype=np.float64)
    ratio = np.abs(g - g64) / (GRAD_RTOL * np.abs(g64) + GRAD_ATOL_MAG * mag)
    over = np.max(ratio)
    ok = over <= 1.0 and (not norm or _grad_err(g, g64) <= GRAD_RTOL)
    if not ok:  # the worst component, shown with the failing assert
        i = np.unravel_index(np.argmax(ratio), ratio.shape)
        print(f"gradient bound: worst {i}: g={g[i]!r} g64={g64[i]!r} m={mag[i]!r} over={over:.3g}; "
              f"norm error {_grad_err(g, g64):.3g}")
    return ok


def _lj_err(t, t64):
    return np.max(np.abs(t.astype(np.float64) - t64) / np.maximum(np.abs(t64), 1e-30))


# ---------------------------------------------------------------- Philox ----
def test_philox_kat_gpu(lib, pins):
    from uncertaintea_b200 import rng
    for case in pins["philox4x32_10_kat"]:
        assert rng.philox4x32(case["key"], case["counter"]) == tuple(case["expected"])


def test_philox_batch_bit_exact_vs_oracle(lib):
    from uncertaintea_b200 import rng
    r = np.random.default_rng(0)
    keys = r.integers(0, 2 ** 32, size=(4096, 2), dtype=np.uint64).astype(np.uint32)
    ctrs = r.integers(0, 2 ** 32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    got = rng.philox4x32_batch(keys, ctrs)
    for i in range(0, 4096, 37):
        assert tuple(got[i]) == oracle.philox4x32(keys[i], ctrs[i])


def test_uniform_bit_exact_and_normal_close(lib):
    from uncertaintea_b200 import rng
    for chain, it, stream in [(0, 0, 0), (7, 123456, 2), (4095, 2 ** 32 - 1, 4)]:
        u = rng.device_rand_uniform(chain, it, stream, 0, n=20000)
        assert np.array_equal(u, oracle.rand_uniform(chain, it, stream, 0, 20000))
        z = rng.device_rand_normal(chain, it, stream, 0, n=20000)
        zo = oracle.rand_normal(chain, it, stream, 0, 20000)
        assert np.all(np.abs(z - zo) <= 2e-6 * np.maximum(1.0, np.abs(zo)))


# ---------------------------------------------------------- densities -------
def _glm_case(N, D, C, intercept, seed, scale=1.0):
    X, y, _ = logistic_regression_data(N, D, seed, x_scale=scale)
    m = BernoulliLogitGLM(D, intercept=intercept, coef_sigma=1.0, intercept_sigma=2.5)
    q = np.random.default_rng(seed + 1).standard_normal((C, m.num_params())).astype(np.float32)
    return m, (X,), {"y": y}, q


@pytest.mark.parametrize("N,D,C,intercept,scale", [
    (1000, 10, 256, False, 1.0),      # 1000x10 GLM, warp path (data staged in shared memory)
    (777, 5, 33, True, 1.0),          # ragged sizes, intercept
    (20000, 100, 200, True, 0.1),     # tiled path
    (3000, 40, 64, False, 1.0),       # tiled path, D just above the warp path
    (5000, 256, 40, False, 0.1),      # the largest GLM (256 parameters), tiled path
    (3000, 255, 20, True, 0.1),       # 255 covariates + intercept = 256 parameters
])
def test_glm_density_vs_fp64_oracle(lib, N, D, C, intercept, scale):
    m, args, cons, q = _glm_case(N, D, C, intercept, 11, scale)
    ws = _ws(m, args, cons, C)
    t, g = ws.logjoint_gradient(q.T)
    t_only = ws.logjoint(q.T)
    om = oracle.OracleModel(ws.lowered)
    t64, g64, mag = _ref(om, q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _lj_err(t_only, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


def test_glm_density_full_size_all_chains(lib):
    """Full size (N=100000, D=100, C=4096) on the tensor-core path: every one of
    the 4096 chains against the FP64 oracle, elementwise."""
    m, args, cons, q = _glm_case(100000, 100, 4096, False, 3, 0.1)
    ws = _ws(m, args, cons, 4096)
    assert ws.kernel_path() == "tensor_core"
    qd = torch.from_numpy(q).cuda()
    t, g = ws.logjoint_gradient_device(qd)
    torch.cuda.synchronize()
    ws.check()
    t, g = t.cpu().numpy(), g.cpu().numpy()
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q)
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(g, g64, mag)
    ws.close()


@pytest.mark.parametrize("live", [1, 127, 300, 2049])
def test_tensor_core_live_chains_vs_oracle(lib, live):
    """The live-chain launch masked NUTS makes at every leaf (only the first
    `live` of 4096 chains evaluated; few live chain tiles re-split the
    observations so the launch still fills the SMs) at the full 100000 x 100
    size: the live rows against the FP64 oracle, the rows past them untouched."""
    m, args, cons, q = _glm_case(100000, 100, 4096, False, 3, 0.1)
    ws = _ws(m, args, cons, 4096)
    assert ws.kernel_path() == "tensor_core"
    fn = lib.ut_internal_tc_glm_live
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p] * 6
    qd = torch.from_numpy(q).cuda()
    t = torch.full((4096,), float("nan"), device="cuda")
    g = torch.full((4096, 100), float("nan"), device="cuda")
    n = torch.tensor([live], dtype=torch.int32, device="cuda")
    nat.check(fn(ws.handle, nat.ptr(qd), nat.ptr(t), nat.ptr(g), nat.ptr(n), None))
    torch.cuda.synchronize()
    ws.check()
    t, g = t.cpu().numpy(), g.cpu().numpy()
    assert np.all(np.isnan(t[live:])) and np.all(np.isnan(g[live:]))
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q[:live])
    assert _lj_err(t[:live], t64) <= 1e-5
    assert _grad_ok(g[:live], g64, mag)
    ws.close()


def test_host_arrays_are_independent_and_any_layout(lib):
    """The host-array entry points return fresh arrays on every call (the
    reference's allocating copies, api.jl:103-106), in page-locked memory; a
    float64 or row-major P x C input gives the same values as the chain-major
    float32 one (bitwise: the same float32 parameters reach the device)."""
    m, args, cons, q = _glm_case(20000, 100, 200, True, 5, 0.1)
    ws = _ws(m, args, cons, 200)
    t1, g1 = ws.logjoint_gradient(q.T)
    t1c, g1c = t1.copy(), np.array(g1)
    t2, g2 = ws.logjoint_gradient((q * 0.5).T)
    assert np.array_equal(t1, t1c) and np.array_equal(g1, g1c)   # the first results were not overwritten
    assert not np.array_equal(t1, t2)
    assert torch.from_numpy(t1).is_pinned() and torch.from_numpy(np.ascontiguousarray(g1.T)).is_pinned()
    for alt in (q.T.astype(np.float64), np.ascontiguousarray(q.T), np.asfortranarray(q.T.astype(np.float64))):
        ta, ga = ws.logjoint_gradient(alt)
        assert np.array_equal(ta, t1) and np.array_equal(ga, g1)
        assert np.array_equal(ws.logjoint(alt), ws.logjoint(q.T))
    ws.close()


@pytest.mark.parametrize("J,n,C", [(64, 20, 512), (8, 5, 3), (150, 7, 40), (542, 2, 8)])  # 542: 544 params, the max
def test_hier_density_vs_fp64_oracle(lib, J, n, C):
    y, sig, sizes, _ = hierarchical_data(J, n, 7)
    m = HierarchicalNormalNoncentered(J)
    q = (np.random.default_rng(4).standard_normal((C, J + 2)) * 0.7).astype(np.float32)
    ws = _ws(m, (sig, sizes), {"y": y}, C)
    t, g = ws.logjoint_gradient(q.T)
    om = oracle.OracleModel(ws.lowered)
    t64, g64, mag = _ref(om, q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


@pytest.mark.parametrize("n,C", [(5, 4), (1000, 300), (20000, 37), (0, 8)])
def test_gauss_density_vs_fp64_oracle(lib, n, C):
    """The normal location/scale family (the reference's gaussian device model);
    n = 5, C = 4 is the reference's own parity case (device_lowering_parity.jl:131-134)."""
    if n == 5:
        y = np.array([0.4, -0.7, 1.1, 0.2, 0.9], dtype=np.float32)
        q = np.array([[0.5, 0.1], [-0.3, 0.7], [1.2, -0.2], [0.05, 0.4]], dtype=np.float32)
    else:
        y, _ = gauss_data(n, 9)
        q = (np.random.default_rng(5).standard_normal((C, 2)) * 0.6).astype(np.float32)
    m = NormalLocationScale()
    ws = _ws(m, (n,), {"y": y}, C)
    assert ws.kernel_path() == "warp"
    t, g = ws.logjoint_gradient(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


@pytest.mark.parametrize("n,C", [(4, 3), (1000, 64), (0, 4)])
def test_bernoulli_beta_density_vs_fp64_oracle(lib, n, C):
    """The Bernoulli-beta family; n = 4, C = 3 is the reference's own parity case
    (device_lowering_parity.jl:150-158)."""
    if n == 4:
        z = np.array([1.0, 0.0, 1.0, 1.0], dtype=np.float32)
        q = np.array([[0.3], [-0.8], [1.5]], dtype=np.float32)
    else:
        z = (np.random.default_rng(3).random(n) < 0.3).astype(np.float32)
        q = (np.random.default_rng(4).standard_normal((C, 1)) * 2).astype(np.float32)
    ws = _ws(BernoulliBeta(), (n,), {"z": z}, C)
    t, g = ws.logjoint_gradient(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


@pytest.mark.parametrize("n,C", [(3, 3), (2000, 64)])
def test_lognormal_gamma_density_vs_fp64_oracle(lib, n, C):
    """The lognormal/gamma family; n = 3, C = 3 is the reference's parity case
    (device_lowering_parity.jl:140-148)."""
    if n == 3:
        y = np.array([0.4, 1.1, -0.7], dtype=np.float32)
        q = np.array([[0.5, 0.1], [-0.3, 0.7], [0.9, -0.2]], dtype=np.float32)
    else:
        y = (1.5 + 2.0 * np.random.default_rng(3).standard_normal(n)).astype(np.float32)
        q = (np.array([0.0, 0.4]) + 0.3 * np.random.default_rng(4).standard_normal((C, 2))).astype(np.float32)
    ws = _ws(LognormalGammaNormal(), (n,), {"y": y}, C)
    t, g = ws.logjoint_gradient(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


@pytest.mark.parametrize("n,C", [(5, 3), (3000, 64)])
def test_heavy_tail_density_vs_fp64_oracle(lib, n, C):
    """The Student-t heavy-tail family; n = 5, C = 3 is the reference's parity case
    (device_lowering_parity.jl:170-176)."""
    if n == 5:
        y = np.array([0.4, -0.7, 1.1, 0.2, 0.9], dtype=np.float32)
        q = np.array([[0.5, 0.1, -0.4], [-0.3, 0.7, 0.2], [1.2, -0.2, 0.6]], dtype=np.float32)
    else:
        y = (0.5 + np.random.default_rng(3).standard_t(5, size=n)).astype(np.float32)
        q = (np.array([0.5, -0.3, 0.0]) + 0.3 * np.random.default_rng(4).standard_normal((C, 3))).astype(np.float32)
    ws = _ws(StudentTHeavyTail(), (n,), {"y": y}, C)
    t, g = ws.logjoint_gradient(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


def test_hier_ragged_groups_with_empty_group(lib):
    J = 6
    sizes = np.array([3, 0, 9, 1, 0, 4])
    rng = np.random.default_rng(9)
    y = rng.standard_normal(sizes.sum()).astype(np.float32)
    sig = rng.uniform(0.5, 2, J).astype(np.float32)
    m = HierarchicalNormalNoncentered(J)
    q = rng.standard_normal((5, J + 2)).astype(np.float32)
    ws = _ws(m, (sig, sizes), {"y": y}, 5)
    t, g = ws.logjoint_gradient(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5 and _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


def test_glm_out_of_support_is_neg_inf(lib):
    X, y, _ = logistic_regression_data(50, 3, 2)
    y = y.copy()
    y[7] = 2.0
    m = BernoulliLogitGLM(3)
    t = _ws(m, (X,), {"y": y}, 4).logjoint(np.zeros((3, 4)))
    assert np.all(t == -np.inf)


def test_shape_errors(lib):
    X, y, _ = logistic_regression_data(50, 3, 2)
    ws = _ws(BernoulliLogitGLM(3), (X,), {"y": y}, 4)
    with pytest.raises(IndexError):
        ws.logjoint(np.zeros((2, 4)))
    with pytest.raises(IndexError):
        ws.logjoint(np.zeros((3, 5)))
    with pytest.raises(ValueError):
        from uncertaintea_b200.device import DeviceBatchedWorkspace
        DeviceBatchedWorkspace(BernoulliLogitGLM(3), 4, args=(X,), constraints={"y": y}, precision=np.float64)


# ------------------------------------------------------------- samplers -----
def _state(ws, q):
    qd = torch.from_numpy(q).cuda()
    t, g = ws.logjoint_gradient_device(qd)
    return qd, g, t


def _hmc_gpu(ws, qd, g, t, im, step, L, coord, want=False, entry="ut_hmc_iteration"):
    C, P = qd.shape
    f = lambda: torch.zeros(C, dtype=torch.float32, device="cuda")  # noqa: E731
    out = {"accept_prob": f(), "energy": f(), "energy_error": f(),
           "accepted": torch.zeros(C, dtype=torch.uint8, device="cuda"),
           "divergent": torch.zeros(C, dtype=torch.uint8, device="cuda")}
    prop = torch.zeros_like(qd) if want else None
    mom = torch.zeros_like(qd) if want else None
    imd = torch.from_numpy(im.astype(np.float32)).cuda()
    sd = torch.from_numpy(step.astype(np.float32)).cuda()
    buf = nat.HmcBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(imd), nat.ptr(sd), nat.ptr(out["accept_prob"]),
                         nat.ptr(out["energy"]), nat.ptr(out["energy_error"]), nat.ptr(out["accepted"]),
                         nat.ptr(out["divergent"]), nat.ptr(prop), nat.ptr(mom))
    nat.check(getattr(nat.load(), entry)(ws.handle, ctypes.byref(buf), L, coord, 1000.0, None))
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in out.items()}
    res["position"], res["gradient"], res["logjoint"] = qd.cpu().numpy(), g.cpu().numpy(), t.cpu().numpy()
    if want:
        res["proposal"], res["endpoint_momentum"] = prop.cpu().numpy(), mom.cpu().numpy()
    return res


def _glm_mode(X, y, sigma=1.0, iters=25):
    """Posterior mode of the logistic regression by Newton's method (float64)."""
    X = X.astype(np.float64)
    b = np.zeros(X.shape[1])
    for _ in range(iters):
        pr = 1 / (1 + np.exp(-X @ b))
        g = X.T @ (y - pr) - b / sigma ** 2
        H = -(X.T * (pr * (1 - pr))) @ X - np.eye(X.shape[1]) / sigma ** 2
        b = b - np.linalg.solve(H, g)
    return b


def _gauss_near_mode(n, C, seed, spread):
    y, _ = gauss_data(n, 3)
    r = np.random.default_rng(seed)
    q = np.empty((C, 2), dtype=np.float32)
    q[:, 0] = y.mean() + spread * r.standard_normal(C)
    q[:, 1] = np.log(y.std()) + spread * r.standard_normal(C)
    return NormalLocationScale(), (n,), {"y": y}, q


def test_chees_iteration_is_the_hmc_iteration_with_its_outputs(lib):
    """ut_chees_iteration (the reference's ChEES device iteration) is
    ut_hmc_iteration with the proposal and endpoint momentum kept: bitwise the
    same state and outputs, and it refuses buffers without them."""
    m, args, cons, q = _glm_case(1000, 10, 64, False, 2)
    q *= 0.3
    ws = _ws(m, args, cons, 64)
    im, step = np.ones(10), np.full(64, 0.05)
    a = _hmc_gpu(ws, *_state(ws, q), im, step, 7, 99, want=True)
    b = _hmc_gpu(ws, *_state(ws, q), im, step, 7, 99, want=True, entry="ut_chees_iteration")
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    with pytest.raises(Exception, match="endpoint-momentum"):
        _hmc_gpu(ws, *_state(ws, q), im, step, 7, 99, want=False, entry="ut_chees_iteration")
    ws.close()


@pytest.mark.parametrize("C,N,D,intercept,L", [(1, 50000, 20, False, 8), (4, 20000, 99, True, 8),
                                                (16, 8000, 36, False, 5), (3, 12000, 12, False, 1),
                                                # more chunks per CTA than ring stages: refills
                                                (4, 100000, 99, True, 4), (1, 100000, 100, False, 3)])
def test_stream_trajectory_in_one_launch_is_the_step_path(lib, monkeypatch, C, N, D, intercept, L):
    """Few chains on the streaming path: ut_hmc_iteration runs the L gradient
    evaluations of a trajectory, and the kicks and drifts between them, in one
    cooperative launch.  Its state and outputs equal those of one launch per
    step bit for bit (the fold keeps the streaming kernel's summation order),
    again on a second call (the grid barrier's state carries over), and the
    iteration agrees with the oracle's under the same Philox streams."""
    m, args, cons, _ = _glm_case(N, D, C, intercept, 7, 0.3)
    X = args[0]
    Xa = np.hstack([np.ones((N, 1)), X]) if intercept else X
    mode = _glm_mode(Xa, cons["y"])
    r = np.random.default_rng(8)
    P = m.num_params()
    q = (mode + 0.02 * r.standard_normal((C, P))).astype(np.float32)
    ws = _ws(m, args, cons, C)
    assert ws.kernel_path() == "stream"
    im = np.linspace(0.5, 1.5, P)
    steps = np.full(C, 0.01) * np.linspace(0.8, 1.2, C)
    monkeypatch.setenv("UT_DISABLE_STREAM_TRAJECTORY", "1")
    a = _hmc_gpu(ws, *_state(ws, q), im, steps, L, 4242, want=True)
    monkeypatch.delenv("UT_DISABLE_STREAM_TRAJECTORY")
    for _ in range(2):
        b = _hmc_gpu(ws, *_state(ws, q), im, steps, L, 4242, want=True)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    ws.check()
    om = oracle.OracleModel(ws.lowered)
    qd, g, t = _state(ws, q)
    qo, go, to = qd.cpu().numpy().copy(), g.cpu().numpy().copy(), t.cpu().numpy().copy()
    ref = om.hmc_iteration(qo, go, to, im, steps, L, 4242, want_proposal=True)
    assert np.array_equal(b["accepted"], ref["accepted"]) and not ref["divergent"].any()
    np.testing.assert_allclose(b["proposal"], ref["proposal"], rtol=1e-3, atol=1e-4)
    # the energy error is a difference of logjoints of magnitude ~1e4 here, whose
    # FP32 roundoff (~1e-3 each) shows in the accept probability
    np.testing.assert_allclose(b["accept_prob"], ref["accept_prob"], atol=1e-2)
    ws.close()


def _assert_accept_flips_are_near_ties(gpu, ref, coord):
    """Every chain whose accept decision differs between the device and the
    oracle is a near-tie: its accept uniform (Philox stream 4, draw 0 of the
    chain at this coordinate, the same on both sides; hmc_kernels.jl:553-577)
    lies between the two sides' accept probabilities, which differ only by the
    FP32 roundoff of the energy error.  A flip with the uniform elsewhere would
    mean the two sides drew different randomness or computed different
    energies."""
    live = (gpu["divergent"] == 0) & (ref["divergent"] == 0)
    for c in np.flatnonzero((gpu["accepted"] != ref["accepted"]) & live):
        u = float(oracle.rand_uniform(int(c), coord, 4, 0, 1)[0])
        lo, hi = sorted((float(gpu["accept_prob"][c]), float(ref["accept_prob"][c])))
        assert lo - 1e-6 <= u <= hi + 1e-6, (int(c), u, lo, hi)


@pytest.mark.parametrize("case", ["glm_c1", "glm_tiled", "hier", "gauss"])
def test_hmc_iteration_vs_oracle(lib, case):
    """One HMC iteration from near-posterior states with stable step sizes:
    the same Philox momenta and accept uniforms on both sides."""
    r = np.random.default_rng(3)
    if case == "glm_c1":
        m, args, cons, _ = _glm_case(1000, 10, 256, False, 1)
        mode = _glm_mode(args[0], cons["y"])
        q = (mode + 0.05 * r.standard_normal((256, 10))).astype(np.float32)
        step, L = 0.05, 8
    elif case == "glm_tiled":
        m, args, cons, q = _glm_case(4000, 48, 96, True, 5, 0.2)
        q *= 0.2
        step, L = 0.02, 5
    else:
        y, sig, sizes, _ = hierarchical_data(64, 20, 7)
        m, args, cons = HierarchicalNormalNoncentered(64), (sig, sizes), {"y": y}
        # near the posterior mode: theta_j at the group means, z_j = (ybar_j - mu) / tau
        starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        ybar = np.array([y[s:s + n].mean() for s, n in zip(starts, sizes)])
        mu0, tau0 = ybar.mean(), ybar.std()
        q = np.empty((256, 66), dtype=np.float32)
        q[:, 0] = mu0 + 0.1 * r.standard_normal(256)
        q[:, 1] = np.log(tau0) + 0.02 * r.standard_normal(256)
        q[:, 2:] = (ybar - mu0) / tau0 + 0.02 * r.standard_normal((256, 64))
        step, L = 0.004, 6
    if case == "gauss":
        m, args, cons, q = _gauss_near_mode(200, 256, 3, 0.05)
        step, L = 0.05, 8
    C, P = q.shape
    ws = _ws(m, args, cons, C)
    qd, g, t = _state(ws, q)
    om = oracle.OracleModel(ws.lowered)
    im = np.linspace(0.5, 1.5, P)
    steps = np.full(C, step) * np.linspace(0.8, 1.2, C)
    qo, go, to = qd.cpu().numpy().copy(), g.cpu().numpy().copy(), t.cpu().numpy().copy()
    gpu = _hmc_gpu(ws, qd, g, t, im, steps, L, 12345, want=True)
    ref = om.hmc_iteration(qo, go, to, im, steps, L, 12345, want_proposal=True)
    same = (gpu["accepted"] == ref["accepted"]) & (gpu["divergent"] == ref["divergent"])
    assert same.mean() >= 0.98
    _assert_accept_flips_are_near_ties(gpu, ref, 12345)
    assert ref["divergent"].mean() <= 0.02
    ok = same & (ref["divergent"] == 0)
    np.testing.assert_allclose(gpu["proposal"][ok], ref["proposal"][ok], rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(gpu["endpoint_momentum"][ok], ref["endpoint_momentum"][ok], rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(gpu["position"][same], qo[same], rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(gpu["accept_prob"][ok], ref["accept_prob"][ok], atol=2e-3)
    np.testing.assert_allclose(gpu["energy_error"][ok], ref["energy_error"][ok], rtol=1e-3, atol=5e-3)
    ws.close()


def test_leapfrog_probe_vs_oracle(lib):
    m, args, cons, _ = _glm_case(1000, 10, 64, False, 2)
    mode = _glm_mode(args[0], cons["y"])
    q = (mode + 0.05 * np.random.default_rng(1).standard_normal((64, 10))).astype(np.float32)
    ws = _ws(m, args, cons, 64)
    qd, g, t = _state(ws, q)
    im = np.ones(10, dtype=np.float32)
    trial = np.geomspace(1e-3, 0.1, 64).astype(np.float32)
    imd = torch.from_numpy(im).cuda()          # kept alive until the kernel has run
    trd = torch.from_numpy(trial).cuda()
    out = torch.empty(64, dtype=torch.float32, device="cuda")
    nat.check(nat.load().ut_leapfrog_probe(ws.handle, nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(imd),
                                           nat.ptr(trd), 777, nat.ptr(out), None))
    torch.cuda.synchronize()
    ref = oracle.OracleModel(ws.lowered).leapfrog_probe(qd.cpu().numpy(), g.cpu().numpy(), t.cpu().numpy(), im, trial,
                                                        777)
    gpu = out.cpu().numpy()
    assert np.all(np.isfinite(ref)) and np.all(np.isfinite(gpu))
    # H ~ |logjoint| ~ 6e2: FP32 rounding of H0 - H1 is ~1e-4 absolute
    np.testing.assert_allclose(gpu, ref, rtol=1e-3, atol=5e-4)
    ws.close()


def _nuts_gpu(ws, qd, g, t, im, step, depth, coord):
    C = qd.shape[0]
    f = lambda dt=torch.float32: torch.zeros(C, dtype=dt, device="cuda")  # noqa: E731
    o = {"accept_prob": f(), "energy": f(), "energy_error": f(), "tree_depth": f(torch.int32),
         "integration_steps": f(torch.int32), "divergent": f(torch.uint8), "moved": f(torch.uint8)}
    imd = torch.from_numpy(im.astype(np.float32)).cuda()
    sd = torch.from_numpy(step.astype(np.float32)).cuda()
    buf = nat.NutsBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(imd), nat.ptr(sd), nat.ptr(o["accept_prob"]),
                          nat.ptr(o["energy"]), nat.ptr(o["energy_error"]), nat.ptr(o["tree_depth"]),
                          nat.ptr(o["integration_steps"]), nat.ptr(o["divergent"]), nat.ptr(o["moved"]))
    nat.check(nat.load().ut_persistent_nuts_iteration(ws.handle, ctypes.byref(buf), depth, 1000.0, coord, None))
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in o.items()}
    res["position"], res["gradient"], res["logjoint"] = qd.cpu().numpy(), g.cpu().numpy(), t.cpu().numpy()
    return res


def test_bernoulli_beta_float32_logit_cliff(lib):
    """The reference's device Float32 logit cliff (device_float32_saturation.jl,
    "device_f32_logit_cliff"; p ~ beta(2, 2), y = 1): -Inf with a finite
    gradient where float32 p rounds to 1 (logit 18, 20, 30), finite and within
    4 eps(f32) e^theta + 1e-5 of float64 at 13, 15, 16, within 1e-5 at -1.5, 0.3, 2."""
    m = BernoulliBeta(alpha=2.0, beta=2.0)
    q = np.array([[18.0], [20.0], [30.0], [13.0], [15.0], [16.0], [-1.5], [0.3], [2.0]], dtype=np.float32)
    ws = _ws(m, (1,), {"z": np.array([1.0])}, len(q))
    t, g = ws.logjoint_gradient(q.T)
    g = np.asarray(g.T)[:, 0]
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert np.all(t[:3] == -np.inf) and not np.any(np.isnan(g[:3]))
    tol = 4 * np.finfo(np.float32).eps * np.exp(q[3:6, 0].astype(np.float64)) + 1e-5
    assert np.all(np.isfinite(t[3:6])) and np.all(np.abs(t[3:6] - t64[3:6]) <= tol)
    assert np.all(np.abs(g[3:6] - g64[3:6, 0]) <= tol)
    assert np.all(np.abs(t[6:] - t64[6:]) <= 1e-5) and np.all(np.abs(g[6:] - g64[6:, 0]) <= 1e-5)
    ws.close()


@pytest.mark.parametrize("n,C", [(1, 4), (500, 100), (0, 8)])
def test_known_scale_density_vs_fp64_oracle(lib, n, C):
    """The normal known-scale family (the reference's conjugate gate model,
    device_persistent_nuts.jl:33-38: y = 0.3 with n = 1), an empty loop, and a
    larger one with another prior and scale."""
    if n == 1:
        m, y = NormalKnownScale(), np.array([0.3], dtype=np.float32)
    else:
        m, y = NormalKnownScale(mu_loc=0.5, mu_scale=2.0, sigma=0.7), gauss_data(n, 4)[0] if n else np.zeros(0)
    q = (np.random.default_rng(6).standard_normal((C, 1)) * 1.5).astype(np.float32)
    ws = _ws(m, (n,), {"y": y}, C)
    assert ws.kernel_path() == "warp"
    t, g = ws.logjoint_gradient(q.T)
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t, t64) <= 1e-5
    assert _grad_ok(np.asarray(g.T), g64, mag)
    ws.close()


@pytest.mark.parametrize("case", ["hier", "glm", "gauss", "bern", "ht", "nks"])
def test_persistent_nuts_iteration_vs_oracle(lib, case):
    if case == "nks":
        m, args, cons = NormalKnownScale(), (1,), {"y": np.array([0.3])}
        q = (0.15 + 0.7 * np.random.default_rng(4).standard_normal((128, 1))).astype(np.float32)
        step = 0.5
    elif case == "ht":
        y = (0.5 + np.random.default_rng(3).standard_t(5, size=200)).astype(np.float32)
        m, args, cons = StudentTHeavyTail(), (200,), {"y": y}
        q = (np.array([0.5, -0.3, 0.0]) + 0.2 * np.random.default_rng(6).standard_normal((128, 3))).astype(np.float32)
        step = 0.1
    elif case == "bern":
        z = (np.random.default_rng(3).random(300) < 0.3).astype(np.float32)
        m, args, cons = BernoulliBeta(), (300,), {"z": z}
        q = (np.log(0.3 / 0.7) + 0.2 * np.random.default_rng(5).standard_normal((128, 1))).astype(np.float32)
        step = 0.3
    elif case == "gauss":
        m, args, cons, q = _gauss_near_mode(200, 128, 8, 0.1)
        step = 0.1
    elif case == "hier":
        y, sig, sizes, _ = hierarchical_data(64, 20, 7)
        m, args, cons = HierarchicalNormalNoncentered(64), (sig, sizes), {"y": y}
        q = (np.random.default_rng(8).standard_normal((128, 66)) * 0.5).astype(np.float32)
        step = 0.05
    else:
        m, args, cons, q = _glm_case(1000, 10, 128, False, 1)
        q *= 0.3
        step = 0.08
    C, P = q.shape
    ws = _ws(m, args, cons, C)
    qd, g, t = _state(ws, q)
    im = np.ones(P)
    steps = np.full(C, step)
    qo, go, to = qd.cpu().numpy().copy(), g.cpu().numpy().copy(), t.cpu().numpy().copy()
    gpu = _nuts_gpu(ws, qd, g, t, im, steps, 10, 4242)
    ref = om_out = oracle.OracleModel(ws.lowered).nuts_iteration(qo, go, to, im, steps, 10, 4242)
    same = ((gpu["tree_depth"] == ref["tree_depth"]) & (gpu["integration_steps"] == ref["integration_steps"])
            & (gpu["moved"] == ref["moved"]) & (gpu["divergent"] == ref["divergent"]))
    assert same.mean() >= 0.95, same.mean()
    np.testing.assert_allclose(gpu["position"][same], qo[same], rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(gpu["accept_prob"][same], om_out["accept_prob"][same], atol=1e-3)
    assert np.all(gpu["tree_depth"] >= 1) and np.all(gpu["tree_depth"] <= 10)
    ws.close()


@pytest.mark.parametrize("case", ["glm", "gauss", "glm_tc"])
def test_advi_step_vs_oracle(lib, case):
    """One device ADVI step (Philox particles, batched gradient, particle means)
    against the oracle's restatement with the same noise coordinates."""
    if case == "glm_tc":
        m, args, cons, _ = _glm_case(3000, 100, 128, False, 5, 0.1)
        loc = (0.1 * np.random.default_rng(2).standard_normal(100)).astype(np.float32)
        sc = np.full(100, 0.05, dtype=np.float32)
    elif case == "glm":
        m, args, cons, _ = _glm_case(1000, 10, 64, False, 1)
        loc = (0.3 * np.random.default_rng(2).standard_normal(10)).astype(np.float32)
        sc = np.full(10, 0.1, dtype=np.float32)
    else:
        y, _ = gauss_data(200, 3)
        m, args, cons = NormalLocationScale(), (200,), {"y": y}
        loc = np.array([y.mean(), np.log(y.std())], dtype=np.float32)
        sc = np.array([0.1, 0.05], dtype=np.float32)
    M = 128 if case == "glm_tc" else 64
    ws = _ws(m, args, cons, M)
    if case == "glm_tc":
        assert ws.kernel_path() == "tensor_core"
    P = loc.size
    f = lambda *sh: torch.empty(sh, dtype=torch.float32, device="cuda")  # noqa: E731
    loc_d, sc_d = torch.from_numpy(loc).cuda(), torch.from_numpy(sc).cuda()
    parts, vals, grads, lg, sg = f(M, P), f(M), f(M, P), f(P), f(P)
    for coord in (5, 6):   # two calls in a row, different noise
        nat.check(lib.ut_advi_step(ws.handle, nat.ptr(loc_d), nat.ptr(sc_d), coord, nat.ptr(parts), nat.ptr(vals),
                                   nat.ptr(grads), nat.ptr(lg), nat.ptr(sg), None))
        torch.cuda.synchronize()
        ref = oracle.OracleModel(ws.lowered).advi_step(loc, sc, M, coord)
        np.testing.assert_allclose(parts.cpu().numpy(), ref["particles"], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(vals.cpu().numpy(), ref["values"], rtol=1e-5)
        scale = max(np.abs(ref["location_gradient"]).max(), 1.0)
        np.testing.assert_allclose(lg.cpu().numpy(), ref["location_gradient"], atol=1e-4 * scale)
        scale = max(np.abs(ref["scale_gradient"]).max(), 1.0)
        np.testing.assert_allclose(sg.cpu().numpy(), ref["scale_gradient"], atol=1e-4 * scale)
    ws.close()


@pytest.mark.parametrize("case", ["glm", "gauss", "hier", "glm_tc"])
def test_meads_iterations_vs_oracle(lib, case):
    """Two MEADS iterations (fold statistics in double, refresh, one leapfrog
    step, persistent-slice accept) against the oracle's literal restatement,
    from the same state and Philox coordinates; glm_tc runs the gradient on the
    tensor-core kernel."""
    if case == "glm_tc":
        m, args, cons, q = _glm_case(3000, 100, 64, False, 5, 0.1)
        q *= 0.1
    elif case == "glm":
        m, args, cons, q = _glm_case(1000, 10, 64, False, 1)
        q *= 0.3
    elif case == "gauss":
        m, args, cons, q = _gauss_near_mode(200, 64, 4, 0.2)
    else:
        y, sig, sizes, _ = hierarchical_data(16, 10, 7)
        m, args, cons = HierarchicalNormalNoncentered(16), (sig, sizes), {"y": y}
        q = (np.random.default_rng(8).standard_normal((64, 18)) * 0.5).astype(np.float32)
    C, P, K = q.shape[0], q.shape[1], 4
    ws = _ws(m, args, cons, C)
    if case == "glm_tc":
        assert ws.kernel_path() == "tensor_core"
    qd, g, t = _state(ws, q)
    f = lambda sh, dt=torch.float32: torch.zeros(sh, dtype=dt, device="cuda")  # noqa: E731
    mom, sl = f((C, P)), f(C)
    out = {"accept_prob": f(C), "energy": f(C), "energy_error": f(C), "accepted": f(C, torch.uint8),
           "divergent": f(C, torch.uint8), "integration_steps": f(C, torch.int32), "fold_parameters": f((K, 4))}
    buf = nat.MeadsBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(mom), nat.ptr(sl),
                           *[nat.ptr(out[k]) for k in ("accept_prob", "energy", "energy_error", "accepted",
                                                       "divergent", "integration_steps", "fold_parameters")])
    nat.check(lib.ut_meads_init(ws.handle, ctypes.byref(buf), 3, None))
    torch.cuda.synchronize()
    state = {"position": qd.cpu().numpy(), "gradient": g.cpu().numpy(), "logjoint": t.cpu().numpy(),
             "momentum": mom.cpu().numpy(), "slice": sl.cpu().numpy()}
    assert np.all(np.abs(state["slice"]) <= 1.0)
    om = oracle.OracleModel(ws.lowered)
    for it in (1, 2):
        ref = om.meads_iteration(state["position"], state["gradient"], state["logjoint"], state["momentum"],
                                 state["slice"], K, it, 100 + it)
        nat.check(lib.ut_meads_iteration(ws.handle, ctypes.byref(buf), K, it, 1000.0, 100 + it, None))
        torch.cuda.synchronize()
        np.testing.assert_allclose(out["fold_parameters"].cpu().numpy(), ref["fold_parameters"], rtol=2e-5, atol=1e-7)
        same = (out["accepted"].cpu().numpy() == ref["accepted"]) & (out["divergent"].cpu().numpy() == ref["divergent"])
        assert same.mean() >= 0.95, same.mean()
        assert np.array_equal(out["integration_steps"].cpu().numpy(), ref["integration_steps"])
        pos = qd.cpu().numpy()
        np.testing.assert_allclose(pos[same], ref["position"][same], rtol=1e-4, atol=1e-4)
        np.testing.assert_allclose(mom.cpu().numpy()[same], ref["momentum"][same], rtol=1e-3, atol=1e-3)
        np.testing.assert_allclose(out["accept_prob"].cpu().numpy()[same], ref["accept_prob"][same], atol=1e-3)
        # carry the device state forward for the next iteration
        state = {"position": pos, "gradient": g.cpu().numpy(), "logjoint": t.cpu().numpy(),
                 "momentum": mom.cpu().numpy(), "slice": sl.cpu().numpy()}
    ws.close()


def test_chees_reduce_vs_oracle(lib):
    C, P = 1000, 37
    r = np.random.default_rng(5)
    ini = r.standard_normal((C, P)).astype(np.float32)
    prop = (ini + 0.3 * r.standard_normal((C, P))).astype(np.float32)
    mom = r.standard_normal((C, P)).astype(np.float32)
    ap = r.uniform(size=C).astype(np.float32)
    div = (r.uniform(size=C) < 0.05).astype(np.uint8)
    prop[3, 5] = np.nan
    im = r.uniform(0.5, 2, P).astype(np.float32)
    m, args, cons, _ = _glm_case(100, P, C, False, 1)
    ws = _ws(m, args, cons, C)
    out = (ctypes.c_double * 2)()
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    tens = [T(ini), T(prop), T(mom), T(ap), T(div), T(im)]
    nat.check(nat.load().ut_chees_reduce(ws.handle, *[nat.ptr(x) for x in tens], out, None))
    ref = oracle.chees_reduce(ini, prop, mom, ap, div, im)
    assert out[0] == pytest.approx(ref[0], rel=1e-9)
    assert out[1] == pytest.approx(ref[1], rel=1e-12)
    ws.close()


def test_running_variance_vs_sequential(lib):
    from uncertaintea_b200.inference import DeviceRunningVariance, _RUNNING_VARIANCE_FLOOR
    C, P, WL = 300, 17, 75
    r = np.random.default_rng(6)
    pos = (r.standard_normal((C, P)) * np.linspace(0.1, 3, P)).astype(np.float32)
    pos[10] *= 50  # a far outlier column exercises the clip
    w = np.where(r.uniform(size=C) < 0.1, 0.0, r.uniform(0.2, 1.0, size=C))
    rv = DeviceRunningVariance(nat.load(), P, WL, torch.device("cuda"))
    rv.update(torch.from_numpy(pos).cuda(), w)
    mean, m2, count, ws_, wss = rv.host_state()
    # sequential restatement of adaptation.jl:83-101, 170-191
    mu, M2, n, S, SS = np.zeros(P), np.zeros(P), 0, 0.0, 0.0
    for c in range(C):
        if w[c] == 0:
            continue
        x = pos[c].astype(np.float64)
        if n >= 4:
            prog = min(max(n - 4, 0) / (WL - 4), 1.0)
            scale = 8.0 if n <= 4 else 8.0 + (5.0 - 8.0) * prog
            bound = scale * np.sqrt(np.maximum(M2 / max(n - 1, 1), _RUNNING_VARIANCE_FLOOR))
            x = mu + np.clip(x - mu, -bound, bound)
        n += 1
        S2 = S + w[c]
        d = x - mu
        mu = mu + (w[c] / S2) * d
        M2 = M2 + w[c] * d * (x - mu)
        S, SS = S2, SS + w[c] ** 2
    np.testing.assert_allclose(mean, mu, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(m2, M2, rtol=1e-12, atol=1e-12)
    assert count == n == rv.count
    assert ws_ == pytest.approx(S, rel=1e-14) and wss == pytest.approx(SS, rel=1e-14)


@pytest.mark.parametrize("N,D,C,intercept", [
    (100000, 100, 4096, False),   # full-size design, 4096 chains
    (5003, 100, 200, True),       # ragged obs tile and chain tile, F=101 -> 104 padded features
    (777, 64, 128, False),
    (70, 3, 5, True),             # tiny: one observation tile, one partial chain tile
])
def test_tensor_core_path_vs_cuda_core_and_oracle(lib, N, D, C, intercept, monkeypatch):
    """The tcgen05 3xTF32 kernel against the CUDA-core tiled kernel and the FP64
    oracle (same tolerances as the other density tests)."""
    m, args, cons, q = _glm_case(N, D, C, intercept, 21, 1.0 / np.sqrt(D))
    ws_tc = _ws(m, args, cons, C)
    assert ws_tc.kernel_path() in ("tensor_core", "warp")
    monkeypatch.setenv("UT_DISABLE_TENSOR_CORES", "1")
    ws_cc = _ws(m, args, cons, C)
    monkeypatch.delenv("UT_DISABLE_TENSOR_CORES")
    qd = torch.from_numpy(q).cuda()
    t1, g1 = ws_tc.logjoint_gradient_device(qd)
    t0 = ws_tc.logjoint_device(qd)
    ws_tc.check()
    t2, g2 = ws_cc.logjoint_gradient_device(qd)
    torch.cuda.synchronize()
    t1, g1, t0, t2, g2 = (x.cpu().numpy() for x in (t1, g1, t0, t2, g2))
    idx = np.unique(np.linspace(0, C - 1, min(C, 16)).astype(int))
    t64, g64, mag = _ref(oracle.OracleModel(ws_tc.lowered), q[idx].astype(np.float64))
    assert _lj_err(t1[idx], t64) <= 1e-5 and _grad_ok(g1[idx], g64, mag)
    assert _lj_err(t0[idx], t64) <= 1e-5
    assert _lj_err(t2[idx], t64) <= 1e-5 and _grad_ok(g2[idx], g64, mag)
    assert _lj_err(t1, t2.astype(np.float64)) <= 2e-5
    ws_tc.close()
    ws_cc.close()


@pytest.mark.parametrize("N,D,C,intercept", [
    (100000, 100, 1, False),      # 100000x100 design, one chain
    (100000, 100, 16, False),     # 100000x100 design, 16 chains
    (5003, 99, 8, True),          # F = 100, ragged last chunk (5003 = 78 x 64 + 11)
    (1000, 63, 3, True),          # F = 64, chains padded to 4
    (130, 35, 5, True),           # F = 36, three chunks
])
def test_streaming_path_vs_oracle_and_tiled(lib, N, D, C, intercept, monkeypatch):
    """The HBM-streaming kernel for a few chains against the FP64 oracle (same
    tolerances as the other density tests) and the CUDA-core tiled kernel."""
    m, args, cons, q = _glm_case(N, D, C, intercept, 33, 1.0 / np.sqrt(D))
    ws = _ws(m, args, cons, C)
    assert ws.kernel_path() == "stream"
    monkeypatch.setenv("UT_DISABLE_STREAM_KERNEL", "1")
    ws_t = _ws(m, args, cons, C)
    monkeypatch.delenv("UT_DISABLE_STREAM_KERNEL")
    assert ws_t.kernel_path() != "stream"
    qd = torch.from_numpy(q).cuda()
    t1, g1 = ws.logjoint_gradient_device(qd)
    t0 = ws.logjoint_device(qd)
    t1b, g1b = ws.logjoint_gradient_device(qd)  # the fold's tickets were reset: same bits again
    t2, g2 = ws_t.logjoint_gradient_device(qd)
    torch.cuda.synchronize()
    ws.check()
    t1, g1, t0, t2, g2 = (x.cpu().numpy() for x in (t1, g1, t0, t2, g2))
    assert np.array_equal(t1, t1b.cpu().numpy()) and np.array_equal(g1, g1b.cpu().numpy())
    t64, g64, mag = _ref(oracle.OracleModel(ws.lowered), q.astype(np.float64))
    assert _lj_err(t1, t64) <= 1e-5 and _lj_err(t0, t64) <= 1e-5
    assert _grad_ok(g1, g64, mag)
    np.testing.assert_allclose(t1, t2, rtol=2e-6)
    np.testing.assert_allclose(g1, g2, rtol=1e-4, atol=1e-4 * np.abs(g64).max())
    ws.close()
    ws_t.close()


def test_streaming_path_needs_feature_count_multiple_of_four(lib):
    m, args, cons, q = _glm_case(2000, 101, 4, False, 34, 0.1)
    ws = _ws(m, args, cons, 4)
    assert ws.kernel_path() != "stream"
    ws.close()



def _nuts_call(fn, ws, qd, g, t, im, step, depth, coord):
    C = qd.shape[0]
    f = lambda dt=torch.float32: torch.zeros(C, dtype=dt, device="cuda")  # noqa: E731
    o = {"accept_prob": f(), "energy": f(), "energy_error": f(), "tree_depth": f(torch.int32),
         "integration_steps": f(torch.int32), "divergent": f(torch.uint8), "moved": f(torch.uint8)}
    imd = torch.from_numpy(im.astype(np.float32)).cuda()
    sd = torch.from_numpy(step.astype(np.float32)).cuda()
    buf = nat.NutsBuffers(nat.ptr(qd), nat.ptr(g), nat.ptr(t), nat.ptr(imd), nat.ptr(sd), nat.ptr(o["accept_prob"]),
                          nat.ptr(o["energy"]), nat.ptr(o["energy_error"]), nat.ptr(o["tree_depth"]),
                          nat.ptr(o["integration_steps"]), nat.ptr(o["divergent"]), nat.ptr(o["moved"]))
    nat.check(fn(ws.handle, ctypes.byref(buf), depth, 1000.0, coord, None))
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in o.items()}
    res["position"], res["gradient"], res["logjoint"] = qd.cpu().numpy(), g.cpu().numpy(), t.cpu().numpy()
    return res


@pytest.mark.parametrize("case", ["glm", "hier", "gauss"])
def test_lockstep_nuts_matches_persistent_bitwise(lib, case):
    """Where both strategies apply (a per-chain evaluator), the lockstep tree and
    the persistent tree are the same computation: identical states and outputs."""
    if case == "gauss":
        m, args, cons, q = _gauss_near_mode(200, 64, 9, 0.3)
        step = 0.1
    elif case == "glm":
        m, args, cons, q = _glm_case(1000, 10, 96, False, 1)
        q *= 0.3
        step = 0.08
    else:
        y, sig, sizes, _ = hierarchical_data(64, 20, 7)
        m, args, cons = HierarchicalNormalNoncentered(64), (sig, sizes), {"y": y}
        q = (np.random.default_rng(8).standard_normal((64, 66)) * 0.5).astype(np.float32)
        step = 0.05
    C, P = q.shape
    ws = _ws(m, args, cons, C)
    im, steps = np.linspace(0.7, 1.3, P), np.full(C, step) * np.linspace(0.9, 1.1, C)
    outs = []
    for fn in (lib.ut_persistent_nuts_iteration, lib.ut_lockstep_nuts_iteration):
        qd, g, t = _state(ws, q)
        outs.append(_nuts_call(fn, ws, qd, g, t, im, steps, 8, 515))
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k
    assert outs[0]["tree_depth"].max() >= 3
    ws.close()


def test_lockstep_nuts_on_tensor_core_path_vs_oracle(lib):
    """Lockstep NUTS over the tensor-core batched gradient against the oracle's
    NUTS (same Philox streams); the gradients differ in the last bits, so the
    trees agree for most chains."""
    m, args, cons, q = _glm_case(20000, 100, 128, False, 7, 0.1)
    X, y = args[0], cons["y"]
    mode = _glm_mode(X, y)
    q = (mode + 0.02 * np.random.default_rng(9).standard_normal((128, 100))).astype(np.float32)
    ws = _ws(m, args, cons, 128)
    assert ws.kernel_path() == "tensor_core"
    qd, g, t = _state(ws, q)
    qo, go, to = qd.cpu().numpy().copy(), g.cpu().numpy().copy(), t.cpu().numpy().copy()
    im, steps = np.ones(100), np.full(128, 0.02)
    gpu = _nuts_call(lib.ut_lockstep_nuts_iteration, ws, qd, g, t, im, steps, 6, 77)
    ref = oracle.OracleModel(ws.lowered).nuts_iteration(qo, go, to, im, steps, 6, 77)
    same = (gpu["tree_depth"] == ref["tree_depth"]) & (gpu["integration_steps"] == ref["integration_steps"]) & \
        (gpu["moved"] == ref["moved"])
    assert same.mean() >= 0.9, same.mean()
    np.testing.assert_allclose(gpu["position"][same], qo[same], rtol=1e-3, atol=1e-3)
    ws.close()
