"""CPU tests of the C-ABI library: it loads, exports every symbol the header
declares, and its pure host-side validation answers without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "ut_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|const char\*)\s+(ut_[a-z0-9_]+)\s*\(", text, re.M)))


def test_header_declarations_match_binding(lib):
    from uncertaintea_b200 import _native
    assert declared_symbols() == sorted(_native.exported_symbols())


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "uncertaintea_b200", "libut_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\s[TW]\s+(ut_[a-z0-9_]+)$", out, re.M))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(lib, s)


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "ut_b200.h"\nint main(void){ ut_plan_desc p; (void)p; return 0; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c", str(src),
                    "-o", str(tmp_path / "t.o")], check=True)


def test_plain_c_host_binds_the_library(tmp_path, lib):
    """A C program bound through include/ut_b200.h alone (tests/c_host/c_caller.c)
    links the shared library and holds the boundary's contract from C: lowering
    report, validation, errors, the no-device path (and, with a device, a closed
    form logjoint and gradient)."""
    exe = tmp_path / "c_caller"
    libdir = os.path.join(ROOT, "uncertaintea_b200")
    subprocess.run(["gcc", "-std=gnu11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_host", "c_caller.c"), "-L", libdir, "-lut_b200",
                    f"-Wl,-rpath,{libdir}", "-lm", "-o", str(exe)], check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr
    assert "all checks passed" in run.stdout


JULIA_EXT = os.path.join(ROOT, "julia", "UncertainTeaB200Ext.jl")


def _julia_struct(text, name):
    body = text[text.index(f"struct {name}"):]
    body = body[body.index("\n") + 1:body.index("\nend")]
    fields = []
    for line in body.splitlines():
        line = line.split("#")[0]
        fields += re.findall(r"([a-z_]+)::([A-Za-z0-9_{}, ]+?)(?:;|$)", line.strip())
    return [(n, t.strip()) for n, t in fields]


def test_julia_shim_struct_matches_the_c_struct():
    """The Julia mirror of ut_plan_desc (julia/UncertainTeaB200Ext.jl) has the C
    struct's fields in the same order with the same widths (a ccall passes it
    by reference, so any drift would shift every later field)."""
    import ctypes as ct
    from uncertaintea_b200 import _native as nat
    fields = _julia_struct(open(JULIA_EXT).read(), "UtPlanDesc")
    widths = {"Int32": ct.c_int32, "Float64": ct.c_double}
    assert [(n, widths[t]) for n, t in fields] == [(n, t) for n, t in nat.PlanDesc._fields_]
    header = open(HEADER).read()
    c_body = header[header.index("typedef struct ut_plan_desc"):header.index("} ut_plan_desc;")]
    c_fields = re.findall(r"(int32_t|double)\s+([a-z_]+);", c_body)
    assert [n for _, n in c_fields] == [n for n, _ in nat.PlanDesc._fields_]


def test_julia_program_mirrors_and_code_tables_match_the_header():
    """The Julia mirrors of ut_program_step / ut_expr_node and its tables of
    distribution and expression codes agree with include/ut_b200.h and the
    Python binding."""
    from uncertaintea_b200 import _native as nat
    text = open(JULIA_EXT).read()
    header = open(HEADER).read()
    for c_name, jl, py in [("ut_program_step", "UtProgramStep", nat.ProgramStep),
                           ("ut_expr_node", "UtExprNode", nat.ExprNode)]:
        body = header[header.index(f"typedef struct {c_name} {{"):header.index(f"}} {c_name};")]
        c_fields = re.findall(r"^\s*(?:int32_t|double)\s+([a-z_]+)(?:\[\d+\])?;", body, re.M)
        jl_fields = [n for n, _ in _julia_struct(text, jl)]
        assert jl_fields == c_fields == [n for n, _ in py._fields_], (c_name, jl_fields, c_fields)
    codes = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"#define UT_DIST_([A-Z_]+)\s+(\d+)", header)}
    jl_dists = {m.group(1): int(m.group(2)) for m in re.finditer(r":Device(\w+)ChoiceStep => \(Int32\((\d+)\)", text)}
    names = {"Normal": "normal", "Lognormal": "lognormal", "Exponential": "exponential", "Gamma": "gamma",
             "Laplace": "laplace", "Cauchy": "cauchy", "HalfNormal": "halfnormal", "HalfCauchy": "halfcauchy",
             "Logistic": "logistic", "Gumbel": "gumbel", "Frechet": "frechet", "Rayleigh": "rayleigh",
             "InverseGaussian": "inversegaussian", "Beta": "beta", "StudentT": "studentt",
             "InverseGamma": "inversegamma", "Weibull": "weibull", "Bernoulli": "bernoulli",
             "BernoulliLogit": "bernoulli_logit", "Poisson": "poisson", "Geometric": "geometric",
             "NegativeBinomial": "negative_binomial", "Binomial": "binomial"}
    assert len(jl_dists) == 23
    for jl_name, code in jl_dists.items():
        assert codes[names[jl_name]] == code == nat.DISTRIBUTIONS[names[jl_name].replace("_", "")], jl_name
    ops = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"#define UT_EXPR_([A-Z0-9]+)\s+(\d+)", header)}
    jl_ops = {m.group(1): int(m.group(2)) for m in re.finditer(r":(\S+?) => (\d+)", text[text.index("const EXPR_OPS"):])}
    sym = {"+": "add", "-": "sub", "*": "mul", "/": "div", "^": "pow"}
    for op, code in jl_ops.items():
        assert ops[sym.get(op, op)] == code, op


def _header_struct_fields(name):
    header = open(HEADER).read()
    body = header[header.index(f"typedef struct {name} {{"):header.index(f"}} {name};")]
    return re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*([a-z_]+);", body, re.M)


def test_buffer_struct_mirrors_match_the_header():
    """The Python (ctypes) and Julia (julia/UncertainTeaB200Ext.jl) mirrors of
    the sampler buffer structs list the header's fields in its order."""
    from uncertaintea_b200 import _native as nat
    text = open(JULIA_EXT).read()
    for c_name, py, jl in [("ut_hmc_buffers", nat.HmcBuffers, "UtHmcBuffers"),
                           ("ut_nuts_buffers", nat.NutsBuffers, "UtNutsBuffers"),
                           ("ut_meads_buffers", nat.MeadsBuffers, "UtMeadsBuffers"),
                           ("ut_multi_view", nat.MultiView, None)]:
        fields = _header_struct_fields(c_name)
        assert fields and fields == [n for n, _ in py._fields_], c_name
        if jl:
            body = text[text.index(f"struct {jl}"):]
            body = body[body.index("\n") + 1:body.index("\nend")]
            jl_fields = [n for line in body.splitlines() for n in re.findall(r"([a-z_]+)::", line.split("#")[0])]
            assert jl_fields == fields, jl


def test_version_and_last_error(lib):
    assert b"sm_100a" in lib.ut_version()
    buf = ctypes.create_string_buffer(64)
    lib.ut_last_error(buf, len(buf))


def test_last_error_is_per_thread_and_truncates(lib):
    """ut_last_error copies this thread's message, truncated and NUL-terminated
    to the buffer, and returns its full length; another thread's failure does
    not overwrite it (the header's contract)."""
    import threading
    from uncertaintea_b200 import _native as nat
    assert lib.ut_workspace_info(None, None, None) == nat.UT_ERR_ARGUMENT
    full = nat.last_error()
    assert "null workspace handle" in full
    small = ctypes.create_string_buffer(5)
    assert lib.ut_last_error(small, 5) == len(full) and small.value == full[:4].encode()
    assert lib.ut_last_error(None, 0) == len(full)
    seen = {}

    def other():
        seen["before"] = nat.last_error()
        lib.ut_chees_reduce(None, None, None, None, None, None, None, None, None)
        seen["after"] = nat.last_error()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen["before"] == "" and "null workspace handle" in seen["after"]
    assert nat.last_error() == full


def test_lowering_report_flags_bad_descriptions(lib):
    from uncertaintea_b200 import _native as nat
    bad = nat.PlanDesc(family=99)
    buf = ctypes.create_string_buffer(1024)
    assert lib.ut_lowering_report(ctypes.byref(bad), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"unsupported kernel-description family 99" in buf.value
    glm = nat.PlanDesc(family=nat.UT_FAMILY_GLM_BERNOULLI_LOGIT, num_params=4, num_obs=10, num_coefs=3,
                       has_intercept=0, coef_sigma=1.0)
    assert lib.ut_lowering_report(ctypes.byref(glm), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"num_params must equal" in buf.value
    glm.num_params = 3
    assert lib.ut_lowering_report(ctypes.byref(glm), buf, len(buf)) == nat.UT_OK
    hier = nat.PlanDesc(family=nat.UT_FAMILY_HIER_NORMAL_NONCENTERED, num_params=66, num_obs=10, num_groups=64,
                        mu_scale=5.0, tau_scale=-1.0)
    assert lib.ut_lowering_report(ctypes.byref(hier), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"tau prior scale" in buf.value
    # one past the largest supported sizes
    wide = nat.PlanDesc(family=nat.UT_FAMILY_GLM_BERNOULLI_LOGIT, num_params=257, num_obs=10, num_coefs=257,
                        has_intercept=0, coef_sigma=1.0)
    assert lib.ut_lowering_report(ctypes.byref(wide), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"more than 256" in buf.value
    wide.num_params = wide.num_coefs = 256
    assert lib.ut_lowering_report(ctypes.byref(wide), buf, len(buf)) == nat.UT_OK
    big = nat.PlanDesc(family=nat.UT_FAMILY_HIER_NORMAL_NONCENTERED, num_params=545, num_obs=10, num_groups=543,
                       mu_scale=5.0, tau_scale=2.5)
    assert lib.ut_lowering_report(ctypes.byref(big), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"more than 544" in buf.value
    big.num_params, big.num_groups = 544, 542
    assert lib.ut_lowering_report(ctypes.byref(big), buf, len(buf)) == nat.UT_OK
    gauss = nat.PlanDesc(family=nat.UT_FAMILY_NORMAL_LOCATION_SCALE, num_params=2, num_obs=5, mu_scale=1.0,
                         scale_shape=2.0, scale_rate=1.0)
    assert lib.ut_lowering_report(ctypes.byref(gauss), buf, len(buf)) == nat.UT_OK
    gauss.scale_rate = 0.0
    gauss.num_params = 3
    assert lib.ut_lowering_report(ctypes.byref(gauss), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"num_params must equal 2" in buf.value and b"gamma shape and rate" in buf.value
    # the observation count bound of the 32-bit observation index arithmetic
    glm.num_obs = (1 << 30) + 1
    assert lib.ut_lowering_report(ctypes.byref(glm), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"num_obs must be <= 2^30" in buf.value
    glm.num_obs = 1 << 30
    assert lib.ut_lowering_report(ctypes.byref(glm), buf, len(buf)) == nat.UT_OK

    nks = nat.PlanDesc(family=nat.UT_FAMILY_NORMAL_KNOWN_SCALE, num_params=1, num_obs=1, mu_scale=1.0, obs_scale=1.0)
    assert lib.ut_lowering_report(ctypes.byref(nks), buf, len(buf)) == nat.UT_OK
    nks.obs_scale = 0.0
    nks.num_params = 2
    assert lib.ut_lowering_report(ctypes.byref(nks), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED
    assert b"num_params must equal 1 (mu)" in buf.value and b"observation scale" in buf.value
    nks.num_params, nks.obs_scale = 1, float("inf")
    assert lib.ut_lowering_report(ctypes.byref(nks), buf, len(buf)) == nat.UT_ERR_UNSUPPORTED



def test_noalloc_rejects_observation_counts_past_the_bound(lib):
    """The allocation-free entry point checks its sizes before it touches a
    device: num_obs beyond 2^30 (where the split plan's 32-bit observation
    bounds could overflow) is an argument error with a clear message, and so
    is a batch past the fixed scratch."""
    from uncertaintea_b200 import _native as nat
    fake = ctypes.c_void_p(16)   # never dereferenced: the size checks come first
    fn = lib.ut_glm_logjoint_gradient_noalloc
    for n in ((1 << 30) + 1, 0, -5):
        assert fn(fake, fake, n, 4, 0, 0.0, 1.0, 0.0, 1.0, fake, 8, fake, fake, None) == nat.UT_ERR_ARGUMENT
        assert "num_obs must be in 1..2^30" in nat.last_error()
    assert fn(fake, fake, 100, 64, 0, 0.0, 1.0, 0.0, 1.0, fake, 70_000, fake, fake, None) == nat.UT_ERR_ARGUMENT
    assert "exceeds the fixed scratch" in nat.last_error()


def test_workspace_create_validates_before_touching_device(lib):
    from uncertaintea_b200 import _native as nat
    plan = nat.PlanDesc(family=nat.UT_FAMILY_GLM_BERNOULLI_LOGIT, num_params=2, num_obs=3, num_coefs=2,
                        coef_sigma=1.0)
    obs = np.zeros(9, dtype=np.float32)
    h = ctypes.c_void_p()
    assert lib.ut_workspace_create(ctypes.byref(plan), obs.ctypes.data, 9, 1, None, None, 0, 4, 64,
                                   ctypes.byref(h)) == nat.UT_ERR_PRECISION
    assert lib.ut_workspace_create(ctypes.byref(plan), obs.ctypes.data, 8, 1, None, None, 0, 4, 32,
                                   ctypes.byref(h)) == nat.UT_ERR_DIMENSION
    assert lib.ut_workspace_create(ctypes.byref(plan), obs.ctypes.data, 9, 4, None, None, 0, 4, 32,
                                   ctypes.byref(h)) == nat.UT_ERR_UNSUPPORTED
    if not HAS_GPU:
        assert lib.ut_workspace_create(ctypes.byref(plan), obs.ctypes.data, 9, 1, None, None, 0, 4, 32,
                                       ctypes.byref(h)) == nat.UT_ERR_NO_DEVICE


_HANDLE_ENTRY_POINTS = [
    "ut_hmc_iteration", "ut_chees_iteration", "ut_surrogate_hmc_iteration", "ut_leapfrog_probe", "ut_persistent_nuts_iteration",
    "ut_meads_init", "ut_meads_iteration", "ut_advi_step", "ut_lockstep_nuts_iteration", "ut_chees_reduce",
    "ut_workspace_check", "ut_workspace_info", "ut_logjoint", "ut_logjoint_gradient", "ut_logjoint_device",
    "ut_logjoint_gradient_device", "ut_surrogate_num_weights", "ut_surrogate_get_weights",
    "ut_surrogate_set_weights", "ut_surrogate_get_normalization", "ut_surrogate_set_normalization",
    "ut_surrogate_fit_normalization", "ut_surrogate_train", "ut_surrogate_loss_gradient", "ut_surrogate_gradient",
    "ut_surrogate_check", "ut_multi_layout", "ut_multi_class_info", "ut_multi_configure", "ut_multi_set_positions",
    "ut_multi_begin", "ut_multi_run", "ut_multi_autotune", "ut_multi_split_rhat", "ut_multi_buffers",
]


def _null_args(fn):
    import ctypes as ct
    out = []
    for t in fn.argtypes:
        if t in (ct.c_float, ct.c_double):
            out.append(0.0)
        elif t in (ct.c_int8, ct.c_uint8, ct.c_int16, ct.c_int32, ct.c_uint32, ct.c_int64, ct.c_uint64):
            out.append(0)
        else:
            out.append(None)
    return out


def test_entry_points_reject_null_handles_and_buffers(lib):
    """Every entry point that takes a workspace, surrogate or multi-model handle
    returns UT_ERR_ARGUMENT (never a crash) for a null handle, the no-allocation
    gradient for null buffers, and the destroy calls accept null; the message
    names the problem."""
    from uncertaintea_b200 import _native as nat
    for name in _HANDLE_ENTRY_POINTS:
        fn = getattr(lib, name)
        assert fn(*_null_args(fn)) == nat.UT_ERR_ARGUMENT, name
        assert b"null" in nat.last_error().encode() or b"handle" in nat.last_error().encode(), name
    fn = lib.ut_glm_logjoint_gradient_noalloc
    assert fn(*_null_args(fn)) == nat.UT_ERR_ARGUMENT
    for name in ("ut_workspace_destroy", "ut_surrogate_destroy", "ut_multi_destroy"):
        assert getattr(lib, name)(None) == nat.UT_OK


def _tc_split(lib, N, C, sms):
    fn = lib.ut_internal_tc_split_plan
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    S, tps = ctypes.c_int32(), ctypes.c_int32()
    assert fn(N, C, sms, ctypes.addressof(S), ctypes.addressof(tps)) == 0
    return S.value, tps.value


def test_tensor_core_split_minimises_the_wave_model(lib):
    """The tensor-core grid's observation split (host planning, no GPU): the
    100000 x 100 design with 4096 chains on 148 SMs gets S = 9 (288 CTAs in two
    waves, 348 tiles each); for every shape the chosen split covers the tiles
    exactly once, keeps >= 8 tiles per CTA when it can, and no other split has a
    lower ceil(CTAs / SMs) x (11 + tiles per CTA) cost."""
    import math
    assert _tc_split(lib, 100000, 4096, 148) == (9, 348)
    for N, C, sms in [(100000, 4096, 148), (20000, 128, 148), (3000, 64, 148), (5000, 300, 148), (100000, 1024, 148),
                      (31, 128, 148), (100, 4096, 132), (777, 33, 148), (1_000_000, 8192, 148)]:
        S, tps = _tc_split(lib, N, C, sms)
        nt, ct = (N + 31) // 32, (C + 127) // 128
        assert S * tps >= nt and (S - 1) * tps < nt
        assert tps >= 8 or S == 1
        cost = lambda s_: math.ceil(ct * s_ / sms) * (11 + (nt + s_ - 1) // s_)  # noqa: E731
        best = min(cost((nt + ((nt + s_ - 1) // s_) - 1) // ((nt + s_ - 1) // s_)) for s_ in range(1, max(1, nt // 8) + 1))
        assert cost(S) == best, (N, C, S)
    assert lib.ut_internal_tc_split_plan(0, 4096, 148, None, None) != 0


def test_tensor_core_live_split_fits_the_launched_grid(lib):
    """The lockstep tree's live-chain split (tc_split with a live count) for
    every live count of several shapes: the live work (chain tiles x splits)
    never exceeds the launched grid, so the partial rows sized for the full
    plan hold it; the splits cover every observation tile once with no empty
    split; few live tiles are re-split to fill the SMs; without a live count
    the full plan comes back unchanged."""
    fn = lib.ut_internal_tc_live_split
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    out = (ctypes.c_int32 * 4)()
    for N, C, sms in [(100000, 4096, 148), (20000, 512, 148), (3000, 300, 148), (100, 4096, 132)]:
        S_full, tps_full = _tc_split(lib, N, C, sms)
        nt_tiles, ctiles = (N + 31) // 32, (C + 127) // 128
        assert fn(N, C, sms, -1, out) == 0
        assert list(out) == [ctiles, S_full, tps_full, C]
        for live in sorted({0, 1, 2, 127, 128, 129, 255, 256, C // 2, C - 1, C} | set(range(0, C + 1, 97))):
            assert fn(N, C, sms, live, out) == 0
            nt, S, tps, Cl = list(out)
            assert nt == max(1, (live + 127) // 128) and Cl == nt * 128 and nt <= ctiles
            assert nt * S <= ctiles * S_full, (N, C, live)
            assert S * tps >= nt_tiles and (S - 1) * tps < nt_tiles
            assert S >= S_full
            if nt * S_full < min(ctiles * S_full, sms):
                assert nt * S >= min(ctiles * S_full, sms, nt * nt_tiles) // 2, (N, C, live, nt, S)
    assert fn(100, 10, 148, 11, out) != 0


def test_streaming_stage_plan_stays_in_shared_memory(lib):
    """The streaming kernel's stage plan for every chain bucket and feature count
    it serves, under the 227 KB a CTA can opt into (less the 1 KB the launch
    keeps): the whole layout fits; stages are a whole multiple of the chunk slots
    (each stage belongs to one slot, so its mbarrier phase is never ambiguous);
    there are at least 4 stages and at most 48 (the mbarrier header's size); the
    ring can hold the warps' partials after the stream, 16 x (chains per warp) x
    (F + 1) floats; and too small a budget is refused, not overrun."""
    fn = lib.ut_internal_stream_plan
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    limit = 227 * 1024 - 1024
    for CB in (1, 2, 4, 8, 16):
        cg = 2 if CB >= 2 else 1
        ch = CB // cg
        for F in range(4, 129, 4):
            st, sl, sm = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
            rc = fn(CB, F, limit, ctypes.addressof(st), ctypes.addressof(sl), ctypes.addressof(sm))
            assert rc == 0, (CB, F)
            stages, slots = st.value, sl.value
            assert sm.value <= limit, (CB, F, sm.value)
            assert 4 <= stages <= 48 and stages % slots == 0 and 1 <= slots <= 16 // cg, (CB, F, stages, slots)
            assert 16 * ch * (F + 1) <= stages * 32 * (F + 1)
            fixed = 1024 + 4 * (CB * F + 16 * 32 * ch)
            assert sm.value == fixed + 4 * stages * (32 * F + 32)
    st, sl, sm = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
    from uncertaintea_b200 import _native as nat
    refs = (ctypes.addressof(st), ctypes.addressof(sl), ctypes.addressof(sm))
    assert fn(16, 128, 40 * 1024, *refs) == nat.UT_ERR_UNSUPPORTED
    assert fn(17, 128, limit, *refs) == nat.UT_ERR_ARGUMENT


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_handle_free_entry_points_report_no_device(lib):
    """Without a device the compute entry points that need no handle return
    UT_ERR_NO_DEVICE: there is no CPU fallback behind the C ABI."""
    import ctypes as ct
    from uncertaintea_b200 import _native as nat
    keys = np.zeros(2, dtype=np.uint32)
    ctrs = np.zeros(4, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    assert lib.ut_philox4x32(keys.ctypes.data, ctrs.ctypes.data, 1, out.ctypes.data) == nat.UT_ERR_NO_DEVICE
    u = np.zeros(8, dtype=np.float32)
    assert lib.ut_rand_uniform(0, 0, 0, 0, 8, u.ctypes.data) == nat.UT_ERR_NO_DEVICE
    assert lib.ut_rand_normal(0, 0, 0, 0, 8, u.ctypes.data) == nat.UT_ERR_NO_DEVICE
    h = ct.c_void_p()
    assert lib.ut_surrogate_create(4, 1, ct.byref(h)) == nat.UT_ERR_NO_DEVICE and not h.value
    assert lib.ut_device_count() == 0


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_no_cpu_fallback_without_device():
    from uncertaintea_b200 import BernoulliLogitGLM, device_batched_logjoint, logistic_regression_data
    X, y, _ = logistic_regression_data(10, 2, 0)
    with pytest.raises(Exception):
        device_batched_logjoint(BernoulliLogitGLM(2), np.zeros((2, 3)), (X,), {"y": y})


def test_tensor_core_tmem_plan_fits_for_every_feature_count(lib):
    """The tensor-core kernel's TMEM columns: Theta hi / lo (KC = F rounded up
    to 8 each), the gradient accumulator (Fp = F rounded up to 16) and 2 or 3
    H/R buffers of 64 columns fit the 512 allocated columns for every feature
    count the path takes (1..128), with 3 buffers at 100 features."""
    fn = lib.ut_internal_tc_tmem_plan
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    out = (ctypes.c_int32 * 4)()
    for F in range(1, 129):
        assert fn(F, out) == 0
        KC, Fp, nb, cols = list(out)
        assert KC == 8 * ((F + 7) // 8) and Fp == 16 * ((F + 15) // 16)
        assert 2 <= nb <= 3 and cols <= 512 and cols == 2 * KC + Fp + 64 * nb, (F, list(out))
    fn(100, out)
    assert list(out) == [104, 112, 3, 512]
    assert fn(129, out) != 0 and fn(0, out) != 0


def test_tensor_core_paired_copy_stays_in_its_stage(lib):
    """The paired GEMM1's 4-D TMA copy ([K-block][hi, lo][32 rows][8 features])
    and its N = 64 B-operand reads (2 KB per K-block) stay inside the stage's
    K-major region for every feature count, and the copy meets the tensor-map
    rules: box dimensions <= 256, a 32-byte innermost box (the 32-byte swizzle
    span), strides that are multiples of 16 bytes and below 2^40 up to 2^30
    observations."""
    fn = lib.ut_internal_tc_pair_plan
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    out = (ctypes.c_int64 * 6)()
    for F in range(1, 129):
        for N in (1, 31, 32, 33, 100_000, 1 << 30):
            assert fn(F, N, out) == 0
            kb, box, region, read_end, hl, inner = list(out)
            Fp = 16 * ((F + 15) // 16)
            assert kb == (F + 7) // 8 and 1 <= kb <= 256
            assert box == 2 * 1024 * kb and box <= region and read_end <= region, (F, list(out))
            assert region == 2 * 1024 * (Fp // 8)
            assert inner == 32 and (Fp * 4) % 16 == 0 and hl % 16 == 0 and hl < (1 << 40)
    assert fn(0, 10, out) != 0 and fn(129, 10, out) != 0 and fn(10, 0, out) != 0
