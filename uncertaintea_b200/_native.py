"""ctypes binding of the C ABI in ``include/ut_b200.h``.

The shared library ``libut_b200.so`` is built in-tree (``__graft_entry__.build``
or ``python -m uncertaintea_b200.build``).  Loading fails loudly when it is
missing: there is no CPU fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int32, c_int64, c_size_t, c_uint32, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libut_b200.so")

UT_OK = 0
UT_ERR_ARGUMENT = 1
UT_ERR_DIMENSION = 2
UT_ERR_UNSUPPORTED = 3
UT_ERR_PRECISION = 4
UT_ERR_CUDA = 5
UT_ERR_NO_DEVICE = 6
UT_ERR_DEVICE_TIMEOUT = 7

UT_FAMILY_GLM_BERNOULLI_LOGIT = 1
UT_FAMILY_HIER_NORMAL_NONCENTERED = 2
UT_FAMILY_NORMAL_LOCATION_SCALE = 3
UT_FAMILY_BERNOULLI_BETA = 4
UT_FAMILY_LOGNORMAL_GAMMA_NORMAL = 5
UT_FAMILY_STUDENTT_HEAVY_TAIL = 6
UT_FAMILY_NORMAL_KNOWN_SCALE = 7


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("family", c_int32),
        ("num_params", c_int32),
        ("num_obs", c_int32),
        ("num_coefs", c_int32),
        ("has_intercept", c_int32),
        ("num_groups", c_int32),
        ("intercept_mu", c_double),
        ("intercept_sigma", c_double),
        ("coef_mu", c_double),
        ("coef_sigma", c_double),
        ("mu_loc", c_double),
        ("mu_scale", c_double),
        ("tau_scale", c_double),
        ("scale_shape", c_double),
        ("scale_rate", c_double),
        ("prob_alpha", c_double),
        ("prob_beta", c_double),
        ("nu_prior", c_double),
        ("nu_obs", c_double),
        ("weibull_shape", c_double),
        ("weibull_scale", c_double),
        ("obs_scale", c_double),
    ]


UT_FAMILY_PROGRAM = 8
UT_MAX_OBS = 1 << 30

UT_STEP_CHOICE, UT_STEP_DETERMINISTIC, UT_STEP_LOOP, UT_STEP_IID_NORMAL, UT_STEP_GLM_BERNOULLI_LOGIT = 1, 2, 3, 4, 5
UT_TRANSFORM_IDENTITY, UT_TRANSFORM_LOG, UT_TRANSFORM_LOGIT = 0, 1, 2
DISTRIBUTIONS = {
    "normal": 1, "lognormal": 2, "exponential": 3, "gamma": 4, "laplace": 5, "cauchy": 6, "halfnormal": 7,
    "halfcauchy": 8, "logistic": 9, "gumbel": 10, "frechet": 11, "rayleigh": 12, "inversegaussian": 13, "beta": 14,
    "studentt": 15, "inversegamma": 16, "weibull": 17, "bernoulli": 18, "bernoullilogit": 19, "poisson": 20,
    "geometric": 21, "negativebinomial": 22, "binomial": 23,
}
EXPR_OPS = {
    "literal": 0, "slot": 1, "obs": 2, "neg": 3, "+": 4, "-": 5, "*": 6, "/": 7, "^": 8, "exp": 9, "log": 10,
    "log1p": 11, "sqrt": 12, "abs": 13, "min": 14, "max": 15, "sin": 16, "cos": 17, "tan": 18, "tanh": 19,
    "sinh": 20, "cosh": 21, "atan": 22, "expm1": 23,
}


class ExprNode(ctypes.Structure):
    _fields_ = [("op", c_int32), ("a", c_int32), ("b", c_int32), ("reserved", c_int32), ("value", c_double)]


class ProgramStep(ctypes.Structure):
    _fields_ = [("kind", c_int32), ("dist", c_int32), ("arg", c_int32 * 4), ("value_source", c_int32),
                ("obs_offset", c_int32), ("transform", c_int32), ("binding_slot", c_int32), ("count", c_int32),
                ("width", c_int32), ("body", c_int32), ("iterator_slot", c_int32), ("iterator_start", c_int32)]


class MeadsBuffers(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("position", "gradient", "logjoint", "momentum", "slice", "accept_prob",
                                         "energy", "energy_error", "accepted", "divergent", "integration_steps",
                                         "fold_parameters")]


class HmcBuffers(ctypes.Structure):
    _fields_ = [
        ("position", c_void_p),
        ("gradient", c_void_p),
        ("logjoint", c_void_p),
        ("inverse_mass", c_void_p),
        ("step", c_void_p),
        ("accept_prob", c_void_p),
        ("energy", c_void_p),
        ("energy_error", c_void_p),
        ("accepted", c_void_p),
        ("divergent", c_void_p),
        ("proposal", c_void_p),
        ("endpoint_momentum", c_void_p),
    ]


class NutsBuffers(ctypes.Structure):
    _fields_ = [
        ("position", c_void_p),
        ("gradient", c_void_p),
        ("logjoint", c_void_p),
        ("inverse_mass", c_void_p),
        ("step", c_void_p),
        ("accept_prob", c_void_p),
        ("energy", c_void_p),
        ("energy_error", c_void_p),
        ("tree_depth", c_void_p),
        ("integration_steps", c_void_p),
        ("divergent", c_void_p),
        ("moved", c_void_p),
    ]


class MultiView(ctypes.Structure):
    _fields_ = [
        ("position", c_void_p),
        ("gradient", c_void_p),
        ("logjoint", c_void_p),
        ("step", c_void_p),
        ("inverse_mass", c_void_p),
        ("accept_prob", c_void_p),
        ("tree_depth", c_void_p),
        ("integration_steps", c_void_p),
        ("divergent", c_void_p),
        ("draws", c_void_p),
        ("draw_accept", c_void_p),
        ("draw_tree_depth", c_void_p),
        ("draw_divergent", c_void_p),
        ("iteration", c_void_p),
        ("state_floats", c_int64),
        ("total_chains", c_int64),
        ("param_floats", c_int64),
        ("draws_capacity", c_int32),
    ]


# (name, restype, argtypes) of every exported entry point, in header order.
SIGNATURES = [
    ("ut_version", c_char_p, []),
    ("ut_last_error", c_int32, [c_char_p, c_size_t]),
    ("ut_device_count", c_int32, []),
    ("ut_lowering_report", c_int32, [POINTER(PlanDesc), c_char_p, c_size_t]),
    ("ut_workspace_create", c_int32,
     [POINTER(PlanDesc), c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_int32, c_int32, c_int32,
      POINTER(c_void_p)]),
    ("ut_workspace_destroy", c_int32, [c_void_p]),
    ("ut_workspace_info", c_int32, [c_void_p, POINTER(c_int32), POINTER(c_int32)]),
    ("ut_workspace_path", c_int32, [c_void_p]),
    ("ut_program_report", c_int32,
     [POINTER(ProgramStep), c_int32, POINTER(ExprNode), c_int32, c_int32, c_int32, c_int64, c_char_p, c_size_t]),
    ("ut_workspace_create_program", c_int32,
     [POINTER(ProgramStep), c_int32, POINTER(ExprNode), c_int32, c_int32, c_int32, c_void_p, c_int64, c_int32,
      c_int32, POINTER(c_void_p)]),
    ("ut_workspace_check", c_int32, [c_void_p, c_void_p]),
    ("ut_logjoint", c_int32, [c_void_p, c_void_p, c_void_p]),
    ("ut_logjoint_gradient", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("ut_logjoint_device", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("ut_logjoint_gradient_device", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("ut_philox4x32", c_int32, [c_void_p, c_void_p, c_int64, c_void_p]),
    ("ut_rand_uniform", c_int32, [c_uint32, c_uint32, c_uint32, c_uint32, c_int64, c_void_p]),
    ("ut_rand_normal", c_int32, [c_uint32, c_uint32, c_uint32, c_uint32, c_int64, c_void_p]),
    ("ut_hmc_iteration", c_int32, [c_void_p, POINTER(HmcBuffers), c_int32, c_uint32, c_float, c_void_p]),
    ("ut_chees_iteration", c_int32, [c_void_p, POINTER(HmcBuffers), c_int32, c_uint32, c_float, c_void_p]),
    ("ut_leapfrog_probe", c_int32,
     [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]),
    ("ut_persistent_nuts_iteration", c_int32,
     [c_void_p, POINTER(NutsBuffers), c_int32, c_float, c_uint32, c_void_p]),
    ("ut_lockstep_nuts_iteration", c_int32,
     [c_void_p, POINTER(NutsBuffers), c_int32, c_float, c_uint32, c_void_p]),
    ("ut_meads_init", c_int32, [c_void_p, POINTER(MeadsBuffers), c_uint32, c_void_p]),
    ("ut_meads_iteration", c_int32, [c_void_p, POINTER(MeadsBuffers), c_int32, c_int32, c_float, c_uint32, c_void_p]),
    ("ut_advi_step", c_int32,
     [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("ut_chees_reduce", c_int32,
     [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_double), c_void_p]),
    ("ut_running_variance_update", c_int32,
     [c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p]),
    ("ut_warmup_adapt", c_int32,
     [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p, c_int32, c_int32,
      c_double, c_void_p, c_void_p]),
    ("ut_dual_averaging_final", c_int32, [c_void_p, c_int32, c_int32, c_void_p, c_void_p]),
    ("ut_glm_logjoint_gradient_noalloc", c_int32,
     [c_void_p, c_void_p, c_int64, c_int32, c_int32, c_double, c_double, c_double, c_double, c_void_p, c_int32,
      c_void_p, c_void_p, c_void_p]),
    ("ut_surrogate_create", c_int32, [c_int32, c_uint32, POINTER(c_void_p)]),
    ("ut_surrogate_destroy", c_int32, [c_void_p]),
    ("ut_surrogate_num_weights", c_int32, [c_void_p, POINTER(c_int64)]),
    ("ut_surrogate_get_weights", c_int32, [c_void_p, c_void_p, c_int64]),
    ("ut_surrogate_set_weights", c_int32, [c_void_p, c_void_p, c_int64]),
    ("ut_surrogate_get_normalization", c_int32, [c_void_p, c_void_p]),
    ("ut_surrogate_set_normalization", c_int32, [c_void_p, c_void_p]),
    ("ut_surrogate_fit_normalization", c_int32, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p]),
    ("ut_surrogate_train", c_int32,
     [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int32, c_int32, c_float, c_float, c_uint32, c_void_p,
      c_void_p]),
    ("ut_surrogate_loss_gradient", c_int32,
     [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    ("ut_surrogate_gradient", c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    ("ut_surrogate_check", c_int32, [c_void_p, c_void_p]),
    ("ut_surrogate_hmc_iteration", c_int32,
     [c_void_p, c_void_p, POINTER(HmcBuffers), c_int32, c_uint32, c_float, c_void_p]),
    ("ut_multi_create", c_int32,
     [c_int32, POINTER(PlanDesc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, POINTER(c_void_p)]),
    ("ut_multi_destroy", c_int32, [c_void_p]),
    ("ut_multi_layout", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("ut_multi_class_info", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("ut_multi_configure", c_int32, [c_void_p, c_int32, c_int32, c_int32]),
    ("ut_multi_set_positions", c_int32, [c_void_p, c_void_p, c_void_p]),
    ("ut_multi_begin", c_int32,
     [c_void_p, c_int32, c_int32, c_uint32, c_float, c_float, c_float, c_void_p, c_int32]),
    ("ut_multi_run", c_int32, [c_void_p, c_int32, c_int32, c_void_p]),
    ("ut_multi_autotune", c_int32, [c_void_p, c_int32, c_void_p, c_void_p]),
    ("ut_multi_split_rhat", c_int32, [c_void_p, c_int32, c_void_p, c_void_p]),
    ("ut_multi_set_stopped", c_int32, [c_void_p, c_void_p, c_void_p]),
    ("ut_multi_buffers", c_int32, [c_void_p, POINTER(MultiView)]),
]

_lib = None


def exported_symbols():
    """Names of every entry point the binding expects the library to export."""
    return [name for name, _, _ in SIGNATURES]


def load():
    """Load (once) and return the shared library, with typed entry points."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY_PATH):
        raise RuntimeError(
            f"{LIBRARY_PATH} is missing: build the CUDA extension first "
            "(python -c 'import __graft_entry__ as g; g.build()'); there is no CPU fallback")
    lib = ctypes.CDLL(LIBRARY_PATH)
    for name, restype, argtypes in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


class DeviceError(RuntimeError):
    """A CUDA-side failure reported by the library."""


class DeviceTimeoutError(DeviceError):
    """A bounded in-kernel wait gave up (UT_ERR_DEVICE_TIMEOUT)."""


def last_error() -> str:
    lib = load()
    buf = ctypes.create_string_buffer(4096)
    lib.ut_last_error(buf, len(buf))
    return buf.value.decode("utf-8", "replace")


def check(status: int) -> None:
    """Translate a status code into the reference's exception types."""
    if status == UT_OK:
        return
    msg = last_error()
    if status in (UT_ERR_ARGUMENT, UT_ERR_UNSUPPORTED, UT_ERR_PRECISION):
        raise ValueError(msg)  # the reference raises ArgumentError
    if status == UT_ERR_DIMENSION:
        raise IndexError(msg)  # the reference raises DimensionMismatch
    if status == UT_ERR_DEVICE_TIMEOUT:
        raise DeviceTimeoutError(msg)
    raise DeviceError(msg)


def ptr(t) -> int:
    """Device or host address of a torch tensor / numpy array (None -> 0)."""
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data
