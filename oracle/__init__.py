"""CPU oracle of the batched density + sampler hot path.

TEST INFRASTRUCTURE: only the tests, ``__graft_entry__.smoke`` and the CPU
baseline leg of ``bench.py`` use this package, as the test oracle.  The product
library never calls it.  See oracle.cpp for what each function restates and
how far parity is pinned: Philox, the ChEES scalar helpers, the NUTS U-turn
helpers and the MEADS estimator / slice drift by the reference's own unit
tests; the densities by closed forms and finite differences on the
reference's parity-case inputs; the samplers by exact posteriors.  None of it
is pinned by reference outputs, which need Julia.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int32, c_int64, c_uint32, c_void_p

import numpy as np

from .build_oracle import LIB, build

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    path = build()
    lib = ctypes.CDLL(path)
    sig = {
        "orc_philox4x32": (None, [c_uint32, c_uint32, c_void_p, c_void_p]),
        "orc_rand_uniform_f32": (None, [c_uint32, c_uint32, c_uint32, c_uint32, c_int64, c_void_p]),
        "orc_rand_normal_f32": (None, [c_uint32, c_uint32, c_uint32, c_uint32, c_int64, c_void_p]),
        "orc_rand_uniform_f64": (None, [c_uint32, c_uint32, c_uint32, c_uint32, c_int64, c_void_p]),
        "orc_rand_normal_f64": (None, [c_uint32, c_uint32, c_uint32, c_uint32, c_int64, c_void_p]),
        "orc_logjoint_gradient_f64": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                                c_void_p, c_int32]),
        "orc_logjoint_gradient_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                                c_void_p, c_int32]),
        "orc_gradient_magnitude_f64": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                                 c_int32]),
        "orc_program_set": (None, [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32]),
        "orc_max_threads": (c_int32, []),
        "orc_meads_max_eig": (c_double, [c_void_p, c_int32, c_int32]),
        "orc_meads_iteration_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32,
                                              c_uint32, c_float] + [c_void_p] * 12),
        "orc_advi_step_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_uint32,
                                        c_void_p, c_void_p, c_void_p, c_void_p]),
        "orc_hmc_iteration_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_void_p, c_int32, c_uint32, c_float, c_void_p,
                                            c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32]),
        "orc_leapfrog_probe_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                                             c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_int32]),
        "orc_nuts_iteration_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                                             c_void_p, c_void_p, c_void_p, c_int32, c_float, c_uint32, c_void_p,
                                             c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32]),
        "orc_nuts_iteration_keyed_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_uint32,
                                                   c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
                                                   c_float, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p,
                                                   c_void_p, c_void_p, c_void_p, c_int32]),
        "orc_chees_reduce": (None, [c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
        "orc_is_turning_f64": (c_int32, [c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
        "orc_meads_slice_drift_f64": (c_double, [c_double, c_double]),
        "orc_store_tree_checkpoint_f64": (None, [c_int32, c_void_p, c_int32, c_void_p, c_void_p]),
        "orc_dyadic_turning_f64": (c_int32, [c_int32, c_void_p, c_int32, c_void_p, c_void_p, c_int32, c_void_p]),
        "orc_mlp_num_weights": (c_int64, [c_int32]),
        "orc_mlp_forward": (None, [c_void_p, c_void_p, c_int32, c_void_p, c_int64, c_void_p, c_int32]),
        "orc_mlp_loss_gradient": (None, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_int64, c_void_p, c_int32,
                                         c_void_p, c_void_p, c_int32]),
        "orc_surrogate_hmc_iteration_f32": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                                      c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                                      c_int32, c_uint32, c_float, c_void_p, c_void_p, c_void_p,
                                                      c_void_p, c_void_p, c_void_p, c_void_p, c_int32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


def philox4x32(key, counter):
    out = np.zeros(4, dtype=np.uint32)
    ctr = np.asarray(counter, dtype=np.uint32)
    load().orc_philox4x32(int(key[0]), int(key[1]), _p(ctr), _p(out))
    return tuple(int(v) for v in out)


def rand_uniform(chain, iteration, stream, draw_start, n, dtype=np.float32):
    out = np.empty(n, dtype=dtype)
    fn = load().orc_rand_uniform_f32 if dtype == np.float32 else load().orc_rand_uniform_f64
    fn(chain, iteration, stream, draw_start, n, _p(out))
    return out


def rand_normal(chain, iteration, stream, draw_start, n, dtype=np.float32):
    out = np.empty(n, dtype=dtype)
    fn = load().orc_rand_normal_f32 if dtype == np.float32 else load().orc_rand_normal_f64
    fn(chain, iteration, stream, draw_start, n, _p(out))
    return out


def meads_max_eig(columns):
    """The MEADS trace-ratio largest-eigenvalue estimate of a P x N matrix whose
    columns are the ensemble members (api_batched_meads.jl:48-78)."""
    c = np.ascontiguousarray(np.asarray(columns, dtype=np.float64).T)   # N x P
    return float(load().orc_meads_max_eig(_p(c), c.shape[1] if c.ndim == 2 else 0, c.shape[0]))


def meads_slice_drift(u, delta):
    """MEADS persistent-slice drift ((u + 1 + delta) mod 2) - 1 (api_batched_meads.jl:140)."""
    return float(load().orc_meads_slice_drift_f64(float(u), float(delta)))


def _vec(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))


def is_turning(q_left, q_right, p_left, p_right, inverse_mass=None):
    """Metric-aware U-turn criterion (state_init.jl:296-350): turning when
    (q_right - q_left) . M^-1 p is <= 0 at either end."""
    ql, qr, pl, pr = _vec(q_left), _vec(q_right), _vec(p_left), _vec(p_right)
    im = np.ones_like(ql) if inverse_mass is None else _vec(inverse_mass)
    return bool(load().orc_is_turning_f64(ql.size, _p(ql), _p(qr), _p(pl), _p(pr), _p(im)))


def new_checkpoints(P, max_depth):
    """Checkpoint storage of one subtree: [slots][position, momentum][P]."""
    return np.zeros((max_depth + 1, 2, P), dtype=np.float64)


def store_tree_checkpoint(ckpt, leaf_index, q, p):
    """Even leaf into slot popcount(leaf_index) (tree_expand.jl:64-76)."""
    qv, pv = _vec(q), _vec(p)
    load().orc_store_tree_checkpoint_f64(qv.size, _p(ckpt), int(leaf_index), _p(qv), _p(pv))


def dyadic_turning(ckpt, leaf_index, q, p, direction, inverse_mass=None):
    """Odd-leaf dyadic U-turn test against the block checkpoints (tree_expand.jl:82-102)."""
    qv, pv = _vec(q), _vec(p)
    im = np.ones_like(qv) if inverse_mass is None else _vec(inverse_mass)
    return bool(load().orc_dyadic_turning_f64(qv.size, _p(ckpt), int(leaf_index), _p(qv), _p(pv), int(direction),
                                              _p(im)))


class OracleModel:
    """Wraps a lowered kernel description for the oracle entry points."""

    def __init__(self, lowered):
        self.lowered = lowered
        self.plan = lowered.plan
        self.P = lowered.num_params
        self.obs = np.ascontiguousarray(lowered.observed, dtype=np.float32)
        self.tc = np.ascontiguousarray(lowered.trip_counts, dtype=np.int32)
        self.ls = np.ascontiguousarray(lowered.loop_starts, dtype=np.int32)

    def _common(self):
        prog = getattr(self.lowered, "program", None)
        if prog is not None:  # a step program: the oracle walks the one set last
            lw = self.lowered
            load().orc_program_set(ctypes.addressof(lw.steps), len(prog.steps), ctypes.addressof(lw.nodes),
                                   len(prog.nodes), prog.num_slots, prog.num_params)
        return (ctypes.byref(self.plan), _p(self.obs), _p(self.tc) if self.tc.size else None,
                _p(self.ls) if self.ls.size else None)

    # Every array handed to the library is bound to a local name first, so it
    # stays alive until the call returns.

    def logjoint_gradient_f64(self, params_cp, threads=0, want_grad=True):
        q = np.ascontiguousarray(params_cp, dtype=np.float64)
        C = q.shape[0]
        totals = np.empty(C)
        grads = np.empty_like(q) if want_grad else None
        load().orc_logjoint_gradient_f64(*self._common(), _p(q), C, _p(totals), _p(grads), threads)
        return totals, grads

    def gradient_magnitude_f64(self, params_cp, threads=0):
        """Per gradient element, the sum of the magnitudes of the terms it adds
        up (the scale FP32 rounding errors of the gradient are relative to)."""
        q = np.ascontiguousarray(params_cp, dtype=np.float64)
        out = np.empty_like(q)
        load().orc_gradient_magnitude_f64(*self._common(), _p(q), q.shape[0], _p(out), threads)
        return out

    def logjoint_gradient_f32(self, params_cp, threads=0, want_grad=True):
        q = np.ascontiguousarray(params_cp, dtype=np.float32)
        C = q.shape[0]
        totals = np.empty(C, dtype=np.float32)
        grads = np.empty_like(q) if want_grad else None
        load().orc_logjoint_gradient_f32(*self._common(), _p(q), C, _p(totals), _p(grads), threads)
        return totals, grads

    def meads_iteration(self, position, gradient, logjoint, momentum, slice_u, num_folds, iteration, coord,
                        thr=1000.0):
        """One MEADS iteration (orc_meads_iteration_f32) on copies of the state."""
        st = {"position": np.array(position, dtype=np.float32), "gradient": np.array(gradient, dtype=np.float32),
              "logjoint": np.array(logjoint, dtype=np.float32), "momentum": np.array(momentum, dtype=np.float32),
              "slice": np.array(slice_u, dtype=np.float32)}
        C = st["position"].shape[0]
        out = {k: np.empty(C, dtype=np.float32) for k in ("accept_prob", "energy", "energy_error")}
        out["accepted"] = np.empty(C, dtype=np.uint8)
        out["divergent"] = np.empty(C, dtype=np.uint8)
        out["integration_steps"] = np.empty(C, dtype=np.int32)
        out["fold_parameters"] = np.empty((num_folds, 4), dtype=np.float32)
        load().orc_meads_iteration_f32(*self._common(), C, num_folds, iteration, coord, thr,
                                       *[_p(st[k]) for k in ("position", "gradient", "logjoint", "momentum", "slice")],
                                       *[_p(out[k]) for k in ("accept_prob", "energy", "energy_error", "accepted",
                                                              "divergent", "integration_steps", "fold_parameters")])
        st.update(out)
        return st

    def advi_step(self, location, scale, num_particles, coord):
        """One mean-field ADVI step (orc_advi_step_f32): particles, values, mean
        gradient and mean gradient * scale * eps."""
        loc = np.ascontiguousarray(location, dtype=np.float32)
        sc = np.ascontiguousarray(scale, dtype=np.float32)
        M, P = int(num_particles), self.P
        particles = np.empty((M, P), dtype=np.float32)
        values = np.empty(M, dtype=np.float32)
        lg = np.empty(P, dtype=np.float32)
        sg = np.empty(P, dtype=np.float32)
        load().orc_advi_step_f32(*self._common(), M, _p(loc), _p(sc), coord, _p(particles), _p(values), _p(lg),
                                 _p(sg))
        return {"particles": particles, "values": values, "location_gradient": lg, "scale_gradient": sg}

    def hmc_iteration(self, position, gradient, logjoint, inverse_mass, step, L, coord, thr=1000.0,
                      want_proposal=False, threads=0):
        C = position.shape[0]
        inverse_mass = np.ascontiguousarray(inverse_mass, dtype=np.float32)  # held for the call
        step = np.ascontiguousarray(step, dtype=np.float32)
        out = {k: np.empty(C, dtype=np.float32) for k in ("accept_prob", "energy", "energy_error")}
        out["accepted"] = np.empty(C, dtype=np.uint8)
        out["divergent"] = np.empty(C, dtype=np.uint8)
        prop = np.empty_like(position) if want_proposal else None
        mom = np.empty_like(position) if want_proposal else None
        load().orc_hmc_iteration_f32(*self._common(), C, _p(position), _p(gradient), _p(logjoint),
                                     _p(inverse_mass), _p(step), L, coord, thr,
                                     _p(out["accept_prob"]), _p(out["energy"]), _p(out["energy_error"]),
                                     _p(out["accepted"]), _p(out["divergent"]), _p(prop), _p(mom), threads)
        out["proposal"], out["endpoint_momentum"] = prop, mom
        return out

    def leapfrog_probe(self, position, gradient, logjoint, inverse_mass, trial_step, coord, threads=0):
        C = position.shape[0]
        lar = np.empty(C, dtype=np.float32)
        inverse_mass = np.ascontiguousarray(inverse_mass, dtype=np.float32)
        trial_step = np.ascontiguousarray(trial_step, dtype=np.float32)
        load().orc_leapfrog_probe_f32(*self._common(), C, _p(position), _p(gradient), _p(logjoint),
                                      _p(inverse_mass), _p(trial_step), coord, _p(lar), threads)
        return lar

    def surrogate_hmc_iteration(self, weights, norm, position, logjoint, inverse_mass, step, L, coord, thr=1000.0,
                                bf16=True, want_proposal=False, threads=0):
        """Surrogate-driven HMC iteration (kicks from the MLP oracle, exact accept);
        position and logjoint are updated in place."""
        C = position.shape[0]
        weights = np.ascontiguousarray(weights, dtype=np.float32)
        norm = np.ascontiguousarray(norm, dtype=np.float32)
        inverse_mass = np.ascontiguousarray(inverse_mass, dtype=np.float32)
        step = np.ascontiguousarray(step, dtype=np.float32)
        out = {k: np.empty(C, dtype=np.float32) for k in ("accept_prob", "energy", "energy_error")}
        out["accepted"] = np.empty(C, dtype=np.uint8)
        out["divergent"] = np.empty(C, dtype=np.uint8)
        prop = np.empty_like(position) if want_proposal else None
        mom = np.empty_like(position) if want_proposal else None
        load().orc_surrogate_hmc_iteration_f32(*self._common(), C, _p(weights), _p(norm), int(bool(bf16)),
                                               _p(position), _p(logjoint), _p(inverse_mass), _p(step), L, coord,
                                               thr, _p(out["accept_prob"]), _p(out["energy"]),
                                               _p(out["energy_error"]), _p(out["accepted"]), _p(out["divergent"]),
                                               _p(prop), _p(mom), threads)
        out["proposal"], out["endpoint_momentum"] = prop, mom
        return out

    def nuts_iteration(self, position, gradient, logjoint, inverse_mass, step, max_depth, coord, thr=1000.0,
                       threads=0, chain_key_offset=0):
        C = position.shape[0]
        inverse_mass = np.ascontiguousarray(inverse_mass, dtype=np.float32)
        step = np.ascontiguousarray(step, dtype=np.float32)
        out = {k: np.empty(C, dtype=np.float32) for k in ("accept_prob", "energy", "energy_error")}
        out["tree_depth"] = np.empty(C, dtype=np.int32)
        out["integration_steps"] = np.empty(C, dtype=np.int32)
        out["divergent"] = np.empty(C, dtype=np.uint8)
        out["moved"] = np.empty(C, dtype=np.uint8)
        load().orc_nuts_iteration_keyed_f32(*self._common(), C, int(chain_key_offset), _p(position), _p(gradient),
                                            _p(logjoint),
                                      _p(inverse_mass), _p(step), max_depth, thr, coord,
                                      _p(out["accept_prob"]), _p(out["energy"]), _p(out["energy_error"]),
                                      _p(out["tree_depth"]), _p(out["integration_steps"]), _p(out["divergent"]),
                                      _p(out["moved"]), threads)
        return out


def chees_reduce(initials, proposals, momenta, accept_prob, divergent, inverse_mass):
    C, P = initials.shape
    out = np.zeros(2)
    held = [np.ascontiguousarray(a, dtype=dt) for a, dt in ((initials, np.float32), (proposals, np.float32),
                                                            (momenta, np.float32), (accept_prob, np.float32),
                                                            (divergent, np.uint8), (inverse_mass, np.float32))]
    load().orc_chees_reduce(P, C, *[_p(a) for a in held], _p(out))
    return out


def mlp_num_weights(P):
    return int(load().orc_mlp_num_weights(P))


def mlp_forward(weights, norm, theta, bf16=True):
    """Surrogate MLP restatement: gradient estimates at the rows of theta (n x P)."""
    theta = np.ascontiguousarray(theta, dtype=np.float32)
    weights = np.ascontiguousarray(weights, dtype=np.float32)
    norm = np.ascontiguousarray(norm, dtype=np.float32)
    n, P = theta.shape
    out = np.empty((n, P), dtype=np.float32)
    load().orc_mlp_forward(_p(weights), _p(norm), P, _p(theta), n, _p(out), int(bool(bf16)))
    return out


def mlp_loss_gradient(weights, norm, theta, grad, index, bf16=True):
    """Loss and FP64 weight gradient of the batch of pair rows `index`."""
    theta = np.ascontiguousarray(theta, dtype=np.float32)
    grad = np.ascontiguousarray(grad, dtype=np.float32)
    weights = np.ascontiguousarray(weights, dtype=np.float32)
    norm = np.ascontiguousarray(norm, dtype=np.float32)
    index = np.ascontiguousarray(index, dtype=np.int32)
    n, P = theta.shape
    wg = np.empty(weights.size, dtype=np.float64)
    loss = np.zeros(1)
    load().orc_mlp_loss_gradient(_p(weights), _p(norm), P, _p(theta), _p(grad), n, _p(index), index.size, _p(wg),
                                 _p(loss), int(bool(bf16)))
    return float(loss[0]), wg


def max_threads():
    return int(load().orc_max_threads())
