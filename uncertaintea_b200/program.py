"""Step programs: the composable kernel description of a model.

The reference lowers a ``@tea static`` model to a ``DeviceExecutionPlan``, a
tuple of typed steps (src/device/plan/steps.jl:6-489) over expressions
(src/device/plan/exprs.jl) that its device kernels walk
(src/device/logjoint_kernel.jl:724, src/device/gradient_kernel.jl:1124).
``Program`` builds the same thing in this library's C form
(``ut_program_step`` / ``ut_expr_node`` in include/ut_b200.h): latent and
observed choice steps of the reference's scalar families, deterministic
bindings, loops over blocks of staged observations, the iid normal vector
prior and the fused Bernoulli-logit GLM likelihood.  ``ProgramModel`` wraps a
program and its staged observations as a model every sampler accepts; the
device evaluates it with one warp per chain and a reverse-mode gradient.

Example (the centred eight-schools model; staged rows y_1, sigma_1, y_2, ...)::

    p = Program()
    mu = p.latent("mu", "normal", 0.0, 5.0)
    tau = p.latent("tau", "halfcauchy", 5.0)            # log transform by default
    for j in range(8):
        theta = p.latent(f"theta[{j + 1}]", "normal", mu, tau)
        p.observe("normal", theta, p.obs(2 * j + 1), row=2 * j)
    model = ProgramModel(p, staged)

Latent values sit outside loops (the reference's device lowering has the same
rule for scalar latents, src/device/plan/lowering.jl:696-734); observations
inside a loop name their row within the loop's block.
"""
from __future__ import annotations

import contextlib
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .models import Lowered, TeaModelSpec

# Default transform of a latent value by the support of its distribution
# (the reference's default parameter transforms, src/parameters.jl).
_POSITIVE = {"lognormal", "exponential", "gamma", "halfnormal", "halfcauchy", "frechet", "rayleigh",
             "inversegaussian", "inversegamma", "weibull"}
_UNIT = {"beta"}
_NARGS = {"normal": 2, "lognormal": 2, "exponential": 1, "gamma": 2, "laplace": 2, "cauchy": 2, "halfnormal": 1,
          "halfcauchy": 1, "logistic": 2, "gumbel": 2, "frechet": 2, "rayleigh": 1, "inversegaussian": 2, "beta": 2,
          "studentt": 3, "inversegamma": 2, "weibull": 2, "bernoulli": 1, "bernoullilogit": 1, "poisson": 1,
          "geometric": 1, "negativebinomial": 2, "binomial": 2}
_TRANSFORMS = {"identity": nat.UT_TRANSFORM_IDENTITY, "log": nat.UT_TRANSFORM_LOG, "logit": nat.UT_TRANSFORM_LOGIT}
_UNARY = ("exp", "log", "log1p", "sqrt", "abs", "sin", "cos", "tan", "tanh", "sinh", "cosh", "atan", "expm1")


class Expr:
    """A node of a program's expression list (operators build new nodes)."""

    def __init__(self, prog: "Program", index: int):
        self.prog, self.index = prog, index

    def _bin(self, op, other, swap=False):
        o = self.prog.expr(other)
        a, b = (o, self) if swap else (self, o)
        return self.prog._node(op, a.index, b.index)

    def __add__(self, o): return self._bin("+", o)
    def __radd__(self, o): return self._bin("+", o, True)
    def __sub__(self, o): return self._bin("-", o)
    def __rsub__(self, o): return self._bin("-", o, True)
    def __mul__(self, o): return self._bin("*", o)
    def __rmul__(self, o): return self._bin("*", o, True)
    def __truediv__(self, o): return self._bin("/", o)
    def __rtruediv__(self, o): return self._bin("/", o, True)
    def __pow__(self, o): return self._bin("^", o)
    def __rpow__(self, o): return self._bin("^", o, True)
    def __neg__(self): return self.prog._node("neg", self.index)


@dataclass
class _Latent:
    name: str
    dist: str
    row: int
    size: int
    transform: int


@dataclass
class Program:
    """Builder of a step program; ``num_params`` rows are assigned in order."""

    steps: list = field(default_factory=list)
    nodes: list = field(default_factory=list)
    num_slots: int = 0
    num_params: int = 0
    latents: list = field(default_factory=list)
    _depth: int = 0

    # ---- expressions -------------------------------------------------------
    def _node(self, op, a=0, b=0, value=0.0):
        self.nodes.append((nat.EXPR_OPS[op], int(a), int(b), float(value)))
        return Expr(self, len(self.nodes) - 1)

    def expr(self, x) -> Expr:
        """A literal for a number, the expression itself otherwise."""
        if isinstance(x, Expr):
            return x
        return self._node("literal", value=float(x))

    def f(self, name: str, x) -> Expr:
        """A unary function of the reference's primitive set (exprs.jl)."""
        if name not in _UNARY:
            raise ValueError(f"unsupported function {name!r}")
        return self._node(name, self.expr(x).index)

    def min(self, a, b): return self._node("min", self.expr(a).index, self.expr(b).index)
    def max(self, a, b): return self._node("max", self.expr(a).index, self.expr(b).index)

    def obs(self, row: int, depth: int | None = None) -> Expr:
        """The staged value at `row` of the observation block of loop depth
        `depth` (default: the current one; 0 = the top-level block)."""
        return self._node("obs", int(row), self._depth if depth is None else int(depth))

    def _slot(self):
        self.num_slots += 1
        return self.num_slots - 1

    # ---- steps -------------------------------------------------------------
    def _step(self, kind, dist=0, args=(), value_source=-1, obs_offset=0, transform=0, binding_slot=-1, count=0,
              width=0, body=0, iterator_slot=-1, iterator_start=0):
        arg = [self.expr(a).index for a in args] + [-1] * (4 - len(args))
        self.steps.append(dict(kind=kind, dist=dist, arg=arg, value_source=value_source, obs_offset=obs_offset,
                               transform=transform, binding_slot=binding_slot, count=count, width=width, body=body,
                               iterator_slot=iterator_slot, iterator_start=iterator_start))
        return len(self.steps) - 1

    def _dist(self, dist, args):
        if dist not in _NARGS:
            raise ValueError(f"unsupported distribution {dist!r}")
        if len(args) != _NARGS[dist]:
            raise ValueError(f"{dist} takes {_NARGS[dist]} arguments, got {len(args)}")
        return nat.DISTRIBUTIONS[dist]

    def latent(self, name: str, dist: str, *args, transform: str | None = None) -> Expr:
        """A scalar latent choice on the next parameter row; returns its
        (constrained) value.  The transform defaults to the support's."""
        d = self._dist(dist, args)
        if self._depth:
            raise ValueError("latent choices live outside loops")
        if transform is None:
            transform = "log" if dist in _POSITIVE else ("logit" if dist in _UNIT else "identity")
        slot = self._slot()
        row = self.num_params
        self.num_params += 1
        self._step(nat.UT_STEP_CHOICE, d, args, value_source=row, transform=_TRANSFORMS[transform], binding_slot=slot)
        self.latents.append(_Latent(name, dist, row, 1, _TRANSFORMS[transform]))
        return self._node("slot", slot)

    def latent_iid_normal(self, name: str, size: int, mu, sigma) -> int:
        """`size` latent rows ~ normal(mu, sigma) (DeviceDiagNormalChoiceStepDyn);
        returns the first row."""
        row = self.num_params
        self.num_params += int(size)
        self._step(nat.UT_STEP_IID_NORMAL, 0, (mu, sigma), value_source=row, count=int(size))
        self.latents.append(_Latent(name, "normal", row, int(size), nat.UT_TRANSFORM_IDENTITY))
        return row

    def observe(self, dist: str, *args, row: int = 0, bind: bool = False):
        """An observed choice: the staged value at `row` of the current block
        scored by `dist`; with bind=True the value is returned as an Expr."""
        d = self._dist(dist, args)
        slot = self._slot() if bind else -1
        self._step(nat.UT_STEP_CHOICE, d, args, value_source=-1, obs_offset=int(row), binding_slot=slot)
        return self._node("slot", slot) if bind else None

    def deterministic(self, value) -> Expr:
        """slot = value (DeviceDeterministicStep)."""
        slot = self._slot()
        self._step(nat.UT_STEP_DETERMINISTIC, 0, (value,), binding_slot=slot)
        return self._node("slot", slot)

    @contextlib.contextmanager
    def loop(self, count: int, width: int, offset: int = 0, start: int = 1):
        """`count` iterations over blocks of `width` staged rows starting at
        row `offset` of the enclosing block; yields the iterator (start + t)."""
        slot = self._slot()
        at = self._step(nat.UT_STEP_LOOP, count=int(count), width=int(width), obs_offset=int(offset),
                        iterator_slot=slot, iterator_start=int(start))
        self._depth += 1
        try:
            yield self._node("slot", slot)
        finally:
            self._depth -= 1
            self.steps[at]["body"] = len(self.steps) - at - 1

    def glm_bernoulli_logit(self, coef_row: int, num_coefs: int, num_obs: int, intercept=None, offset: int = 0):
        """num_obs observations, each num_coefs covariates then y, y ~
        bernoullilogit(intercept + x . beta) with beta = rows coef_row ...
        (DeviceBernoulliLogitGLMChoiceStep[Dyn] in its DeviceLoopStep)."""
        args = (intercept,) if intercept is not None else ()
        self._step(nat.UT_STEP_GLM_BERNOULLI_LOGIT, 0, args, value_source=int(coef_row), obs_offset=int(offset),
                   count=int(num_obs), width=int(num_coefs))

    # ---- C form ------------------------------------------------------------
    def c_arrays(self):
        steps = (nat.ProgramStep * len(self.steps))()
        for i, s in enumerate(self.steps):
            st = steps[i]
            for k, v in s.items():
                if k == "arg":
                    for j in range(4):
                        st.arg[j] = v[j]
                else:
                    setattr(st, k, v)
        nodes = (nat.ExprNode * max(len(self.nodes), 1))()
        for i, (op, a, b, v) in enumerate(self.nodes):
            nodes[i].op, nodes[i].a, nodes[i].b, nodes[i].value = op, a, b, v
        return steps, nodes


@dataclass
class LoweredProgram(Lowered):
    program: Program = None
    steps: object = None
    nodes: object = None


class ProgramModel(TeaModelSpec):
    """A model given as a step program plus its staged observation rows."""

    name = "program"

    def __init__(self, program: Program, observed, name: str = "program"):
        self.program = program
        self.observed = np.ascontiguousarray(np.asarray(observed, dtype=np.float32).reshape(-1))
        self.name = name

    def parameter_names(self, args=(), constraints=None):
        out = []
        for lat in self.program.latents:
            out += [lat.name] if lat.size == 1 else [f"{lat.name}[{i + 1}]" for i in range(lat.size)]
        return out

    def lower(self, args=(), constraints=None) -> LoweredProgram:
        steps, nodes = self.program.c_arrays()
        plan = nat.PlanDesc(family=nat.UT_FAMILY_PROGRAM, num_params=self.program.num_params,
                            num_obs=int(self.observed.size))
        empty = np.zeros(0, dtype=np.int32)
        return LoweredProgram(plan=plan, observed=self.observed, trip_counts=empty, loop_starts=empty,
                              num_params=self.program.num_params, program=self.program, steps=steps, nodes=nodes)

    def constrain(self, unconstrained, args=(), constraints=None):
        u = np.asarray(unconstrained, dtype=np.float64)
        out = u.copy()
        for lat in self.program.latents:
            sl = slice(lat.row, lat.row + lat.size)
            if lat.transform == nat.UT_TRANSFORM_LOG:
                out[..., sl] = np.exp(u[..., sl])
            elif lat.transform == nat.UT_TRANSFORM_LOGIT:
                out[..., sl] = 1.0 / (1.0 + np.exp(-u[..., sl]))
        return out

    def initial_positions(self, rng, num_chains, args=(), constraints=None, init_strategy="prior"):
        """init_strategy="uniform": every unconstrained coordinate from U[-2, 2)
        (init_robustness_batched.jl:40-48); "prior": the same uniform draw
        (a program's priors may depend on one another, so no ancestral
        sampling is attempted)."""
        P = self.program.num_params
        return rng.uniform(-2.0, 2.0, size=(num_chains, P))


def report(model: ProgramModel):
    """(supported, issues) of a program (device_lowering_report)."""
    lib = nat.load()
    steps, nodes = model.program.c_arrays()
    buf = ctypes.create_string_buffer(4096)
    status = lib.ut_program_report(steps, len(model.program.steps), nodes, len(model.program.nodes),
                                   model.program.num_slots, model.program.num_params, int(model.observed.size), buf,
                                   len(buf))
    return status == nat.UT_OK, [s for s in buf.value.decode().split("\n") if s]
