"""Generates tests/golden/reference_pins.json from the reference's own tests.

Reads (as text, at generation time only) the Philox4x32-10 known-answer
vectors of test/uncertaintea/core/device_rng.jl:77-87, the ChEES scalar
pins of test/uncertaintea/core/batched_chees_adaptation.jl:50-72 and the
scalar log-density pins of test/uncertaintea/core/dist_*.jl (each
`@test logpdf(family(args), x) ≈ closed form` and `== -Inf` line of the
families the step programs support, its closed form evaluated here), and
writes them as a small JSON fixture that the test suite loads.  The GPU box
never needs the reference tree.

Usage: python tests/golden/make_golden.py <reference_root>   (a checkout of shohei81/uncertaintea)
"""
from __future__ import annotations

import ast
import glob
import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_kat(text: str):
    block = text[text.index("kat = ["): text.index("for (key, ctr, expected) in kat")]
    words = [int(w, 16) for w in re.findall(r"0x([0-9a-fA-F]{8})", block)]
    assert len(words) == 3 * 10, len(words)
    out = []
    for i in range(3):
        w = words[10 * i: 10 * (i + 1)]
        out.append({"key": w[0:2], "counter": w[2:6], "expected": w[6:10]})
    return out


def parse_chees(text: str):
    pins = []
    for m in re.finditer(r"_chees_leapfrog_steps_from_jitter\(([-0-9.e]+), ([0-9]+) \* ([0-9.]+), ([0-9.]+)\) == ([0-9]+)",
                         text):
        pins.append({"jitter": float(m.group(1)), "trajectory_length": int(m.group(2)) * float(m.group(3)),
                     "step_size": float(m.group(4)), "steps": int(m.group(5))})
    hm = re.search(r"_chees_harmonic_mean_accept\(\[([0-9., ]+)\], Bool\[false, false, false\]\)", text)
    adam = re.search(r"_ChEESAdamState\(([0-9.]+), ([0-9.]+), ([0-9.]+), ([0-9.e-]+)\)", text)
    return {
        "steps_from_jitter": pins,
        "harmonic_mean_input": [float(v) for v in hm.group(1).split(",")],
        "harmonic_mean_expected": 3.0 / 7.0,
        "adam": {"learning_rate": float(adam.group(1)), "beta1": float(adam.group(2)), "beta2": float(adam.group(3)),
                 "epsilon": float(adam.group(4)), "constant_gradient": 2.0, "limit": 0.5, "atol": 1e-3},
    }


# the scalar families of the step programs, by the reference's constructor names
LOGPDF_FAMILIES = {"normal", "lognormal", "exponential", "gamma", "laplace", "cauchy", "halfnormal", "halfcauchy",
                   "logistic", "gumbel", "frechet", "rayleigh", "inversegaussian", "beta", "studentt",
                   "inversegamma", "weibull", "bernoulli", "poisson", "geometric", "negativebinomial", "binomial"}
_FUNCS = {"log": math.log, "exp": math.exp, "sqrt": math.sqrt, "log1p": math.log1p, "loggamma": math.lgamma,
          "pi": math.pi}
_NODES = (ast.Expression, ast.BinOp, ast.UnaryOp, ast.Call, ast.Name, ast.Constant, ast.Load, ast.Add, ast.Sub,
          ast.Mult, ast.Div, ast.Pow, ast.USub, ast.UAdd)


def eval_closed_form(expr: str, env: dict) -> float:
    """A Julia closed form of the reference's tests (numbers, + - * / ^,
    log / exp / sqrt / log1p / loggamma, pi, let-bound names) evaluated in
    float64; anything else is rejected."""
    e = expr.replace("UncertainTea.", "").replace("^", "**")
    e = re.sub(r"(?<![\w.])(\d+(?:\.\d*)?)(pi)\b", r"\1*\2", e)     # 2pi -> 2*pi
    tree = ast.parse(e.strip(), mode="eval")
    for node in ast.walk(tree):
        if not isinstance(node, _NODES):
            raise ValueError(f"unsupported syntax in {expr!r}")
        if isinstance(node, ast.Call) and not (isinstance(node.func, ast.Name) and node.func.id in _FUNCS):
            raise ValueError(f"unsupported call in {expr!r}")
    names = {**_FUNCS, **env}
    return float(eval(compile(tree, "<closed form>", "eval"), {"__builtins__": {}}, names))


_STMT = re.compile(r"@test\s+(?:UncertainTea\.logpdf|lp)\((?:UncertainTea\.)?(\w+)\(([^()]*)\),\s*([^()]+?)\)\s*"
                   r"(?:≈\s*(.+?)\s+(?:atol|rtol)\s*=\s*[0-9.eE+-]+|==\s*(-Inf))\s*$", re.S)


def parse_logpdf_pins(text: str, fname: str):
    """Every `@test logpdf(family(args), x) ≈ closed form` (or `== -Inf`) of a
    supported family in one test file, with `let` bindings substituted."""
    pins, envs, stmt, start = [], [{}], None, 0
    for no, line in enumerate(text.splitlines(), 1):
        s = line.strip()
        m = re.match(r"let (.+)$", s)
        if m:
            env = dict(envs[-1])
            for part in re.split(r",\s*(?=\w+\s*=)", m.group(1)):
                if "=" not in part:
                    continue
                k, v = part.split("=", 1)
                try:
                    env[k.strip()] = eval_closed_form(v, env)
                except (ValueError, SyntaxError, NameError):
                    env.pop(k.strip(), None)   # a value no closed form here needs (vectors, matrices)
            envs.append(env)
            continue
        if s == "end" and len(envs) > 1:
            envs.pop()
            continue
        if stmt is None and s.startswith("@test") and ("logpdf(" in s or "lp(" in s):
            stmt, start = s, no
        elif stmt is not None:
            stmt += " " + s
        if stmt is not None and (re.search(r"\b(atol|rtol)\s*=", stmt) or "-Inf" in stmt):
            m = _STMT.match(stmt)
            stmt_done, stmt = stmt, None
            if not m or m.group(1) not in LOGPDF_FAMILIES:
                continue
            env = envs[-1]
            try:
                args = [eval_closed_form(a, env) for a in m.group(2).split(",")]
                x = eval_closed_form(m.group(3), env)
                want = -math.inf if m.group(5) else eval_closed_form(m.group(4), env)
            except (ValueError, SyntaxError, NameError):
                continue
            pins.append({"family": m.group(1), "args": args, "x": x, "logpdf": want,
                         "source": f"test/uncertaintea/core/{fname}:{start}"})
    return pins


def main(root: str) -> None:
    rng = open(os.path.join(root, "test/uncertaintea/core/device_rng.jl")).read()
    chees = open(os.path.join(root, "test/uncertaintea/core/batched_chees_adaptation.jl")).read()
    data = {
        "source": {"philox": "test/uncertaintea/core/device_rng.jl:77-87",
                   "chees": "test/uncertaintea/core/batched_chees_adaptation.jl:50-72",
                   "logpdf": "test/uncertaintea/core/dist_*.jl (file:line per pin)"},
        "philox4x32_10_kat": parse_kat(rng),
        "chees": parse_chees(chees),
        "logpdf": [p for f in sorted(glob.glob(os.path.join(root, "test/uncertaintea/core/dist_*.jl")))
                   for p in parse_logpdf_pins(open(f).read(), os.path.basename(f))],
    }
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <checkout of shohei81/uncertaintea>")
    main(sys.argv[1])
