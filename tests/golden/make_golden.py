"""Generates tests/golden/reference_pins.json from the reference's own tests.

Reads (as text, at generation time only) the Philox4x32-10 known-answer
vectors of test/uncertaintea/core/device_rng.jl:77-87 and the ChEES scalar
pins of test/uncertaintea/core/batched_chees_adaptation.jl:50-72, and writes
them as a small JSON fixture that the test suite loads.  The GPU box never
needs the reference tree.

Usage: python tests/golden/make_golden.py <reference_root>   (a checkout of shohei81/uncertaintea)
"""
from __future__ import annotations

import json
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


def main(root: str) -> None:
    rng = open(os.path.join(root, "test/uncertaintea/core/device_rng.jl")).read()
    chees = open(os.path.join(root, "test/uncertaintea/core/batched_chees_adaptation.jl")).read()
    data = {
        "source": {"philox": "test/uncertaintea/core/device_rng.jl:77-87",
                   "chees": "test/uncertaintea/core/batched_chees_adaptation.jl:50-72"},
        "philox4x32_10_kat": parse_kat(rng),
        "chees": parse_chees(chees),
    }
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <checkout of shohei81/uncertaintea>")
    main(sys.argv[1])
