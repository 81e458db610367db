"""Philox4x32-10 stream on the GPU (reference: src/device/rng.jl:95-219).

``philox4x32(key, counter)`` is the bijection; ``device_rand_uniform`` /
``device_rand_normal`` draw Float32 values at the coordinate
(chain_id, iteration, stream_id, draw_index), key = (chain_id, iteration),
counter = (stream_id, draw_index, 0, 0).  All computed by the library's
kernels.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat


def philox4x32_batch(keys, counters) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint32).reshape(-1, 2)
    counters = np.ascontiguousarray(counters, dtype=np.uint32).reshape(-1, 4)
    if keys.shape[0] != counters.shape[0]:
        raise IndexError("keys and counters must have the same number of rows")
    out = np.empty((keys.shape[0], 4), dtype=np.uint32)
    nat.check(nat.load().ut_philox4x32(nat.ptr(keys), nat.ptr(counters), keys.shape[0], nat.ptr(out)))
    return out


def philox4x32(key, counter):
    return tuple(int(v) for v in philox4x32_batch([key], [counter])[0])


def device_rand_uniform(chain_id, iteration, stream_id, draw_index, n=None) -> np.ndarray:
    count = 1 if n is None else int(n)
    out = np.empty(count, dtype=np.float32)
    nat.check(nat.load().ut_rand_uniform(chain_id, iteration, stream_id, draw_index, count, nat.ptr(out)))
    return out[0] if n is None else out


def device_rand_normal(chain_id, iteration, stream_id, draw_index, n=None) -> np.ndarray:
    count = 1 if n is None else int(n)
    out = np.empty(count, dtype=np.float32)
    nat.check(nat.load().ut_rand_normal(chain_id, iteration, stream_id, draw_index, count, nat.ptr(out)))
    return out[0] if n is None else out
