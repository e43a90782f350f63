"""Helpers shared by the GPU tests: build a GPU case and the matching oracle
with the same controls."""
import numpy as np

import inputs as I
from conftest import OracleParams
from pydsmc import gpu


def make_case(dm, mess, zones=None, precision=gpu.PRECISION_FP64, seed=0, capacity=0, **kw):
    zones = I.REF_ZONES if zones is None else zones
    p = gpu.default_params(precision=precision, seed=seed, capacity=capacity, zones=zones,
                           inflow_dir=I.inflow_dir(), **kw)
    return gpu.Case(dm, mess, p, device=0)


def make_oracle(dm, mess, zones=None, seed=0, **kw):
    from oracle import oracle as O
    zones = I.REF_ZONES if zones is None else zones
    return O.Oracle(dm, mess, OracleParams(zones, I.inflow_dir(), seed=seed, **kw))


def rel_close(a, b, rtol, atol=0.0):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))
