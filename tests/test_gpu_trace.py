"""Tracing parity on the B200: the move kernel's face-crossing trace
(dsmc_trace through the C ABI) against the reference's own tracing outputs
(tests/golden/trace_pin.npz) and the oracle.

FP64: final cell, ifout, first non-interface face and triangle, crossing
count, position and remaining dt are bit-exact. Mixed precision: cell ids and
hit faces agree for all particles whose decisions the FP32 guard could not
resolve only through its FP64 fallback; the mismatch rate must stay below
1e-4 (the FP32 positions carry ~1e-7 relative rounding the reference does not
have)."""
import numpy as np
import pytest

import inputs as I
from conftest import golden
from gpu_util import make_case, make_oracle
from pydsmc import gpu

pytestmark = pytest.mark.gpu


def test_fp64_trace_bit_exact_vs_reference(block):
    raw, dm, mess = block
    g = golden("trace_pin.npz")
    x, v, dt, cell = I.trace_inputs(dm, mess, len(g["cell_1"]), seed=1)
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
        for k in ("cell", "ifout", "face", "tri", "ncross"):
            assert np.array_equal(r[k], g[f"{k}_1"]), k
        assert np.array_equal(r["x"], g["x_1"])
        assert np.array_equal(r["dt"], g["dt_1"])
        r0 = case.trace(x, v, dt, cell, stop_at_wall=False)
        nowall = g["face_0"] < 0
        for k in ("cell", "ifout", "ncross"):
            assert np.array_equal(r0[k][nowall], g[f"{k}_0"][nowall]), k
        assert np.array_equal(r0["face"], g["face_0"])


def test_fp64_trace_bit_exact_vs_oracle_large(block):
    raw, dm, mess = block
    x, v, dt, cell = I.trace_inputs(dm, mess, 200_000, seed=7)
    o = make_oracle(dm, mess)
    ro = o.trace(x, v, dt, cell, stop_at_wall=True)
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross"):
        assert np.array_equal(r[k], ro[k]), k
    assert np.array_equal(r["x"], ro["x"])
    assert np.array_equal(r["dt"], ro["dt"])


def test_mixed_trace_matches_fp64(block):
    raw, dm, mess = block
    x, v, dt, cell = I.trace_inputs(dm, mess, 200_000, seed=8)
    # the reference is fed the FP32-rounded state the mixed path stores
    cc = dm.cells["cellXY"][cell]
    x32 = cc + (x - cc).astype(np.float32).astype(np.float64)
    v32 = v.astype(np.float32).astype(np.float64)
    o = make_oracle(dm, mess)
    ro = o.trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        r = case.trace(x32, v32, dt, cell, stop_at_wall=True)
        c = case.counters()
    mism = np.mean(r["cell"] != ro["cell"])
    assert mism <= 1e-4, mism
    assert np.mean(r["face"] != ro["face"]) <= 1e-4
    same = r["cell"] == ro["cell"]
    # positions agree to FP32 rounding relative to the cell size
    assert np.max(np.abs(r["x"][same] - ro["x"][same])) < 1e-4
    assert c["fp64_fallbacks"] > 0


@pytest.fixture(scope="module")
def capsule_small():
    return I.capsule_small()


def test_fp64_tet_trace_bit_exact_vs_reference(capsule_small):
    raw, dm, mess = capsule_small
    g = golden("tet_trace_pin.npz")
    x, v, dt, cell = I.tet_trace_inputs(dm, mess, len(g["cell"]), seed=4)
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross"):
        assert np.array_equal(r[k], g[k]), k
    assert np.array_equal(r["x"], g["x"])
    assert np.array_equal(r["dt"], g["dt"])


def test_tet_trace_large_fp64_exact_mixed_close(capsule_small):
    raw, dm, mess = capsule_small
    x, v, dt, cell = I.tet_trace_inputs(dm, mess, 200_000, seed=9)
    cc = dm.cells["cellXY"][cell]
    x32 = cc + (x - cc).astype(np.float32).astype(np.float64)
    v32 = v.astype(np.float32).astype(np.float64)
    o = make_oracle(dm, mess)
    ro = o.trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess) as case:
        r64 = case.trace(x32, v32, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross"):
        assert np.array_equal(r64[k], ro[k]), k
    assert np.array_equal(r64["x"], ro["x"])
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        r = case.trace(x32, v32, dt, cell, stop_at_wall=True)
    assert np.mean(r["cell"] != ro["cell"]) <= 1e-4
    assert np.mean(r["face"] != ro["face"]) <= 1e-4
