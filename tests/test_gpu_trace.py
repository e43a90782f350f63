"""Tracing parity on the B200: the move kernel's face-crossing trace
(dsmc_trace through the C ABI) against the reference's own tracing outputs
(tests/golden/*trace*_pin.npz, made by oracle/_ref/ref_harness) and the
oracle.

FP64: final cell, ifout, first non-interface face and triangle, crossing
count, position and remaining dt are bit-exact.

Mixed precision, fed the FP32 state it stores (FP32 offsets from the cell
centre, FP32 velocities), against the reference / oracle fed the same state
widened to FP64: final cell, ifout, face, triangle, crossings and remaining
dt are bit-exact, and the stored position is the FP32 rounding of the
reference's position relative to the final cell's centre (the mixed trace
advances FP64 positions with the reference's own arithmetic; its FP32 plane
test only settles the exit searches whose answer it can prove).
"""
import numpy as np
import pytest

import inputs as I
from conftest import golden
from gpu_util import make_case, make_oracle
from pydsmc import gpu

pytestmark = pytest.mark.gpu

KEYS = ("cell", "ifout", "face", "tri", "ncross")


def _assert_mixed_equal(dm, r, ro):
    """A mixed trace against the FP64 reference on the same FP32 state."""
    for k in KEYS:
        assert np.array_equal(r[k], ro[k]), k
    assert np.array_equal(r["dt"], ro["dt"])
    kept = ro["cell"] >= 0
    assert np.array_equal(r["x"][kept], I.fp32_positions(dm, ro["x"][kept], ro["cell"][kept]))


def _fallback_rate(c, n):
    return c["fp64_fallbacks"] / max(1, n + c["crossings"])


def test_fp64_trace_bit_exact_vs_reference(block):
    raw, dm, mess = block
    g = golden("trace_pin.npz")
    x, v, dt, cell = I.trace_inputs(dm, mess, len(g["cell_1"]), seed=1)
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
        for k in KEYS:
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
    for k in KEYS:
        assert np.array_equal(r[k], ro[k]), k
    assert np.array_equal(r["x"], ro["x"])
    assert np.array_equal(r["dt"], ro["dt"])


def test_mixed_trace_bit_exact(block):
    raw, dm, mess = block
    x, v, dt, cell = I.trace_inputs(dm, mess, 200_000, seed=8)
    x32, v32 = I.fp32_state(dm, x, v, cell)
    ro = make_oracle(dm, mess).trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        r = case.trace(x32, v32, dt, cell, stop_at_wall=True)
        c = case.counters()
    _assert_mixed_equal(dm, r, ro)
    rate = _fallback_rate(c, len(cell))
    print(f"mixed block trace: {c['fp64_fallbacks']} FP64 scans in {len(cell) + c['crossings']} exit searches "
          f"({rate:.2e})")
    # the side faces (zone 7) have no role in the reference's table: every
    # search after such a hit is the FP64 scan, as in the reference
    assert 0 < c["fp64_fallbacks"] and rate < 0.1


@pytest.fixture(scope="module")
def capsule_small():
    return I.capsule_small()


def test_fp64_tet_trace_bit_exact_vs_reference(capsule_small):
    raw, dm, mess = capsule_small
    g = golden("tet_trace_pin.npz")
    x, v, dt, cell = I.tet_trace_inputs(dm, mess, len(g["cell"]), seed=4)
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
    for k in KEYS:
        assert np.array_equal(r[k], g[k]), k
    assert np.array_equal(r["x"], g["x"])
    assert np.array_equal(r["dt"], g["dt"])


def test_tet_trace_large_fp64_and_mixed_exact(capsule_small):
    raw, dm, mess = capsule_small
    x, v, dt, cell = I.tet_trace_inputs(dm, mess, 200_000, seed=9)
    x32, v32 = I.fp32_state(dm, x, v, cell)
    ro = make_oracle(dm, mess).trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess) as case:
        r64 = case.trace(x32, v32, dt, cell, stop_at_wall=True)
    for k in KEYS:
        assert np.array_equal(r64[k], ro[k]), k
    assert np.array_equal(r64["x"], ro["x"])
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        r = case.trace(x32, v32, dt, cell, stop_at_wall=True)
        c = case.counters()
    _assert_mixed_equal(dm, r, ro)
    rate = _fallback_rate(c, len(cell))
    print(f"mixed tet trace: FP64 scans in {rate:.2e} of exit searches")
    assert rate < 0.05


@pytest.fixture(scope="module")
def block_full():
    raw, dm = I.block_mesh(scale=1)
    return raw, dm, I.block_mess(dm, 20)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_trace_config_full_block(block_full, precision):
    """The TRACE configuration: 10^6 particles uniform in random cells of the
    full 48,640-cell block mesh, isotropic velocities at 3x the freestream
    speed, one dt. Every output array bit-exact with the reference's own
    tracing (SHA-256 digests of its outputs in trace_full_pin.npz), and the
    final per-cell counts equal."""
    raw, dm, mess = block_full
    g = golden("trace_full_pin.npz")
    assert dm.ncell == int(g["ncell"]) == 48640
    x, v, dt, cell = I.trace_inputs(dm, mess, int(g["n"]), seed=int(g["seed"]))
    prec = gpu.PRECISION_FP64
    if precision == "mixed":
        x, v = I.fp32_state(dm, x, v, cell)
        prec = gpu.PRECISION_MIXED
    with make_case(dm, mess, precision=prec) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
        c = case.counters()
    p = g["pick"]
    for k in KEYS + ("dt",):
        assert np.array_equal(r[k][p], g[f"{precision}_sample_{k}"]), k
        assert I.digest(r[k]) == str(g[f"{precision}_{k}_sha"]), k
    kept = r["cell"] >= 0
    assert np.array_equal(np.bincount(r["cell"][kept], minlength=dm.ncell), g[f"{precision}_ppc"])
    if precision == "fp64":
        assert I.digest(r["x"]) == str(g["fp64_x_sha"])
    else:
        ref_kept = g["mixed_sample_cell"] >= 0
        want = I.fp32_positions(dm, g["mixed_sample_x"][ref_kept], g["mixed_sample_cell"][ref_kept])
        assert np.array_equal(r["x"][p][ref_kept], want)
        assert I.digest(r["x"][kept]) == str(g["mixed_x_sha"])
        print(f"TRACE mixed: FP64 scans in {_fallback_rate(c, len(cell)):.2e} of exit searches")
    assert int(np.sum(r["face"] >= 0)) == int(g[f"{precision}_hits"])


def test_degenerate_traces_on_the_gpu(block, capsule_small):
    """Exact, degenerate paths (through face centres on the split diagonals,
    along edges, through vertices, from corners and faces, at rest, dt = 0,
    denormal speed, along a face): the FP64 trace bit-exact with the
    reference wherever its loop returns, the particles it spins on (split
    quads on role-less faces) lost at max_crossings as in the oracle; the
    same on the capsule tets. The mixed trace on the FP32-rounded inputs is
    bit-exact with the oracle on them."""
    raw, dm, mess = block
    g = golden("degenerate_trace_pin.npz")
    x, v, dt, cell = I.degenerate_trace_inputs(dm, mess, int(g["ncells"]), int(g["seed"]))
    ok, spins = g["ok"], g["spins"]
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
        c = case.counters()
    for k in KEYS + ("x", "dt"):
        assert np.array_equal(r[k][ok], g[k]), k
    assert c["lost"] == len(spins) and np.all(r["ncross"][spins] == 4096)
    ro = make_oracle(dm, mess).trace(x, v, dt, cell, stop_at_wall=True)
    for k in KEYS + ("x", "dt"):
        assert np.array_equal(r[k], ro[k]), k
    x32, v32 = I.fp32_state(dm, x, v, cell)
    ro32 = make_oracle(dm, mess).trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        rm = case.trace(x32, v32, dt, cell, stop_at_wall=True)
    _assert_mixed_equal(dm, rm, ro32)

    raw, dm, mess = capsule_small
    x, v, dt, cell = I.degenerate_tet_trace_inputs(dm, mess, int(g["tet_ncells"]), int(g["seed"]))
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
    for k in KEYS + ("x", "dt"):
        assert np.array_equal(r[k], g["tet_" + k]), k
    x32, v32 = I.fp32_state(dm, x, v, cell)
    ro32 = make_oracle(dm, mess).trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        rm = case.trace(x32, v32, dt, cell, stop_at_wall=True)
    _assert_mixed_equal(dm, rm, ro32)


@pytest.mark.parametrize("name", ["pyramid", "prism"])
def test_split_box_traces_on_the_gpu(name):
    """Pyramids and wedges (mixed triangle / quad faces): the FP64 trace
    bit-exact with the reference's (pyramid_trace_pin.npz, prism_pin.npz),
    the mixed trace on the FP32-rounded inputs bit-exact with the oracle."""
    import gen_golden as G
    raw, dm, mess = getattr(G, name + "_case")()
    g = golden("pyramid_trace_pin.npz" if name == "pyramid" else "prism_pin.npz")
    p = "" if name == "pyramid" else "trace_"
    tseed = 6 if name == "pyramid" else 7
    x, v, dt, cell = I.split_box_trace_inputs(raw, mess, len(g[p + "cell"]), seed=tseed)
    with make_case(dm, mess) as case:
        r = case.trace(x, v, dt, cell, stop_at_wall=True)
    for k in KEYS + ("x", "dt"):
        assert np.array_equal(r[k], g[p + k]), k
    x32, v32 = I.fp32_state(dm, x, v, cell)
    ro32 = make_oracle(dm, mess).trace(x32, v32, dt, cell, stop_at_wall=True)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
        rm = case.trace(x32, v32, dt, cell, stop_at_wall=True)
    _assert_mixed_equal(dm, rm, ro32)
