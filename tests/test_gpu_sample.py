"""Sampling on the B200 against the reference's own statistic_macro
(tests/golden/sample_pin.npz, made by oracle/_ref/ref_harness's "sample"
command).

5,200 steps of a particle sequence with no random draws (inputs.sampled_at:
thinned and rescaled particles; cells that hold one particle on two steps
of each 100-step window), sampled by the library's statistic_macro stage
alone: local (exponential window past NSCHEME), record (the GSIS window,
with the sparse-cell state machine), final_record (steady average past
NSS), the window samples and validity and the sparse states equal the
reference's. The second pass writes the host's sparse-state decisions back
after every exchange step through dsmc_upload_sparse_state (the
write-back of ProcessGSIS::DSMC2NS, src/ProcessGSIS.cpp:1660-1674; the
harness's host rule stands in for its decisions), as the coupled loop does.
"""
import numpy as np
import pytest

import inputs as I
from conftest import golden
from gpu_util import make_case
from pydsmc import gpu

pytestmark = pytest.mark.gpu

STAGE_SAMPLE = 0x10


@pytest.mark.parametrize("pre", ["", "rule_"])
def test_sampling_and_sparse_write_back_match_the_reference(pre):
    g = golden("sample_pin.npz")
    raw, dm = I.block_mesh(scale=8)
    ppc = int(g["ppc"])
    mess = I.block_mess(dm, ppc)
    x, v, ir, cell = I.fill_inputs(dm, mess, ppc, int(g["seed"]))
    with make_case(dm, mess, nss=5000, nscheme=2000, nevery=1, nrepeat=100) as case:
        # the reference's statistic_macroPre runs on empty buckets
        case.upload_particles(x[:0], v[:0], ir[:0], cell[:0])
        case.statistic_macroPre()
        for k in range(1, int(g["steps"]) + 1):
            keep, s = I.sampled_at(k, cell, ppc)
            case.upload_particles(x[keep], v[keep] * s, ir[keep] * (s * s), cell[keep])
            case.step(k, STAGE_SAMPLE)
            if pre and k % 100 == 0:
                case.set_sparse_state(I.host_sparse_rule(case.counts()["sparse_state"], k))
        for name, which in (("local", gpu.MACRO_LOCAL), ("record", gpu.MACRO_RECORD),
                            ("final_record", gpu.MACRO_FINAL_RECORD)):
            assert np.array_equal(case.macro(which), g[pre + name]), pre + name
        cn = case.counts()
        assert np.array_equal(cn["window_samples"], g[pre + "window_samples"])
        assert np.array_equal(cn["window_valid"], g[pre + "window_valid"].astype(cn["window_valid"].dtype))
        assert np.array_equal(cn["sparse_state"], g[pre + "sparse_state"])
    if pre:
        assert (g["rule_sparse_state"] == 2).sum() > 5


def test_mixed_sampling_sums_every_particle_once(block):
    """Mixed path: every cell's 18 raw moments are the sums over exactly its
    particles (ragged cells, empty ones and cells longer than a warp
    included), within FP64 rounding of numpy's sums of the same FP32
    state."""
    raw, dm, mess = block
    x, v, ir, cell = I.ragged(I.fill_inputs(dm, mess, 70, seed=41), dm.ncell, 70, seed=42)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED, keep_step_moments=1) as case:
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        case.step(1, STAGE_SAMPLE)
        got = case.step_moments()
    vf = v.astype(np.float32).astype(np.float64)
    irf = ir.astype(np.float32).astype(np.float64)
    X, Y, Z = vf[:, 0], vf[:, 1], vf[:, 2]
    v2 = X * X + Y * Y + Z * Z
    terms = np.stack([np.ones_like(X), X, Y, Z, v2, X * X, X * Y, Y * Y, Y * Z, Z * Z, Z * X,
                      X * v2, Y * v2, Z * v2, irf, X * irf, Y * irf, Z * irf], 1)
    want = np.zeros((dm.ncell, 18))
    np.add.at(want, cell, terms)
    assert (want[:, 0] == 0).any() and want[:, 0].max() > 32      # empty cells and cells over a warp
    assert np.array_equal(got[:, 0], want[:, 0])
    scale = np.abs(terms).max(0) * np.maximum(want[:, :1], 1.0)
    assert np.all(np.abs(got - want) <= 1e-12 * scale)


def test_mixed_full_step_moments_sum_every_particle_once(block):
    """Mixed path, full steps: the moments the sampling pass folds (made by
    the collide pass for the cells it staged, summed from the particles for
    the others) are the sums over exactly each cell's particles after the
    step, within FP64 rounding of numpy's sums of the same FP32 state."""
    raw, dm, mess = block
    x, v, ir, cell = I.ragged(I.fill_inputs(dm, mess, 70, seed=43), dm.ncell, 70, seed=44)
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED, keep_step_moments=1) as case:
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        for s in (1, 2):
            case.step(s)
        got = case.step_moments()
        _, vd, ird, celld = case.download_particles()
        c = case.counters()
    assert c["collisions"] > 0
    X, Y, Z = vd[:, 0], vd[:, 1], vd[:, 2]
    v2 = X * X + Y * Y + Z * Z
    terms = np.stack([np.ones_like(X), X, Y, Z, v2, X * X, X * Y, Y * Y, Y * Z, Z * Z, Z * X,
                      X * v2, Y * v2, Z * v2, ird, X * ird, Y * ird, Z * ird], 1)
    want = np.zeros((dm.ncell, 18))
    np.add.at(want, celld, terms)
    n = want[:, 0]
    assert (n > 16).sum() > 100 and (n <= 16).any()          # cells of the two-cell collide path and others
    assert np.array_equal(got[:, 0], n)
    scale = np.abs(terms).max(0) * np.maximum(want[:, :1], 1.0)
    assert np.all(np.abs(got - want) <= 1e-12 * scale)
