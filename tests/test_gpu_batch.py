"""Launch shapes, the autotuner and batched steps on the B200.

- The result of a step does not depend on the launch shape: the same case
  run with the default shape and with a different shape at every step gives
  the same bits (counter-based random streams keyed by particle, cell and
  pair, canonical particle order, cell-local collision state).
- The autotuner runs ordinary steps: a case that is autotuned for its first
  steps and then stepped on equals, bit for bit, the same case stepped with
  the default shape throughout.
- A batch of independent cases (different meshes, constants, precisions,
  seeds and particle counts) stepped together as one CUDA graph per step
  equals each case stepped on its own; cases keep their own step counts.
"""
import numpy as np
import pytest

import inputs as I
from gpu_util import make_case
from pydsmc import case as CS
from pydsmc import gpu

pytestmark = pytest.mark.gpu

SPECULAR = I.REF_ZONES + [(7, gpu.ROLE_SPECULAR, 0)]


def _state(case):
    xg, vg, irg, cg = case.download_particles()
    return {"x": xg, "v": vg, "ir": irg, "cell": cg, "record": case.macro(gpu.MACRO_RECORD),
            "local": case.macro(gpu.MACRO_LOCAL), "cs": case.cell_state(),
            "counters": {k: v for k, v in case.counters().items()}}


def _same(a, b):
    for k in ("x", "v", "ir", "cell"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("record", "local"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    for u, w in zip(a["cs"], b["cs"]):
        assert np.array_equal(u, w)
    for k in ("injected", "removed", "crossings", "candidate_pairs", "collisions", "wall_hits"):
        assert a["counters"][k] == b["counters"][k], k


SHAPES = [dict(move_threads=128, move_blocks_per_sm=3, sort_blocks_per_sm=1, collide_blocks_per_sm=1,
               stay_per_thread=1),
          dict(move_threads=128, move_blocks_per_sm=2, sort_blocks_per_sm=16, collide_blocks_per_sm=5,
               stay_per_thread=4),
          dict(move_threads=256, move_blocks_per_sm=32, sort_blocks_per_sm=3, collide_blocks_per_sm=9,
               stay_per_thread=2)]


@pytest.mark.parametrize("precision", [gpu.PRECISION_FP64, gpu.PRECISION_MIXED])
def test_results_do_not_depend_on_launch_shape(block, precision):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=6)
    out = []
    for vary in (False, True):
        with make_case(dm, mess, seed=31, precision=precision, zones=SPECULAR) as case:
            case.upload_particles(x, v, ir, cell)
            case.statistic_macroPre()
            for s in range(1, 7):
                if vary:
                    case.set_launch_shape(**SHAPES[s % len(SHAPES)])
                case.step(s)
            out.append(_state(case))
    _same(out[0], out[1])


def test_autotune_runs_ordinary_steps(block):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=7)
    with make_case(dm, mess, seed=41, precision=gpu.PRECISION_MIXED, zones=SPECULAR) as tuned:
        tuned.upload_particles(x, v, ir, cell)
        tuned.statistic_macroPre()
        nxt, shape = tuned.autotune(1, trial_steps=1)
        assert nxt > 10
        assert shape["move_threads"] in (128, 256)
        assert tuned.launch_shape() == shape
        for s in range(nxt, nxt + 2):
            tuned.step(s)
        a = _state(tuned)
    with make_case(dm, mess, seed=41, precision=gpu.PRECISION_MIXED, zones=SPECULAR) as plain:
        plain.upload_particles(x, v, ir, cell)
        plain.statistic_macroPre()
        for s in range(1, nxt + 2):
            plain.step(s)
        b = _state(plain)
    _same(a, b)


def _cases():
    """Four cases on the 1/4- and 1/8-resolution block meshes with different
    Mach and Knudsen numbers, fills, seeds and precisions."""
    raw4, dm4 = I.block_mesh(scale=4)
    raw8, dm8 = I.block_mesh(scale=8)
    out = []
    for k, (dm, ma, kn, ppc, prec) in enumerate([(dm4, 5.0, 0.1, 20, gpu.PRECISION_MIXED),
                                                  (dm8, 8.0, 0.05, 40, gpu.PRECISION_FP64),
                                                  (dm4, 3.0, 0.5, 10, gpu.PRECISION_FP64),
                                                  (dm8, 6.0, 0.02, 25, gpu.PRECISION_MIXED)]):
        mess = CS.mesh_message(dm, ma, kn, ppc=ppc, L0=I.BLOCK_L0)
        fill = I.fill_inputs(dm, mess, ppc, seed=50 + k)
        out.append((dm, mess, prec, 60 + k, fill))
    return out


def test_batch_continues_each_case_from_its_own_step():
    specs = _cases()
    alone = []
    for dm, mess, prec, seed, (x, v, ir, cell) in specs:
        with make_case(dm, mess, seed=seed, precision=prec, zones=SPECULAR) as case:
            case.upload_particles(x, v, ir, cell)
            case.statistic_macroPre()
            for s in range(1, 6):
                case.step(s)
            alone.append(_state(case))
    cases = []
    for dm, mess, prec, seed, (x, v, ir, cell) in specs:
        case = make_case(dm, mess, seed=seed, precision=prec, zones=SPECULAR)
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        cases.append(case)
    try:
        # case 0 takes steps 1 and 2 on its own, the others step 1; the batch
        # then advances everyone; the others then catch up on their own
        cases[0].step(1)
        cases[0].step(2)
        for c in cases[1:]:
            c.step(1)
        with gpu.Batch(cases) as batch:
            batch.step(2)          # case 0: steps 3, 4; others: 2, 3
            batch.step(1)          # case 0: 5; others: 4
            batch.sync()
        for c in cases[1:]:
            c.step(5)
        for c, want in zip(cases, alone):
            _same(_state(c), want)
    finally:
        for c in cases:
            c.close()
