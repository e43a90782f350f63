"""Particle upload on the B200 (dsmc_upload_particles through the C ABI).

Particles that arrive in cell-major order (the order of the reference's
per-cell buckets and of dsmc_download_particles) go to the device as they
are: a kernel checks the cell ids and lays out each cell's first slot, and
the mixed path converts positions to FP32 offsets from the cell centres on
the device. Any other order is sorted on the host (a stable counting sort by
cell). Both must leave the same particles in the same slots, from pageable
and from pinned host memory, in both precisions."""
import numpy as np
import pytest

import inputs as I
from gpu_util import make_case
from pydsmc import gpu

pytestmark = pytest.mark.gpu


def _interleaved(cell):
    """A permutation that mixes the cells but keeps each cell's particles in
    their order (a stable sort by cell restores the input)."""
    rank = np.zeros(len(cell), dtype=np.int64)
    starts = np.r_[0, np.flatnonzero(np.diff(cell)) + 1]
    for b, e in zip(starts, np.r_[starts[1:], len(cell)]):
        rank[b:e] = np.arange(e - b)
    return np.lexsort((cell, rank))


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out, t


@pytest.mark.parametrize("precision", [gpu.PRECISION_FP64, gpu.PRECISION_MIXED])
def test_cell_major_upload_equals_host_ordering(block, precision):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 30, seed=21)
    assert np.all(np.diff(cell) >= 0)
    perm = _interleaved(cell)
    cols = [x[:, 0], x[:, 1], x[:, 2], v[:, 0], v[:, 1], v[:, 2], ir]
    with make_case(dm, mess, precision=precision) as a, make_case(dm, mess, precision=precision) as b, \
            make_case(dm, mess, precision=precision) as c:
        a.upload_columns(*cols, cell)                               # cell-major, pageable
        b.upload_columns(*[col[perm] for col in cols], cell[perm])  # host ordering
        keep = [_pinned(np.ascontiguousarray(col)) for col in cols] + [_pinned(cell)]
        c.upload_columns(*[k[0] for k in keep])                     # cell-major, pinned
        ra, rb, rc = a.download_particles(), b.download_particles(), c.download_particles()
        for k in range(4):
            assert np.array_equal(ra[k], rb[k]) and np.array_equal(ra[k], rc[k]), k
        if precision == gpu.PRECISION_FP64:
            assert np.array_equal(ra[0], x) and np.array_equal(ra[1], v) and np.array_equal(ra[2], ir)
        else:
            assert np.array_equal(ra[0], I.fp32_positions(dm, x, cell))
            assert np.array_equal(ra[1], v.astype(np.float32).astype(np.float64))
        assert np.array_equal(ra[3], cell)
        # and the same steps from there
        for case in (a, b, c):
            case.step(1)
            case.step(2)
        assert np.array_equal(a.counts()["ppc"], b.counts()["ppc"])
        assert np.array_equal(a.counts()["ppc"], c.counts()["ppc"])
        ra, rb = a.download_particles(), b.download_particles()
        for k in range(4):
            assert np.array_equal(ra[k], rb[k]), k


def test_cell_major_upload_rejects_bad_cells(block):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 4, seed=22)
    bad = cell.copy()
    bad[-1] = dm.ncell          # still non-decreasing, out of range
    with make_case(dm, mess) as case:
        with pytest.raises(gpu.DsmcError, match="out of range"):
            case.upload_particles(x, v, ir, bad)
        case.upload_particles(x, v, ir, cell)
        assert case.particle_count() == len(cell)
