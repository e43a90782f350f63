"""dsmc_trace_noalloc: the tracing check for callers that cannot allocate
device memory at the call site (a solver that reserved the whole GPU for its
own pool; a coupling loop that forbids allocation after start-up). It
stages its work in one static device array of the library instead of
allocating per call.

Its results must equal those of dsmc_trace on the same particles, on two
calls in a row (the second call reuses the array the first one left
behind), and the device's free memory must be the same before and after the
second call (the first one sets up the array's address and loads the
kernels). The file is named to run last, so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process, where its first call sets up the array's device address."""
import numpy as np
import pytest

import inputs as I
from gpu_util import make_case
from pydsmc import gpu

pytestmark = pytest.mark.gpu


def _free_device_bytes():
    import torch
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.parametrize("precision", [gpu.PRECISION_FP64, gpu.PRECISION_MIXED])
def test_noalloc_trace_equals_trace_on_two_calls(block, precision):
    raw, dm, mess = block
    with make_case(dm, mess, precision=precision) as case:
        for call, seed in enumerate((11, 12)):
            x, v, dt, cell = I.trace_inputs(dm, mess, gpu.NOALLOC_MAX_TRACE if call == 0 else 5000, seed=seed)
            ref = case.trace(x, v, dt, cell, stop_at_wall=True)
            free0 = _free_device_bytes() if call == 1 else None
            got = case.trace(x, v, dt, cell, stop_at_wall=True, noalloc=True)
            if call == 1:
                assert _free_device_bytes() == free0
            for k in ("cell", "ifout", "face", "tri", "ncross", "x", "v", "dt"):
                assert np.array_equal(got[k], ref[k]), (call, k)


def test_noalloc_trace_rejects_more_than_its_maximum(block):
    raw, dm, mess = block
    x, v, dt, cell = I.trace_inputs(dm, mess, gpu.NOALLOC_MAX_TRACE + 1, seed=3)
    with make_case(dm, mess) as case:
        with pytest.raises(gpu.DsmcError, match="DSMC_NOALLOC_MAX_TRACE"):
            case.trace(x, v, dt, cell, stop_at_wall=True, noalloc=True)
        # the handle stays usable after the rejection
        r = case.trace(x[:100], v[:100], dt[:100], cell[:100], stop_at_wall=True, noalloc=True)
        assert r["cell"].shape == (100,)
