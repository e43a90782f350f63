"""Cases built from the native CAS reader, and the device-side field
writers, on the B200.

- A case created from dsmc_mesh_read_cas's arrays and case constants steps
  bit for bit like the case built from the pinned Python builder.
- dsmc_out2dat writes the Fluent file dsmc_write_fluent_cells makes from the
  downloaded record (up to NSS) or final_record (after; record for sparse
  cells), and dsmc_out_boundary_stress_heat the file dsmc_write_fluent_wall
  makes from the downloaded wall tallies (nothing when wall statistics are
  off).
"""
import os

import numpy as np
import pytest

import inputs as I
from gpu_util import make_case
from pydsmc import gpu
from pydsmc import mesh as M
from pydsmc import meshio as IO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cas_case(tmp_path_factory):
    raw, dm = I.block_mesh()
    p = str(tmp_path_factory.mktemp("cas") / "b4.cas")
    M.write_cas(p, raw)
    mf = IO.MeshFile(p)
    return mf, dm


def test_case_from_the_native_reader_steps_like_the_builder(cas_case):
    mf, dm = cas_case
    mess_py = I.block_mess(dm, 20)
    mess_io = mf.message(I.BLOCK_MA, I.BLOCK_KN, ppc=20, L0=I.BLOCK_L0)
    dmf = mf.dsmc_mesh()
    x, v, ir, cell = I.fill_inputs(dm, mess_py, 20, seed=21)
    out = []
    for mesh, mess in ((dm, mess_py), (dmf, mess_io)):
        with make_case(mesh, mess, seed=5, precision=gpu.PRECISION_MIXED) as case:
            case.upload_particles(x, v, ir, cell)
            case.statistic_macroPre()
            for s in range(1, 4):
                case.step(s)
            out.append(case.download_particles() + (case.macro(gpu.MACRO_LOCAL),))
    for a, b in zip(*out):
        assert np.array_equal(a, b, equal_nan=True)


def test_device_writers_match_the_host_writers(cas_case, tmp_path):
    mf, dm = cas_case
    zones = mf.zones()
    mess = mf.message(I.BLOCK_MA, I.BLOCK_KN, ppc=20, L0=I.BLOCK_L0)
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=22)
    nss = 3
    params = gpu.default_params(precision=gpu.PRECISION_FP64, seed=9, zones=I.REF_ZONES, inflow_dir=I.inflow_dir(),
                                nss=nss, nscheme=2, nevery=1, nrepeat=2, wall_stats=1)
    case = gpu.Case(mf.dsmc_mesh(), mess, params, device=0)
    try:
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        for s in range(1, 7):
            case.step(s)
            if s in (2, 6):                      # before and after NSS
                got = str(tmp_path / f"o{s}.dat")
                IO.out2dat(case, s, zones, got)
                rec = case.macro(gpu.MACRO_RECORD)
                if s > nss:
                    fin = case.macro(gpu.MACRO_FINAL_RECORD)
                    st = case.counts()["sparse_state"]
                    use = (st == 1) | (st == 2)
                    rec = np.where(use[:, None], rec, fin)
                want = str(tmp_path / f"w{s}.dat")
                IO.write_fluent_cells(want, mess, zones, rec)
                assert open(got, "rb").read() == open(want, "rb").read()
        got = str(tmp_path / "wall.dat")
        IO.out_boundary_stress_heat(case, 6, zones, got)
        tally = case.wall()
        assert (tally[:, 0] > 0).any()
        want = str(tmp_path / "wall_want.dat")
        IO.write_fluent_wall(want, mess, params, zones, dm.edges, tally, 6)
        assert open(got, "rb").read() == open(want, "rb").read()
    finally:
        case.close()
    # wall statistics off: nothing written (the reference's build)
    with make_case(mf.dsmc_mesh(), mess, seed=9) as case:
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        case.step(1)
        none = str(tmp_path / "none.dat")
        IO.out_boundary_stress_heat(case, 1, zones, none)
        assert not os.path.exists(none)
