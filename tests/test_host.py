"""Host-side logic: synthetic meshes, the CAS format, case constants, the
seeded workloads and the Python binding's argument handling (CPU only)."""
import os
import tempfile

import numpy as np
import pytest

import inputs as I
from pydsmc import case as C
from pydsmc import mesh as M
from pydsmc import workload as W


def test_block_case_mesh_sizes():
    raw = M.block_case_mesh(scale=1)
    assert raw.ncell == 48 * 32 * 32 - 8 ** 3 == 48640
    dm = M.build_dsmc_mesh(raw)
    # volumes sum to the box minus the block
    assert abs(dm.area_sum - (0.5 * 0.5 * 1.0 - (8 / 48) * (8 / 32) * (8 / 32) * 0.5 * 0.5)) < 1e-12
    # each hex has 6 faces; face normals point from c0 to c1
    assert np.all(dm.cells["num"] == 6)
    z = raw.zone
    assert (z == M.ZONE_WALL).sum() == 6 * 8 * 8
    assert (z == M.ZONE_INLET).sum() == 32 * 32 and (z == M.ZONE_OUTLET).sum() == 32 * 32


def test_normals_point_from_c0_to_c1():
    raw, dm = I.block_mesh()
    e = dm.edges
    c0, c1 = e["faceMap"][:, 4], e["faceMap"][:, 5]
    inner = c1 < dm.ncell
    d = dm.cells["cellXY"][c1[inner]] - dm.cells["cellXY"][c0[inner]]
    assert np.all((d * e["edgeNormal"][inner]).sum(1) > 0)
    # boundary normals point out of the gas
    bc = ~inner
    out = e["edgeCenter"][bc] - dm.cells["cellXY"][c0[bc]]
    assert np.all((out * e["edgeNormal"][bc]).sum(1) > 0)


def test_cas_writer_format():
    raw, dm = I.block_mesh(scale=8)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.cas")
        M.write_cas(p, raw)
        txt = open(p).read()
    assert txt.count("(13 (") == 1 + 5       # declaration + 5 face zones
    assert f"(12 (0 1 {raw.ncell:x} 0))" in txt
    assert "(13 (3 1 " in txt and "(13 (6 " in txt


def test_mesh_message_free_constants():
    raw, dm = I.block_mesh()
    a = C.mesh_message(dm, 5.0, 0.1, ppc=20, L0=0.125)
    b = C.mesh_message(dm, 5.0, 0.1, ppc=40, L0=0.125)
    assert a["Neff"] == 2 * b["Neff"]
    assert a["dtime"] == 0.2 * dm.min_edge
    c = C.mesh_message(dm, 5.0, 0.05, ppc=20, L0=0.125)
    assert c["n_ref"] > a["n_ref"]          # smaller Kn, denser gas
    assert C.inflow_direction(30.0) == (np.sqrt(3.0) / 2.0, 0.5)
    assert C.inflow_direction(0.0) == (1.0, 0.0)


def test_workload_generators():
    raw, dm = I.block_mesh()
    mess = I.block_mess(dm, 20)
    f = W.initial_fill(dm, mess, 5, 0, C.inflow_direction(30.0))
    assert f["x"].shape == (5 * dm.ncell, 3)
    lo = np.array([0.0, 0.0, 0.0])
    hi = np.array([1.0, 0.5, 0.5])
    assert np.all(f["x"] >= lo) and np.all(f["x"] <= hi)
    u, sig, tN = W.freestream(mess, C.inflow_direction(30.0))
    assert np.allclose(f["v"].mean(0), u, atol=5 * sig / np.sqrt(len(f["v"])))
    t = W.trace_particles(dm, mess, 1000, 1, C.inflow_direction(30.0))
    assert t["cell"].min() >= 0 and t["cell"].max() < dm.ncell


def test_batch_specs_follow_the_batched_configuration():
    import bench
    sp = bench.batch_specs(64, 0)
    assert sp == bench.batch_specs(64, 0)                    # seeded
    cells = [bench.batch_mesh_cells(s["k"]) for s in sp]
    assert min(cells) >= 4000 and max(cells) <= 90000        # log-uniform 5k-80k, rounded to even k
    assert all(20 <= s["ppc"] <= 200 and 3 <= s["Ma"] <= 10 and 0 <= s["aoa"] <= 40 for s in sp)
    assert all(0.01 <= s["Kn"] <= 1.0 for s in sp)
    dm, L0 = bench.batch_mesh(8)
    assert dm.ncell == bench.batch_mesh_cells(8)


def test_bench_reads_and_scales_profile_traffic(tmp_path, monkeypatch):
    """bench.py's roofline traffic: the summary of the benchmarked workload
    itself, else one of the same mesh at another particle count scaled by
    the particle ratio, else none."""
    import bench
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "move_kernel_meshA_ppc40.md").write_text("x\nparticles: 1000\ndram_bytes_per_launch: 5000\n")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    b, src = bench.measured_traffic("move_kernel", "meshA_ppc100", 2500.0)
    assert b == 12500.0 and "scaled by particles x2.500" in src
    (prof / "move_kernel_meshA_ppc100.md").write_text("dram_bytes_per_launch: 7000\n")
    b, src = bench.measured_traffic("move_kernel", "meshA_ppc100", 2500.0)
    assert b == 7000.0 and src == os.path.join("profiles", "move_kernel_meshA_ppc100.md")
    assert bench.measured_traffic("move_kernel", "meshB_ppc100", 2500.0) == (None, None)
    assert bench.measured_traffic("collide_kernel", "meshA_ppc100", 2500.0) == (None, None)
    # the workload's own summary with its particle count: scaled to the timed count
    (prof / "move_kernel_meshA_ppc100.md").write_text("dram_bytes_per_launch: 7000\nparticles: 2000\n")
    b, src = bench.measured_traffic("move_kernel", "meshA_ppc100", 2500.0)
    assert b == 8750.0 and "scaled by particles x1.250" in src


def test_bench_stage_rooflines():
    """Every stage with a byte model gets its algorithmic bytes over its
    event-timed stage time as a fraction of the peak; stages without one
    (inject) or without a time are left out."""
    import numpy as np
    import bench
    names = ["inject", "move", "sort", "collide", "sample"]
    kernels = {k: k + "_kernel" for k in names}
    ab = {"inject": None, "move": 2.0e9, "sort": 3.0e9, "collide": 1.0e9, "sample": 0.5e9}
    st = bench.stage_rooflines(ab, np.array([0.1, 2.0, 1.0, 0.0, 0.5]), names, kernels, 4000.0)
    assert set(st) == {"move", "sort", "sample"}
    assert st["move"]["achieved"] == 1000.0 and st["move"]["frac"] == 0.25
    assert st["sort"]["achieved"] == 3000.0 and st["sample"]["kernel"] == "sample_kernel"


def test_upload_columns_passes_what_upload_particles_passes():
    """pydsmc.gpu.Case.upload_columns (the bench's end-to-end upload) hands
    dsmc_upload_particles the same count and data as upload_particles, passes
    contiguous float64 columns without copying them, and refuses columns of
    unequal length; checked against a stand-in for the library."""
    import ctypes as C
    from pydsmc import gpu

    calls = []

    class FakeLib:
        def dsmc_upload_particles(self, h, n, *ptrs):
            cols = [np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n,)).copy() for p in ptrs[:7]]
            cell = np.ctypeslib.as_array(C.cast(ptrs[7], C.POINTER(C.c_int32)), shape=(n,)).copy()
            calls.append({"h": h, "n": n, "cols": cols, "cell": cell, "addr": [p.value for p in ptrs]})
            return 0

        def dsmc_destroy(self, h):
            pass

    case = gpu.Case.__new__(gpu.Case)
    case.lib, case.h = FakeLib(), 7
    rs = np.random.RandomState(0)
    n = 1000
    x, v = rs.standard_normal((n, 3)), rs.standard_normal((n, 3))
    ir, cell = rs.random_sample(n), rs.randint(0, 50, n).astype(np.int32)
    case.upload_particles(x, v, ir, cell)
    cols = [np.ascontiguousarray(x[:, k]) for k in range(3)] + [np.ascontiguousarray(v[:, k]) for k in range(3)]
    case.upload_columns(*cols, ir, cell)
    case.upload_columns(*(x[:, k] for k in range(3)), *(v[:, k] for k in range(3)), ir, cell)   # strided views
    a = calls[0]
    for b in calls[1:]:
        assert b["h"] == 7 and b["n"] == n
        assert all(np.array_equal(p, q) for p, q in zip(a["cols"], b["cols"]))
        assert np.array_equal(a["cell"], b["cell"])
    assert calls[1]["addr"] == [c.ctypes.data for c in cols] + [ir.ctypes.data, cell.ctypes.data]
    with pytest.raises(ValueError):
        case.upload_columns(*cols, ir[:-1], cell)
    assert len(calls) == 3
    case.h = None


def test_set_sparse_state_hands_over_one_byte_per_cell():
    """pydsmc.gpu.Case.set_sparse_state passes dsmc_upload_sparse_state one
    uint8 per cell, whatever integer type it is given, and refuses a wrong
    length; checked against a stand-in for the library."""
    import ctypes as C
    from pydsmc import gpu

    seen = []

    class FakeLib:
        def dsmc_upload_sparse_state(self, h, p):
            seen.append(np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(5,)).copy())
            return 0

        def dsmc_destroy(self, h):
            pass

    case = gpu.Case.__new__(gpu.Case)
    case.lib, case.h, case.ncell = FakeLib(), 3, 5
    case.set_sparse_state([0, 1, 2, 1, 0])
    case.set_sparse_state(np.array([2, 2, 0, 0, 1], dtype=np.int64))
    assert [s.tolist() for s in seen] == [[0, 1, 2, 1, 0], [2, 2, 0, 0, 1]]
    with pytest.raises(ValueError):
        case.set_sparse_state([0, 1])
    case.h = None
