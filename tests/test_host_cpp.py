"""The C++ host layer (dig-appolo_b200/host/ProcessDSMCGpu.hpp), the
reference's ProcessDSMC interface over the C-ABI.

CPU: the header and tests/cpp/host_driver.cpp compile with g++ and link
against the built library.
GPU: the driver runs the block case through the reference's stage calls
(and through the fused step) and gives the same bits as the Python binding
of the same C-ABI; an invalid case raises DsmcError with the library's
message; out2dat and outBoundaryStressHeat write the Fluent files that the
library's writers make from the Python binding's fields and tallies (with
the zone declarations the host layer derives: cell zone 2 and one face zone
per run of equal face tags), and the wall fields follow outBoundaryStressHeat's
formula (src/ProcessDSMC.cpp:3494-3550) evaluated here on the downloaded
tallies.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import inputs as I
from gpu_util import make_case
from pydsmc import gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "dig-appolo_b200", "lib")


def _compile(out_dir):
    exe = os.path.join(out_dir, "host_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "dig-appolo_b200", "host"),
           os.path.join(ROOT, "tests", "cpp", "host_driver.cpp"), "-o", exe,
           "-L", LIB_DIR, "-ldsmcgpu", f"-Wl,-rpath,{LIB_DIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_hostpack_matches_the_serial_loops(tmp_path):
    """The threaded host loops of the particle upload and download
    (csrc/dsmc_hostpack.h) against serial restatements, every thread count,
    edge cases included (tests/cpp/hostpack_test.cpp)."""
    if not shutil.which("g++"):
        pytest.skip("no g++")
    exe = os.path.join(str(tmp_path), "hostpack_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-pthread",
           "-I", os.path.join(ROOT, "dig-appolo_b200", "csrc"),
           os.path.join(ROOT, "tests", "cpp", "hostpack_test.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_host_mesh_file_reads_the_reference_arrays(tmp_path):
    """The C++ host layer's MeshFile (readCAS + preprocess + DSMC topology
    through dsmc_mesh_read_cas) on the CPU: the 1/8 block mesh's arrays equal
    the reference's (tests/golden/mesh_pin.npz), the zone declarations its
    zonemap (fluent_pin.npz) and the mesh message the pinned restatement;
    a missing file raises DsmcError (tests/cpp/meshfile_driver.cpp)."""
    if not shutil.which("g++"):
        pytest.skip("no g++")
    if not os.path.exists(os.path.join(LIB_DIR, "libdsmcgpu.so")):
        pytest.skip("library not built")
    import inputs as I
    from conftest import golden
    from pydsmc import case as CS
    from pydsmc import mesh as M
    from pydsmc import meshio as IO
    exe = os.path.join(str(tmp_path), "meshfile_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "dig-appolo_b200", "host"),
           os.path.join(ROOT, "tests", "cpp", "meshfile_driver.cpp"), "-o", exe,
           "-L", LIB_DIR, "-ldsmcgpu", f"-Wl,-rpath,{LIB_DIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw, dm = I.block_mesh(scale=8)
    cas = str(tmp_path / "b8.cas")
    M.write_cas(cas, raw)
    r = subprocess.run([exe, cas, str(tmp_path), str(I.BLOCK_MA), str(I.BLOCK_KN), "20", str(I.BLOCK_L0)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
    assert "cannot open" in r.stdout
    g = golden("mesh_pin.npz")
    cells = np.fromfile(tmp_path / "cells.bin", dtype=M.DSMC_CELL_DTYPE)
    edges = np.fromfile(tmp_path / "edges.bin", dtype=M.DSMC_EDGE_DTYPE)
    for f in M.DSMC_CELL_DTYPE.names:
        if f != "no":
            assert np.array_equal(cells[f], g["cells"][f]), f
    for f in M.DSMC_EDGE_DTYPE.names:
        assert np.array_equal(edges[f], g["edges"][f]), f
    assert np.array_equal(np.fromfile(tmp_path / "points.bin"), g["points"])
    assert np.array_equal(np.fromfile(tmp_path / "split.bin", dtype=np.uint8), g["split"])
    zones = np.fromfile(tmp_path / "zones.bin", dtype=IO.ZONE_DTYPE)
    fz = golden("fluent_pin.npz")["zones"]
    assert [(int(z["id"]), int(z["first"]), int(z["last"])) for z in zones] == [tuple(t) for t in fz]
    mess = np.fromfile(tmp_path / "mess.bin", dtype=CS.MESH_MESSAGE_DTYPE)[0]
    want = CS.mesh_message(dm, I.BLOCK_MA, I.BLOCK_KN, ppc=20, L0=I.BLOCK_L0)
    for f in CS.MESH_MESSAGE_DTYPE.names:
        assert mess[f] == want[f], f


def test_host_layer_compiles_and_links(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("no g++")
    if not os.path.exists(os.path.join(LIB_DIR, "libdsmcgpu.so")):
        pytest.skip("library not built")
    exe = _compile(str(tmp_path))
    assert os.path.exists(exe)


def _write_case(d, dm, mess, params, x, v, ir, cell):
    with open(os.path.join(d, "case.txt"), "w") as f:
        f.write(f"{dm.ncell} {dm.nface} {dm.npoint} {len(cell)}\n")
    np.ascontiguousarray(dm.cells).tofile(os.path.join(d, "cells.bin"))
    np.ascontiguousarray(dm.edges).tofile(os.path.join(d, "edges.bin"))
    np.ascontiguousarray(dm.points, dtype=np.float64).tofile(os.path.join(d, "points.bin"))
    np.ascontiguousarray(dm.split, dtype=np.uint8).tofile(os.path.join(d, "split.bin"))
    np.ascontiguousarray(mess).tofile(os.path.join(d, "mess.bin"))
    with open(os.path.join(d, "params.bin"), "wb") as f:
        f.write(bytes(params))
    for k, a in (("x", x[:, 0]), ("y", x[:, 1]), ("z", x[:, 2]), ("vx", v[:, 0]), ("vy", v[:, 1]), ("vz", v[:, 2]),
                 ("ir", ir)):
        np.ascontiguousarray(a, dtype=np.float64).tofile(os.path.join(d, f"{k}.bin"))
    np.ascontiguousarray(cell, dtype=np.int32).tofile(os.path.join(d, "cell.bin"))


def _wall_fields(dm, mess, zones, tally, istep, nss):
    """outBoundaryStressHeat's conversion, src/ProcessDSMC.cpp:3494-3550."""
    role = {t: r for t, r, _ in zones}
    ts = float(mess["Neff"]) / (float(mess["dtime"]) * (istep - nss if istep > nss else 1.0))
    rows = []
    for f in range(dm.nface):
        e = dm.edges[f]
        if role.get(int(e["faceTag"]), 0) != gpu.ROLE_WALL:
            continue
        n = np.array(e["edgeNormal"], dtype=float)
        n = n / np.linalg.norm(n)
        ni = -n
        t = tally[f]
        pn = t[1:4] @ ni
        pt = t[1:4] - pn * ni
        scale = 2.0 * ts / float(e["length"]) / float(mess["n_ref"])
        p = pn * scale
        sh = -pt * scale
        rows.append([f, *n, p, *sh, *(p * n + sh), -t[4] * scale, -t[5] * scale, -(t[4] + t[5]) * scale])
    return np.array(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("fused", [0, 1])
def test_host_layer_matches_python_binding(block, tmp_path, fused):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=5)
    nsteps, nss = 6, 2
    params = gpu.default_params(precision=gpu.PRECISION_FP64, seed=17, zones=I.REF_ZONES, inflow_dir=I.inflow_dir(),
                                nss=nss, nscheme=3, nevery=1, nrepeat=2, wall_stats=1)
    d = str(tmp_path)
    _write_case(d, dm, mess, params, x, v, ir, cell)
    exe = _compile(d)
    r = subprocess.run([exe, d, str(nsteps), str(fused)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with make_case(dm, mess, seed=17, nss=nss, nscheme=3, nevery=1, nrepeat=2, wall_stats=1) as case:
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        for s in range(1, nsteps + 1):
            case.step(s)
        xg, vg, irg, cg = case.download_particles()
        local = case.macro(gpu.MACRO_LOCAL)
        record = case.macro(gpu.MACRO_RECORD)
        final = case.macro(gpu.MACRO_FINAL_RECORD)
        tally = case.wall()
        sparse_state = case.counts()["sparse_state"]
    n = len(cg)
    got = {k: np.fromfile(os.path.join(d, f"out_{k}.bin"), dtype=np.float64) for k in
           ("x", "y", "z", "vx", "vy", "vz", "ir")}
    assert np.array_equal(np.fromfile(os.path.join(d, "out_cell.bin"), dtype=np.int32), cg)
    assert np.array_equal(np.stack([got["x"], got["y"], got["z"]], 1), xg)
    assert np.array_equal(np.stack([got["vx"], got["vy"], got["vz"]], 1), vg)
    assert np.array_equal(got["ir"], irg)
    assert len(got["x"]) == n
    for k, ref in (("local", local), ("record", record), ("final", final)):
        assert np.array_equal(np.fromfile(os.path.join(d, f"out_{k}.bin")).reshape(ref.shape), ref, equal_nan=True), k
    # out2dat after NSS: final_record except for sparse cells
    o2d = np.fromfile(os.path.join(d, "out_out2dat.bin")).reshape(final.shape)
    sparse = (sparse_state == 1) | (sparse_state == 2)
    assert np.array_equal(o2d[~sparse], final[~sparse], equal_nan=True)
    assert np.array_equal(o2d[sparse], record[sparse], equal_nan=True)
    # Fluent files: the library's writers on the binding's fields and tallies
    from pydsmc import meshio as IO
    tags = dm.edges["faceTag"]
    runs = np.flatnonzero(np.diff(tags)) + 1
    bounds = np.concatenate([[0], runs, [dm.nface]])
    zones = [(12, 2, 1, dm.ncell)] + [(13, int(tags[a]), int(a) + 1, int(b)) for a, b in zip(bounds[:-1], bounds[1:])]
    IO.write_fluent_cells(os.path.join(d, "want_fluent.dat"), mess, zones, o2d)
    assert open(os.path.join(d, "out_fluent.dat"), "rb").read() == open(os.path.join(d, "want_fluent.dat"), "rb").read()
    IO.write_fluent_wall(os.path.join(d, "want_wall.dat"), mess, params, zones, dm.edges, tally, nsteps)
    # wall tallies are sums of atomic adds: two runs agree to rounding, so
    # the section structure is compared exactly and the numbers to 1e-12
    ga = open(os.path.join(d, "out_wall.dat")).read().splitlines()
    wa = open(os.path.join(d, "want_wall.dat")).read().splitlines()
    assert len(ga) == len(wa)
    for a, b in zip(ga, wa):
        if a.startswith("(") or a == "))":
            assert a == b
        else:
            assert np.allclose(np.array(a.split(), float), np.array(b.split(), float), rtol=1e-12, atol=1e-300)
    # the wall fields follow the reference's formula
    want = _wall_fields(dm, mess, I.REF_ZONES, tally, nsteps, nss)
    lines = open(os.path.join(d, "out_wall.dat")).read().splitlines()
    wz = [z for z in zones if z[1] == 6][0]
    k = lines.index(f"(300 (704 6 1 0 0 {wz[2]} {wz[3]})") + 2
    pressure = np.array([float(lines[k + j]) for j in range(wz[3] - wz[2] + 1)])
    assert np.allclose(pressure, want[:, 4], rtol=1e-13, atol=1e-300)
    assert (tally[:, 0] > 0).sum() > 0
    err = open(os.path.join(d, "out_error.txt")).read()
    assert "nzones" in err


@pytest.mark.gpu
def test_host_gsis_matches_python_binding(block, tmp_path):
    """ProcessGSISGpu::molecular_velocity_change between steps (gate on, a
    NaN cell) equals the Python binding's call on the same case."""
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=6)
    nsteps = 3
    params = gpu.default_params(precision=gpu.PRECISION_FP64, seed=23, zones=I.REF_ZONES, inflow_dir=I.inflow_dir(),
                                nss=2, nscheme=3, nevery=1, nrepeat=2)
    ns, acc, nan_cell = I.gsis_inputs(dm, mess, 20, seed=31)
    d = str(tmp_path)
    _write_case(d, dm, mess, params, x, v, ir, cell)
    ns.tofile(os.path.join(d, "ns.bin"))
    acc.tofile(os.path.join(d, "acc.bin"))
    exe = _compile(d)
    r = subprocess.run([exe, d, str(nsteps), "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with make_case(dm, mess, seed=23, nss=2, nscheme=3, nevery=1, nrepeat=2) as case:
        case.upload_particles(x, v, ir, cell)
        case.statistic_macroPre()
        for s in range(1, nsteps + 1):
            case.step(s)
        rep = case.molecular_velocity_change(ns, acc)
        case.step(nsteps + 1)
        xg, vg, irg, cg = case.download_particles()
    got = [int(t) for t in open(os.path.join(d, "out_gsis.txt")).read().split()]
    assert got == [rep[k] for k in ("nan_cell", "cells_updated", "cells_skipped", "added", "removed", "particles")]
    assert rep["nan_cell"] == nan_cell
    assert np.array_equal(np.fromfile(os.path.join(d, "out_cell.bin"), dtype=np.int32), cg)
    assert np.array_equal(np.fromfile(os.path.join(d, "out_vx.bin")), vg[:, 0])
    assert np.array_equal(np.fromfile(os.path.join(d, "out_x.bin")), xg[:, 0])
