"""Native mesh input and field output (include/dsmc_meshio.h), on the CPU.

- dsmc_mesh_read_cas reads a Fluent ASCII case into the DSMC arrays bit for
  bit as the reference's readCAS + preprocess + DSMC topology build them:
  against the reference's own arrays (tests/golden/mesh_pin.npz) and against
  the Python builder (pinned the same way) on the block meshes and the
  capsule tetrahedra; zone declarations as the reference's zonemap.
- The parser follows readCAS on the variants the format allows: mixed face
  zones (node count per line), upper-case hexadecimal, CR-LF line ends,
  blank and "(labels" lines, comments; broken files fail with a message.
- dsmc_mesh_message equals setMeshMessage / setParticleMessage (pinned
  Python restatement) for several cases.
- dsmc_write_fluent_cells writes the reference's out2Fluent_dsmc file byte
  for byte (tests/golden/fluent_pin.npz); dsmc_write_fluent_wall writes
  outBoundaryStressHeat's sections with its formula and zone selection.
"""
import os

import numpy as np
import pytest

import inputs as I
from conftest import golden
from pydsmc import case as CS
from pydsmc import gpu
from pydsmc import mesh as M
from pydsmc import meshio as IO


def _same_mesh(a, b):
    for f in M.DSMC_CELL_DTYPE.names:
        assert np.array_equal(a.cells[f], b.cells[f]), f
    for f in M.DSMC_EDGE_DTYPE.names:
        assert np.array_equal(a.edges[f], b.edges[f]), f
    assert np.array_equal(a.points, b.points)
    assert np.array_equal(a.split, b.split)


def _read(path):
    with IO.MeshFile(path) as mf:
        return mf.dsmc_mesh(), mf.zones()


@pytest.fixture(scope="module")
def block8_cas(tmp_path_factory):
    raw, dm = I.block_mesh(scale=8)
    p = str(tmp_path_factory.mktemp("cas") / "b8.cas")
    M.write_cas(p, raw)
    return p, raw, dm


def test_read_matches_the_reference_arrays(block8_cas):
    path, raw, dm = block8_cas
    mine, zones = _read(path)
    g = golden("mesh_pin.npz")
    for f in M.DSMC_CELL_DTYPE.names:
        if f == "no":
            continue
        assert np.array_equal(mine.cells[f], g["cells"][f]), f
    for f in M.DSMC_EDGE_DTYPE.names:
        assert np.array_equal(mine.edges[f], g["edges"][f]), f
    assert np.array_equal(mine.points, g["points"])
    assert np.array_equal(mine.split, g["split"])
    fz = golden("fluent_pin.npz")["zones"]
    assert [(int(z["id"]), int(z["first"]), int(z["last"])) for z in zones] == [tuple(r) for r in fz]
    assert zones["section"].tolist() == [12] + [13] * (len(zones) - 1)


@pytest.mark.parametrize("which", ["block4", "capsule"])
def test_read_matches_the_python_builder(tmp_path, which):
    raw, dm = I.block_mesh(scale=4) if which == "block4" else I.capsule_small()[:2]
    p = str(tmp_path / "m.cas")
    M.write_cas(p, raw)
    mine, _ = _read(p)
    _same_mesh(mine, dm)
    assert mine.area_sum == dm.area_sum and mine.min_edge == dm.min_edge and mine.bcnumber == dm.bcnumber


def _variant(text: str) -> str:
    """The same case written another legal way: the first face zone as a
    mixed zone (node count on each line), upper-case hexadecimal in the face
    lines, CR-LF line ends, blank lines, a labels section and comments."""
    out = ['(0 "variant")', "(45 (2 fluid fluid)())", ""]
    in_first = False
    done_first = False
    for line in text.splitlines():
        if line.startswith("(13 (") and not line.startswith("(13 (0") and not done_first:
            parts = line.split()
            parts[-1] = "0)("                     # face type 0: mixed
            out.append(" ".join(parts))
            in_first = True
            continue
        if in_first:
            if line.startswith("))"):
                in_first = False
                done_first = True
                out.append(line)
                continue
            out.append(line.upper())             # "3 a b c d e" keeps its count, digits go upper case
            continue
        if line.startswith("(13 (") and not line.startswith("(13 (0"):
            out.append(line)
            continue
        out.append(line)
        if line.startswith("(10 (0"):
            out.append("(10 (labels 1 2))")
            out.append("")
    return "\r\n".join(out) + "\r\n"


def test_read_accepts_the_format_variants(tmp_path, block8_cas):
    path, raw, dm = block8_cas
    v = _variant(open(path).read())
    p = str(tmp_path / "v.cas")
    with open(p, "w", newline="") as f:
        f.write(v)
    mine, zones = _read(p)
    _same_mesh(mine, dm)
    assert len(zones) == len(_read(path)[1])


def test_read_reports_broken_files(tmp_path, block8_cas):
    path, raw, dm = block8_cas
    with pytest.raises(IO.MeshIOError, match="cannot open"):
        IO.MeshFile(str(tmp_path / "missing.cas"))
    text = open(path).read()
    cut = text[: text.rindex("(13 (")]                 # the last face zone is missing
    p = str(tmp_path / "cut.cas")
    open(p, "w").write(cut)
    with pytest.raises(IO.MeshIOError, match="declared but not given"):
        IO.MeshFile(p)
    lines = text.splitlines()
    k = next(i for i, s in enumerate(lines) if s.startswith("(13 (3 "))
    node = lines[k + 1].split()
    node[1] = "fffff"                                   # a node beyond the declared ones
    lines[k + 1] = " ".join(node)
    p2 = str(tmp_path / "bad.cas")
    open(p2, "w").write("\n".join(lines) + "\n")
    with pytest.raises(IO.MeshIOError, match="node out of range"):
        IO.MeshFile(p2)


@pytest.mark.parametrize("ma,kn,ppc,L0", [(5.0, 0.1, 20, 0.125), (8.0, 0.01, 100, 3.912), (3.0, 1.0, 7, 1.0)])
def test_mesh_message_matches_the_reference(block8_cas, ma, kn, ppc, L0):
    path, raw, dm = block8_cas
    with IO.MeshFile(path) as mf:
        mine = mf.message(ma, kn, ppc=ppc, L0=L0)
    ref = CS.mesh_message(dm, ma, kn, ppc=ppc, L0=L0)
    for f in CS.MESH_MESSAGE_DTYPE.names:
        assert mine[f] == ref[f], f


def test_fluent_cells_writer_is_the_reference_byte_for_byte(tmp_path, block8_cas):
    from gen_golden import fluent_fields
    path, raw, dm = block8_cas
    g = golden("fluent_pin.npz")
    with IO.MeshFile(path) as mf:
        zones = mf.zones()
    out = str(tmp_path / "f.dat")
    IO.write_fluent_cells(out, g["mess"], zones, fluent_fields(dm.ncell))
    assert open(out, "rb").read() == g["text"].tobytes()
    # no cell zone with id 2: refused
    with pytest.raises(IO.MeshIOError, match="id 2"):
        IO.write_fluent_cells(out, g["mess"], zones[1:], fluent_fields(dm.ncell))


def _wall_rows(dm, mess, zones, tally, istep, nss):
    """outBoundaryStressHeat's conversion (src/ProcessDSMC.cpp:3494-3552)."""
    role = {t: r for t, r, _ in I.REF_ZONES}
    ts = float(mess["Neff"]) / (float(mess["dtime"]) * ((istep - nss) if istep > nss else 1.0))
    rows = {}
    for f in range(dm.nface):
        e = dm.edges[f]
        if role.get(int(e["faceTag"]), 0) != gpu.ROLE_WALL:
            continue
        n = np.array(e["edgeNormal"], dtype=float)
        n = n / np.sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])
        ni = -n
        ni = ni / np.sqrt(ni[0] * ni[0] + ni[1] * ni[1] + ni[2] * ni[2])
        t = tally[f]
        pn = t[1] * ni[0] + t[2] * ni[1] + t[3] * ni[2]
        pt = t[1:4] - pn * ni
        scale = 2.0 * ts / float(e["length"]) / float(mess["n_ref"])
        p = pn * scale
        sh = -pt * scale
        rows[f] = {700: p * n + sh, 701: -t[4] * scale, 702: -t[5] * scale, 703: n, 704: p, 705: sh,
                   706: -t[4] * scale + -t[5] * scale}
    return rows


def test_fluent_wall_writer_follows_the_reference_formula(tmp_path, block8_cas):
    path, raw, dm = block8_cas
    with IO.MeshFile(path) as mf:
        zones = mf.zones()
        mess = mf.message(I.BLOCK_MA, I.BLOCK_KN, ppc=20, L0=I.BLOCK_L0)
    rs = np.random.RandomState(3)
    tally = rs.standard_normal((dm.nface, 6))
    params = gpu.default_params(zones=I.REF_ZONES, nss=10)
    out = str(tmp_path / "w.dat")
    IO.write_fluent_wall(out, mess, params, zones, dm.edges, tally, 25)
    lines = open(out).read().splitlines()
    assert lines[0].startswith('(0 " (300 (var-id zone-id var-size')
    assert lines[1].startswith('(0 "DSMC normalized wall fields: 700 stress vector')
    want = _wall_rows(dm, mess, zones, tally, 25, 10)
    wall_zone = [z for z in zones if z["id"] == 6][0]
    first, last = int(wall_zone["first"]), int(wall_zone["last"])
    k = 2
    for var, width in ((700, 3), (701, 1), (702, 1), (703, 3), (704, 1), (705, 3), (706, 1)):
        assert lines[k] == f"(300 ({var} 6 {width} 0 0 {first} {last})" and lines[k + 1] == "("
        for j, f in enumerate(range(first - 1, last)):
            vals = np.atleast_1d(want[f][var])
            assert lines[k + 2 + j] == " ".join("%.16g" % x for x in vals)
        k += 2 + (last - first + 1)
        assert lines[k] == "))"
        k += 1
    assert k == len(lines)                               # only the all-wall zone is written
    # no wall zone: nothing written
    out2 = str(tmp_path / "none.dat")
    IO.write_fluent_wall(out2, mess, gpu.default_params(zones=I.NOWALL_ZONES), zones, dm.edges, tally, 25)
    assert not os.path.exists(out2)


def test_capsule_mesh_has_the_reference_cell_count():
    """The CAP mesh: the seeded jittered-lattice Delaunay fill around the
    capsule, brought to the reference mesh's 372,500 cells by splitting a
    few far-field cells; every cell keeps a positive volume, every face has
    one or two cells, and the body wall, inlets and outlets are all there."""
    from pydsmc import capsule
    raw = capsule.capsule_mesh(target_cells=capsule.CAP_CELLS)
    dm = M.build_dsmc_mesh(raw)
    assert dm.ncell == 372500 == raw.ncell
    assert np.all(dm.cells["area"] > 0)
    assert np.all(raw.c0 >= 0)
    tags = set(np.unique(dm.edges["faceTag"]).tolist())
    assert {3, 4, 5, 6} <= tags
    # the split cells lie in the far field: the body and its fine region are
    # those of the plain fill
    plain = capsule.capsule_mesh()
    assert plain.ncell < raw.ncell
    wall = dm.edges["faceTag"] == 6
    assert wall.sum() == int((M.build_dsmc_mesh(plain).edges["faceTag"] == 6).sum())


def test_morton_numbering_keeps_the_mesh_and_brings_neighbours_close():
    """Cells numbered along a Morton curve of their centroids (the bench's
    CAP mesh): the same cells and faces, renumbered; on a point lattice the
    order is the Z-order curve; neighbour ids lie closer in the numbering
    than in the triangulator's order."""
    from pydsmc import capsule
    g = np.stack(np.meshgrid(np.arange(4), np.arange(4), np.arange(4), indexing="ij"), -1).reshape(-1, 3)
    order = M.morton_order(g.astype(float))
    assert sorted(order.tolist()) == list(range(64))
    first = g[order[:8]]                                  # the first octant's 2x2x2 block, x fastest
    assert np.array_equal(first, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0],
                                  [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]])
    raw0 = capsule.capsule_mesh(h_fine=0.5, h_coarse=1.0)
    raw1 = capsule.capsule_mesh(h_fine=0.5, h_coarse=1.0, morton=True)
    dm0, dm1 = M.build_dsmc_mesh(raw0), M.build_dsmc_mesh(raw1)
    assert dm0.ncell == dm1.ncell and len(dm0.edges) == len(dm1.edges)
    assert np.isclose(dm0.cells["area"].sum(), dm1.cells["area"].sum(), rtol=1e-12)
    assert np.array_equal(np.sort(dm0.cells["area"]), np.sort(dm1.cells["area"]))

    def spread(dm):
        c2c = dm.cells["cell2cell"][:, :4]
        d = np.abs(c2c - np.arange(dm.ncell)[:, None])[c2c >= 0]
        return np.percentile(d, 90)
    assert spread(dm1) < spread(dm0)
