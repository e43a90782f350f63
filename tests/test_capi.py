"""The C-ABI library builds, loads and exports every entry point that
include/dsmc_gpu.h and include/dsmc_meshio.h declare (no GPU calls), and
the product fails loudly without its library or without a GPU."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in ("dsmc_gpu.h", "dsmc_meshio.h")]


def declared_symbols(headers=HEADERS):
    out = set()
    for h in headers:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        out |= set(re.findall(r"\b(dsmc_[a-zA-Z0-9_]+)\s*\(", txt))
    return sorted(out)


def test_header_declares_the_stage_entry_points():
    syms = declared_symbols()
    for s in ("dsmc_create", "dsmc_step", "dsmc_preprocesseffquad", "dsmc_advection", "dsmc_cache2chain",
              "dsmc_collisionDSMC", "dsmc_statistic_macro", "dsmc_statistic_macroPre", "dsmc_download_macro",
              "dsmc_download_counts", "dsmc_trace", "dsmc_destroy", "dsmc_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from pydsmc import gpu
    if not os.path.exists(gpu.lib_path()):
        import build as b  # dig-appolo_b200/build.py
        b.build()
    lib = ctypes.CDLL(gpu.lib_path())
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # the Python bindings cover the same sets
    from pydsmc import meshio
    assert sorted(gpu.EXPORTED) == declared_symbols(HEADERS[:1])
    assert sorted(meshio.EXPORTED) == declared_symbols(HEADERS[1:])
    assert set(os.listdir(os.path.join(ROOT, "include"))) == {"dsmc_gpu.h", "dsmc_meshio.h"}


def test_struct_layouts_match_header():
    from pydsmc import case, gpu, mesh
    assert mesh.DSMC_CELL_DTYPE.itemsize == 120
    assert mesh.DSMC_EDGE_DTYPE.itemsize == 88
    assert case.MESH_MESSAGE_DTYPE.itemsize == 344
    assert ctypes.sizeof(gpu.Counters) == 12 * 8


def test_default_params_are_the_reference_constants():
    from pydsmc import gpu
    p = gpu.default_params()
    assert (p.nss, p.nscheme, p.nevery, p.nrepeat, p.wall_stats) == (5000, 2000, 1, 100, 0)
    assert p.inflow_dir[0] == np.sqrt(3.0) / 2.0 and p.inflow_dir[1] == 0.5
    zones = {(p.zone_tag[i], p.zone_role[i], p.zone_inject[i]) for i in range(p.nzones)}
    assert zones == {(3, gpu.ROLE_INTERFACE, 0), (4, gpu.ROLE_INLET, 1), (5, gpu.ROLE_OUTLET, 0), (6, gpu.ROLE_WALL, 0)}


def _run_python(code: str):
    env = dict(os.environ)
    paths = [os.path.join(ROOT, "dig-appolo_b200"), os.path.join(ROOT, "tests", "golden"), ROOT]
    env["PYTHONPATH"] = os.pathsep.join(paths + [env.get("PYTHONPATH", "")])
    return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, env=env)


def test_product_fails_loudly_without_its_library():
    r = _run_python("from pydsmc import gpu\n"
                    "gpu.LIB_PATH = '/nonexistent/libdsmcgpu.so'\n"
                    "gpu.load()\n")
    assert r.returncode != 0
    assert "OSError" in r.stderr and "not built" in r.stderr


def test_case_creation_reports_a_missing_gpu():
    """Where no GPU can be used, dsmc_create returns the CUDA runtime's error
    and the binding raises it; nothing falls back to the CPU."""
    if not os.path.exists(os.path.join(ROOT, "dig-appolo_b200", "lib", "libdsmcgpu.so")):
        pytest.skip("library not built")
    r = _run_python("import torch\n"
                    "if torch.cuda.is_available(): raise SystemExit(3)\n"
                    "import inputs as I\n"
                    "from pydsmc import gpu\n"
                    "raw, dm = I.block_mesh(scale=8)\n"
                    "mess = I.block_mess(dm, 5)\n"
                    "try:\n"
                    "    gpu.Case(dm, mess, gpu.default_params(), device=0)\n"
                    "except gpu.DsmcError as e:\n"
                    "    print('DsmcError', e)\n"
                    "    raise SystemExit(0)\n"
                    "raise SystemExit(1)\n")
    if r.returncode == 3:
        pytest.skip("a GPU is available here")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dsmc_create failed" in r.stdout and "cuda" in r.stdout.lower()
