import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "dig-appolo_b200"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


class OracleParams:
    """Case controls in the field layout of DsmcCaseParams, for the oracle."""

    def __init__(self, zones, inflow_dir, seed=0, nss=5000, nscheme=2000, nevery=1, nrepeat=100,
                 wall_stats=0, max_crossings=4096):
        self.nzones = len(zones)
        self.zone_tag = [z[0] for z in zones]
        self.zone_role = [z[1] for z in zones]
        self.zone_inject = [z[2] for z in zones]
        self.inflow_dir = tuple(inflow_dir)
        self.seed = seed
        self.nss, self.nscheme, self.nevery, self.nrepeat = nss, nscheme, nevery, nrepeat
        self.wall_stats = wall_stats
        self.max_crossings = max_crossings


@pytest.fixture(scope="session")
def block():
    import inputs as I
    raw, dm = I.block_mesh()
    mess = I.block_mess(dm, 20)
    return raw, dm, mess


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.load()
    return O
