import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
MOLS = ["formaldehyde", "benzene", "caffeine", "taxol", "ala25", "crambin"]
TOBOHR = 1.0 / 0.52917721092   # main.f90:99
TOKCAL = 627.509469           # main.f90:99


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        g = json.load(f)
    a = np.array(g["atoms"], dtype=np.float64)
    g["mol"] = dict(q=a[:, 0], x=a[:, 1] * TOBOHR, y=a[:, 2] * TOBOHR, z=a[:, 3] * TOBOHR,
                    r=a[:, 4] * TOBOHR)
    return g


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
