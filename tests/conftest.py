import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libqchem_b200.so")


@pytest.fixture(scope="session")
def anchors():
    with open(os.path.join(GOLDEN, "anchors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def dzvp_text():
    with open(os.path.join(GOLDEN, "dzvp_HNO.bsd")) as f:
        return f.read()


def molecule_from(anchor):
    from qchem_b200.basis import Molecule
    return Molecule(list(anchor["Z"]), np.array(anchor["R"], dtype=float))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
