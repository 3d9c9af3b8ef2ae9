"""RHF on the GPU: the incremental (density-difference, density-screened) J/K path must converge to the same
energy as the plain all-FP64 path within 1e-8 Eh, and the plain path must match the CPU oracle."""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W
from tests.conftest import molecule_from

pytestmark = pytest.mark.gpu

E_TOL = 1e-8


def _pair(mol, shells):
    plain = api.Engine(shells).rhf(mol)
    chosen = api.Engine(shells).rhf(mol, incremental=True)
    assert plain["converged"] and chosen["converged"]
    assert chosen["incremental_builds"] > 0
    assert abs(plain["energy"] - chosen["energy"]) <= E_TOL, (plain["energy"], chosen["energy"])
    return plain, chosen


def test_incremental_water_config1():
    mol = W.water()
    _pair(mol, B.even_tempered(mol))


def test_incremental_water_dzvp(anchors, dzvp_text):
    mol = molecule_from(anchors["water"])
    plain, chosen = _pair(mol, B.read_gaussian94(dzvp_text, mol))
    assert abs((chosen["energy"] - anchors["water"]["energy"]) / anchors["water"]["energy"]) < 1e-5


def test_incremental_water_dimer():
    mol = W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)   # 114 functions
    _pair(mol, B.even_tempered(mol))


def test_incremental_rebuild_every_iteration_equals_plain_trajectory():
    mol = W.water()
    sh = B.even_tempered(mol)
    a = api.Engine(sh).rhf(mol)
    b = api.Engine(sh).rhf(mol, incremental=True, rebuild_every=0)
    assert b["incremental_builds"] == 0 and b["iterations"] == a["iterations"]
    assert abs(a["energy"] - b["energy"]) < 1e-12
