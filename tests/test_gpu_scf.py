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


@pytest.mark.parametrize("open_diis", [False, True])
def test_incremental_scf_converges_on_the_water8_cluster(open_diis):
    """456 functions: every density-screened build adds an error of about 1e-8 Eh, more than the 1e-10 Eh
    convergence test allows, so the incremental SCF must finish on full builds (once |dE| < 1000 de_tol) and
    reach the plain SCF's energy instead of wandering until the iteration limit."""
    mol = W.water_cluster(nx=2, ny=2, nz=2, seed=W.SEED0 + 3650)
    sh = B.even_tempered(mol)
    kw = {"diis_fdmax": 1e6} if open_diis else {}
    plain = api.Engine(sh).rhf(mol)
    inc = api.Engine(sh).rhf(mol, incremental=True, **kw)
    assert plain["converged"] and inc["converged"]
    assert inc["incremental_builds"] > 0
    assert abs(plain["energy"] - inc["energy"]) <= E_TOL, (plain["energy"], inc["energy"])


def test_deterministic_scf_repeats_bit_for_bit():
    """With deterministic J/K builds (exact integer accumulation) the SCF's trajectory repeats: the 456-function
    water cluster, whose iteration count otherwise moves between runs with the FP64 atomics' rounding, gives the
    same energy bits and iteration count twice, and the plain SCF's energy to 1e-8 Eh; a batch handle does too."""
    mol = W.water_cluster(nx=2, ny=2, nz=2, seed=W.SEED0 + 3650)
    sh = B.even_tempered(mol)
    a = api.Engine(sh).rhf(mol, diis_fdmax=1e6, deterministic=True)
    b = api.Engine(sh).rhf(mol, diis_fdmax=1e6, deterministic=True)
    assert a["converged"] and b["converged"]
    assert a["energy"] == b["energy"] and a["iterations"] == b["iterations"]
    plain = api.Engine(sh).rhf(mol)
    assert abs(a["energy"] - plain["energy"]) <= E_TOL
    mols = [W.water(), W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)]
    shells = [B.even_tempered(m) for m in mols]
    r1 = api.BatchEngine(shells).rhf(mols, diis_fdmax=1e6, deterministic=True)
    r2 = api.BatchEngine(shells).rhf(mols, diis_fdmax=1e6, deterministic=True)
    assert [r["energy"] for r in r1] == [r["energy"] for r in r2]
    with pytest.raises(api.QcgError):
        api.Engine(sh).rhf(mol, deterministic=True, fp32_below=1e-7)
