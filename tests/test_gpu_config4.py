"""The random-molecule set (256 H/C/N/O chains, even-tempered bases): the GPU's plain SCF follows the oracle's
trajectory on two of its smallest molecules, one that converges late and one that does not converge in 100
iterations.  qchem's SCF loop (src/SCFIterator/Imp/SCFIterator.C) reports a run that reaches its iteration
limit as not converged; the GPU must report the same, with the same iteration count and the same energy at
the limit, rather than a converged result the oracle does not reach.  With the DIIS switch-on bound opened
(diis_fdmax) the GPU converges the same molecule to the variational minimum."""
import os

import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

# 57 basis functions each: index 33 converges at iteration 79, index 9 does not converge in 100 iterations
# (both in the oracle and on the GPU)
LATE, STUCK = 33, 9


@pytest.fixture(scope="module")
def molecules():
    return W.random_molecules(256)


@pytest.mark.parametrize("i", [LATE, STUCK])
def test_plain_scf_follows_the_oracle(i, molecules, oracle_mod):
    mol = molecules[i]
    sh = B.even_tempered(mol)
    ref = oracle_mod.OracleBasis(sh).rhf(mol, maxiter=100, nthreads=os.cpu_count() or 1)
    got = api.Engine(sh).rhf(mol, max_iter=100)
    assert got["converged"] == ref["converged"], (got["converged"], ref["converged"])
    assert got["iterations"] == ref["iterations"], (got["iterations"], ref["iterations"])
    # a converged run agrees at the SCF tolerance; a stuck one oscillates, and still agrees to 1e-6 Eh after
    # 100 iterations because both sides take the same DIIS steps
    tol = 1e-8 if ref["converged"] else 1e-6
    assert abs(got["energy"] - ref["energy"]) <= tol, (got["energy"], ref["energy"])


def test_open_diis_converges_the_stuck_molecule(molecules):
    mol = molecules[STUCK]
    sh = B.even_tempered(mol)
    plain = api.Engine(sh).rhf(mol, max_iter=100)
    opened = api.Engine(sh).rhf(mol, max_iter=100, diis_fdmax=1e6)
    assert not plain["converged"]
    assert opened["converged"] and opened["iterations"] < 30
    assert opened["energy"] < plain["energy"] - 1.0   # the stuck run sits > 3 Eh above the minimum


def test_open_diis_keeps_a_converging_molecule(molecules):
    mol = molecules[LATE]
    sh = B.even_tempered(mol)
    plain = api.Engine(sh).rhf(mol, max_iter=100)
    opened = api.Engine(sh).rhf(mol, max_iter=100, diis_fdmax=1e6)
    assert plain["converged"] and opened["converged"]
    assert abs(plain["energy"] - opened["energy"]) <= 1e-8


def test_dropped_overlap_mode_scf_matches_the_oracle(molecules, oracle_mod):
    """Molecule 34 (136 functions) has one near-null overlap mode behind a clean spectral gap, which the
    reference's default orthogonaliser drops.  The GPU SCF and the oracle both drop it, and with DIIS from the
    first iteration both converge to the same energy."""
    mol = molecules[34]
    sh = B.even_tempered(mol)
    ref = oracle_mod.OracleBasis(sh).rhf(mol, maxiter=60, nthreads=os.cpu_count() or 1, diis_fdmax=1e6)
    got = api.Engine(sh).rhf(mol, max_iter=60, diis_fdmax=1e6)
    assert ref["dropped_modes"] == 1
    assert ref["converged"] and got["converged"]
    assert abs(got["iterations"] - ref["iterations"]) <= 1
    assert abs(got["energy"] - ref["energy"]) <= 1e-8, (got["energy"], ref["energy"])
