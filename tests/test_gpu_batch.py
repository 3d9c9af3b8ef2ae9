"""Batched SCF (several molecules in one handle, one J/K build over all of them per iteration): every
molecule's J, K and converged energy must equal those of its own single-molecule handle, and those of the
CPU oracle (the oracle's direct J/K build and its plain SCF, which takes the same DIIS steps)."""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-10
E_TOL = 1e-8


def _density(n, nocc, seed):
    Q, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(n, nocc)))
    return 2 * Q @ Q.T


@pytest.fixture(scope="module")
def mols():
    ms = [W.water(), W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)] + W.random_molecules(3, max_atoms=6)
    return ms


def test_batch_jk_equals_single_builds(mols, oracle_mod):
    shells = [B.even_tempered(m) for m in mols]
    be = api.BatchEngine(shells)
    assert be.nmol == len(mols) and be.mol_nbf == [B.nbf(s) for s in shells]
    Ds = [_density(B.nbf(s), max(1, m.nelec // 2), 40 + k) for k, (m, s) in enumerate(zip(mols, shells))]
    J, K, st = be.fock_jk(Ds)
    total = 0
    for k, (s, D) in enumerate(zip(shells, Ds)):
        Js, Ks, sts = api.Engine(s).fock_jk(D)
        assert np.abs(J[k] - Js).max() <= FOCK_TOL and np.abs(K[k] - Ks).max() <= FOCK_TOL, k
        Jo, Ko, _ = oracle_mod.OracleBasis(s).jk_direct(D, 1e-10)
        assert np.abs(J[k] - Jo).max() <= FOCK_TOL and np.abs(K[k] - Ko).max() <= FOCK_TOL, k
        total += sts.quartets
    assert st.quartets == total


def test_batch_rhf_equals_single_rhf(mols, oracle_mod):
    shells = [B.even_tempered(m) for m in mols]
    res = api.BatchEngine(shells).rhf(mols)
    for m, s, r in zip(mols, shells, res):
        ref = api.Engine(s).rhf(m)
        assert r["converged"] == ref["converged"]
        if ref["converged"]:
            assert abs(r["energy"] - ref["energy"]) <= E_TOL
            assert abs(r["iterations"] - ref["iterations"]) <= 1   # same trajectory up to summation order
        orc = oracle_mod.OracleBasis(s).rhf(m)
        assert r["converged"] == orc["converged"]
        if orc["converged"]:
            assert abs(r["energy"] - orc["energy"]) <= E_TOL
            assert abs(r["iterations"] - orc["iterations"]) <= 1


def test_batch_rejects_single_molecule_only_calls(mols):
    be = api.BatchEngine([B.even_tempered(m) for m in mols[:2]])
    with pytest.raises(api.QcgError):
        be.one_electron(mols[0])
    with pytest.raises(api.QcgError):
        Engine_rhf = api.Engine.rhf
        Engine_rhf(be, mols[0])


def test_batch_rhf_from_per_molecule_guesses(mols):
    """Packed initial densities (one per molecule): started from each molecule's own converged density,
    every SCF of the batch stops within a few iterations at the energy of its single-molecule run, and a
    guess list of the wrong length is refused."""
    shells = [B.even_tempered(m) for m in mols]
    refs = [api.Engine(s).rhf(m, want_density=True) for m, s in zip(mols, shells)]
    keep = [k for k, r in enumerate(refs) if r["converged"]]
    ms, ss = [mols[k] for k in keep], [shells[k] for k in keep]
    res = api.BatchEngine(ss).rhf(ms, guesses=[refs[k]["D"] for k in keep])
    for k, r in zip(keep, res):
        assert r["converged"] and r["iterations"] <= 3, (k, r["iterations"])
        assert abs(r["energy"] - refs[k]["energy"]) <= E_TOL
    with pytest.raises(api.QcgError):
        api.BatchEngine(ss).rhf(ms, guesses=[refs[keep[0]]["D"]] * (len(keep) + 1))
