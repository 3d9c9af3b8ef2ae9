"""The team form of the direct J/K build (jk_team_kernel) against the CPU oracle.

Every class is forced into the team form (qcg_set_jk_team_classes) and J and K are checked at the Fock
tolerance, 1e-10: on a basis of contracted random shells (contraction 1-3, every class present), on the
config-1 water and on a four-water cluster, and in a handle holding two molecules.  Under
QCG_JK_DETERMINISTIC the team build repeats bit for bit, and it agrees with the thread-per-quartet form to
rounding.
"""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-10
ALL = (1 << 21) - 1


def _density(n, seed, nocc=6):
    return W.cluster_density(n, nocc=nocc, seed=seed)


@pytest.mark.parametrize("case", ["contracted_pool", "water", "water4"])
def test_team_jk_matches_oracle(case, oracle_mod):
    if case == "contracted_pool":
        sh = W.shell_pool(6, seed=W.SEED0 + 3700, box=4.0)
    elif case == "water":
        sh = B.even_tempered(W.water())
    else:
        sh = B.even_tempered(W.water_cluster(nx=2, ny=2, nz=1, seed=W.SEED0 + 3600))
    ob = oracle_mod.OracleBasis(sh)
    D = _density(ob.nbf, W.SEED0 + 3701)
    eng = api.Engine(sh)
    eng.set_jk_team_classes(ALL)
    J, K, st = eng.fock_jk(D)
    Jr, Kr, cnt = ob.jk_direct(D)
    assert st.quartets == cnt
    assert np.abs(J - Jr).max() <= FOCK_TOL and np.abs(K - Kr).max() <= FOCK_TOL


def test_team_jk_deterministic_and_equal_to_thread_form():
    sh = W.shell_pool(6, seed=W.SEED0 + 3700, box=4.0)
    eng = api.Engine(sh)
    n = eng.nbf
    D = _density(n, W.SEED0 + 3702)
    eng.set_jk_team_classes(ALL)
    J1, K1, _ = eng.fock_jk(D, deterministic=True)
    for _ in range(3):
        J2, K2, _ = eng.fock_jk(D, deterministic=True)
        assert np.array_equal(J1, J2) and np.array_equal(K1, K2)
    eng.set_jk_team_classes(0)
    J3, K3, _ = eng.fock_jk(D)
    eng.set_jk_team_classes(-1)
    assert np.abs(J1 - J3).max() <= 1e-12 and np.abs(K1 - K3).max() <= 1e-12


def test_team_jk_two_molecule_handle():
    mols = [W.water(), W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)]
    be = api.BatchEngine([B.even_tempered(m) for m in mols])
    Ds = [_density(B.nbf(B.even_tempered(m)), W.SEED0 + 3703 + k) for k, m in enumerate(mols)]
    be.set_jk_team_classes(ALL)
    Js, Ks, _ = be.fock_jk(Ds)
    for m, D, J, K in zip(mols, Ds, Js, Ks):
        e = api.Engine(B.even_tempered(m))
        e.set_jk_team_classes(0)
        Jr, Kr, _ = e.fock_jk(D)
        assert np.abs(J - Jr).max() <= FOCK_TOL and np.abs(K - Kr).max() <= FOCK_TOL
