"""The warp-shared form of the direct J/K build (jk_warp_kernel) against the CPU oracle.

Every class is forced into the warp-shared form (qcg_set_jk_warp_classes, the team form off) and J and K are
checked at the Fock tolerance, 1e-10: on a basis of contracted random shells (contraction 1-3: lanes with
different primitive counts in one warp), on the config-1 water and on a four-water cluster, in a handle
holding two molecules, under density screening (an incremental SCF) and with a precision band.  Requests
the form does not serve (several ranks, the deterministic mode) fall back to the other forms and still
match.
"""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-10
ALL = (1 << 21) - 1


def _density(n, seed, nocc=6):
    return W.cluster_density(n, nocc=nocc, seed=seed)


def _warp_engine(shells):
    eng = api.Engine(shells)
    eng.set_jk_team_classes(0)
    eng.set_jk_warp_classes(ALL)
    return eng


@pytest.mark.parametrize("case", ["contracted_pool", "water", "water4"])
def test_warp_jk_matches_oracle(case, oracle_mod):
    if case == "contracted_pool":
        sh = W.shell_pool(6, seed=W.SEED0 + 3700, box=4.0)
    elif case == "water":
        sh = B.even_tempered(W.water())
    else:
        sh = B.even_tempered(W.water_cluster(nx=2, ny=2, nz=1, seed=W.SEED0 + 3600))
    ob = oracle_mod.OracleBasis(sh)
    D = _density(ob.nbf, W.SEED0 + 3711)
    eng = _warp_engine(sh)
    J, K, st = eng.fock_jk(D)
    Jr, Kr, cnt = ob.jk_direct(D)
    assert st.quartets == cnt
    assert np.abs(J - Jr).max() <= FOCK_TOL and np.abs(K - Kr).max() <= FOCK_TOL


def test_warp_jk_two_molecule_handle():
    mols = [W.water(), W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)]
    be = api.BatchEngine([B.even_tempered(m) for m in mols])
    Ds = [_density(B.nbf(B.even_tempered(m)), W.SEED0 + 3713 + k) for k, m in enumerate(mols)]
    be.set_jk_team_classes(0)
    be.set_jk_warp_classes(ALL)
    Js, Ks, _ = be.fock_jk(Ds)
    for m, D, J, K in zip(mols, Ds, Js, Ks):
        e = api.Engine(B.even_tempered(m))
        e.set_jk_warp_classes(0)
        Jr, Kr, _ = e.fock_jk(D)
        assert np.abs(J - Jr).max() <= FOCK_TOL and np.abs(K - Kr).max() <= FOCK_TOL


def test_warp_jk_incremental_scf_and_precision_band():
    """Density screening (skipped quartets inside a warp) through an incremental SCF, and a build split into
    an FP32 and an FP64 band, against the same runs in the thread-per-quartet form."""
    mol = W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)
    sh = B.even_tempered(mol)
    eng = _warp_engine(sh)
    ref = api.Engine(sh)
    ref.set_jk_warp_classes(0)
    a = eng.rhf(mol, incremental=True)
    b = ref.rhf(mol, incremental=True)
    assert a["converged"] and b["converged"] and abs(a["energy"] - b["energy"]) <= 1e-8
    D = _density(eng.nbf, W.SEED0 + 3714, nocc=10)
    eng.set_fp32_bound(1e-7)
    ref.set_fp32_bound(1e-7)
    J1, K1, _ = eng.fock_jk(D)
    J2, K2, _ = ref.fock_jk(D)
    assert np.abs(J1 - J2).max() <= 1e-10 and np.abs(K1 - K2).max() <= 1e-10


def test_warp_jk_falls_back_where_it_does_not_apply():
    sh = W.shell_pool(6, seed=W.SEED0 + 3700, box=4.0)
    eng = _warp_engine(sh)
    D = _density(eng.nbf, W.SEED0 + 3715)
    J, K, _ = eng.fock_jk(D)
    Jd, Kd, _ = eng.fock_jk(D, deterministic=True)   # deterministic: thread-per-quartet form
    assert np.abs(J - Jd).max() <= 1e-12 and np.abs(K - Kd).max() <= 1e-12
    Js, Ks = np.zeros_like(J), np.zeros_like(K)
    for r in range(2):                               # shards: thread-per-quartet form
        eng.set_shard(r, 2)
        Jr, Kr, _ = eng.fock_jk(D)
        Js += Jr
        Ks += Kr
    eng.set_shard(0, 1)
    assert np.abs(Js - J).max() <= 1e-10 and np.abs(Ks - K).max() <= 1e-10
    with pytest.raises(api.QcgError):
        eng.set_jk_warp_classes(1 << 21)
