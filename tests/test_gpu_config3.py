"""The 32-water cluster's direct J/K build (1824 functions, 928 shells) against the CPU oracle on slices.

A whole-build oracle run at this size is days of CPU time, so both sides evaluate the same slice: a seeded
random 3% of the shell pairs (qcg_set_pair_subset on the GPU, the oracle's subset build on the CPU), and every
Schwarz-screened quartet whose two pairs are both in it -- more than 10^7 quartets of every class.  J and K
must agree to the Fock tolerance, 1e-10 absolute.
"""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-10


@pytest.mark.parametrize("seed", [0, 1])
def test_config3_slice_matches_oracle(seed, oracle_mod):
    import os
    mol = W.water_cluster()
    sh = B.even_tempered(mol)
    eng = api.Engine(sh)
    eng.schwarz(1e-10)
    ob = oracle_mod.OracleBasis(sh)
    assert eng.nbf == 1824
    D = W.cluster_density(eng.nbf)
    ns = len(sh)
    rng = np.random.default_rng(W.SEED0 + 3400 + seed)
    a, b = np.tril_indices(ns)
    sel = rng.random(len(a)) < 0.03
    mask = np.zeros((ns, ns), bool)
    mask[a[sel], b[sel]] = True
    eng.set_pair_subset(mask)
    J, K, _ = eng.fock_jk(D)
    eng.set_pair_subset(None)
    Jr, Kr, cnt = ob.jk_direct_subset(D, mask, nthreads=os.cpu_count() or 1)
    assert cnt >= 10_000_000, cnt
    assert np.abs(Jr).max() > 1e-3
    errJ, errK = np.abs(J - Jr).max(), np.abs(K - Kr).max()
    assert errJ <= FOCK_TOL and errK <= FOCK_TOL, (cnt, errJ, errK)
