"""Handles reuse the device slabs, pinned staging buffers, streams and events that destroyed handles left
in the process-wide cache.  Reused slabs still hold the previous handle's data, so every result must be
the same as from fresh allocations; qcg_release_cache empties the cache and later handles allocate again."""
import numpy as np
import pytest
import torch

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu


def _jk(shells, D):
    eng = api.Engine(shells)
    J, K, _ = eng.fock_jk(D)
    return J, K


def test_results_do_not_depend_on_reused_resources(oracle_mod):
    mol = W.water()
    sh = B.even_tempered(mol)
    D = oracle_mod.OracleBasis(sh).rhf(mol)["D"]
    api.release_cache()
    J0, K0 = _jk(sh, D)                      # fresh allocations
    # a larger basis fills the cache with slabs holding other data
    dimer = W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)
    shd = B.even_tempered(dimer)
    Dd = W.cluster_density(B.nbf(shd), nocc=10)
    _jk(shd, Dd)
    for _ in range(3):
        J, K = _jk(sh, D)                    # reused slabs, streams and events
        assert np.abs(J - J0).max() <= 1e-12 and np.abs(K - K0).max() <= 1e-12
    e_plain = api.Engine(sh).rhf(mol)["energy"]
    for _ in range(3):
        assert abs(api.Engine(sh).rhf(mol)["energy"] - e_plain) <= 1e-10


def test_release_cache_then_new_handles_on_a_user_stream():
    mol = W.water()
    sh = B.even_tempered(mol)
    e_ref = api.Engine(sh).rhf(mol)["energy"]
    api.release_cache()
    api.release_cache()                      # an empty cache is fine
    s = torch.cuda.Stream()
    eng = api.Engine(sh)
    eng.set_stream(s.cuda_stream)
    assert abs(eng.rhf(mol)["energy"] - e_ref) <= 1e-10
    del eng
    assert abs(api.Engine(sh).rhf(mol)["energy"] - e_ref) <= 1e-10


def test_many_short_lived_handles():
    """500 handles created and destroyed in a row take their resources from the cache: the device memory
    the process holds does not grow with the number of handles."""
    mol = W.water()
    sh = B.even_tempered(mol)
    D = W.cluster_density(B.nbf(sh), nocc=5)
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(500):
        eng = api.Engine(sh)
        eng.schwarz(1e-10)
        del eng
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < (64 << 20), (free0, free1)
    J, K = _jk(sh, D)
    assert np.isfinite(J).all() and np.isfinite(K).all()
