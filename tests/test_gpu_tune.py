"""The J/K launch-shape autotuner: it picks a valid shape for every class with quartets, and builds with
the tuned shapes give the same J, K and SCF energy as builds with the default shapes."""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results():
    import torch
    mol = W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)
    sh = B.even_tempered(mol)
    eng = api.Engine(sh)
    eng.schwarz(1e-10)
    Dh = W.cluster_density(eng.nbf, nocc=10)
    J0, K0, _ = eng.fock_jk(Dh)
    D = torch.tensor(Dh, device="cuda")
    choice = eng.autotune_jk(D.data_ptr(), reps=1)
    assert len(choice) == 21
    for run, cap in choice:
        assert (run, cap) == (0, 0) or (run in (1, 2, 4, 8, 16) and cap in (8, 16))
    assert any(run > 0 for run, _ in choice)
    J1, K1, _ = eng.fock_jk(Dh)
    assert np.abs(J1 - J0).max() <= 1e-10 and np.abs(K1 - K0).max() <= 1e-10


def test_scf_with_autotune_same_energy():
    mol = W.water()
    sh = B.even_tempered(mol)
    a = api.Engine(sh).rhf(mol)
    b = api.Engine(sh).rhf(mol, autotune=True)
    assert b["converged"] and abs(a["energy"] - b["energy"]) <= 1e-8
