"""3-centre Coulomb integrals (ab|c) (qcg_eri3_batch) against the oracle's restatement of the reference's
Repulsion3C/RepulsionThreeC, 1e-12 absolute, in both orientations of the underlying 4-centre class."""
import itertools

import numpy as np
import pytest

from qchem_b200 import api, workloads as W

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-12
NPOOL = 64


@pytest.fixture(scope="module")
def engines(oracle_mod):
    pool = W.shell_pool(NPOOL, seed=W.SEED0 + 2100)
    return api.Engine(pool), oracle_mod.OracleBasis(pool)


CLASSES = [(la, lb, lc) for la in range(3) for lb in range(la + 1) for lc in range(3)]


@pytest.mark.parametrize("cls3", CLASSES)
def test_eri3_class(cls3, engines):
    eng, ob = engines
    rng = np.random.default_rng(sum(10 ** i * l for i, l in enumerate(cls3)))
    t = np.stack([L * NPOOL + rng.integers(0, NPOOL, size=100) for L in cls3], axis=1).astype(np.int32)
    got = eng.eri3_batch(cls3, t)
    ref = ob.eri3_batch(t)
    assert got.shape == ref.shape and np.all(np.isfinite(got))
    err = np.abs(got - ref).max()
    assert err <= ERI_TOL, f"{cls3}: {err:.2e} (max |eri| {np.abs(ref).max():.2e})"


def test_eri3_rejects_bad_classes(engines):
    eng, _ = engines
    t = np.array([[0, NPOOL, 0]], dtype=np.int32)     # s, p, s shells
    with pytest.raises(api.QcgError):
        eng.eri3_batch((0, 1, 0), t)                   # la < lb
    with pytest.raises(api.QcgError):
        eng.eri3_batch((1, 0, 0), t)                   # shells do not match the class
