"""The team form of the FP64 ERI batches (eri_team.cuh) against the CPU oracle.

Every class is forced into the team form (qcg_set_eri_team_classes) and checked at the ERI bar, 1e-12
absolute, on 10^4 quartets per class drawn like the ERI benchmark (contraction 1-3 per shell, exponents
log-uniform in [0.05, 50], centres in a 12-bohr box).  Batch sizes that leave a group of 32 partly empty,
and small batches whose groups mix contraction patterns, are checked as well, and the team form is compared
with the one-thread-per-quartet form on the same batch.
"""
import numpy as np
import pytest

from qchem_b200 import api, workloads as W

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-12
ALL_CLASSES = (1 << 21) - 1
NPOOL = 512
NQ = 10_000


@pytest.fixture(scope="module")
def bench_pool():
    return W.shell_pool(NPOOL, seed=W.SEED0 + 4000)


@pytest.fixture(scope="module")
def team_engines(bench_pool, oracle_mod):
    eng = api.Engine(bench_pool)
    eng.set_eri_team_classes(ALL_CLASSES)
    return eng, oracle_mod.OracleBasis(bench_pool)


@pytest.mark.parametrize("k", range(21))
def test_team_form_matches_oracle_on_1e4_quartets(k, team_engines):
    eng, ob = team_engines
    cls = W.quartet_classes()[k]
    q = W.eri_class_batch(cls, NQ, NPOOL, seed=W.SEED0 + 4000 + k)
    got = eng.eri_batch(cls, q)
    ref = ob.eri_batch(q)
    assert np.all(np.isfinite(got))
    err = np.abs(got - ref).max()
    assert err <= ERI_TOL, f"class {cls}: max abs error {err:.3e} (max |eri| {np.abs(ref).max():.3e})"


@pytest.mark.parametrize("nq", [1, 31, 33, 95])
@pytest.mark.parametrize("cls", [(2, 2, 2, 2), (2, 1, 2, 1), (1, 1, 0, 0)])
def test_team_form_ragged_and_mixed_groups(nq, cls, team_engines):
    """Partial last groups, and groups whose lanes have different primitive counts (a small batch spreads
    over many contraction patterns, so its groups mix them)."""
    eng, ob = team_engines
    q = W.eri_class_batch(cls, nq, NPOOL, seed=W.SEED0 + 4100 + nq)
    got = eng.eri_batch(cls, q)
    ref = ob.eri_batch(q)
    assert np.abs(got - ref).max() <= ERI_TOL


def test_team_form_equals_thread_per_quartet_form(bench_pool):
    eng = api.Engine(bench_pool)
    cls = (2, 2, 2, 1)
    q = W.eri_class_batch(cls, 2000, NPOOL, seed=W.SEED0 + 4200)
    eng.set_eri_team_classes(0)
    a = eng.eri_batch(cls, q)
    eng.set_eri_team_classes(ALL_CLASSES)
    b = eng.eri_batch(cls, q)
    eng.set_eri_team_classes(-1)
    assert np.abs(a - b).max() <= ERI_TOL


def test_team_mask_rejects_bad_values(bench_pool):
    eng = api.Engine(bench_pool[:3])
    for bad in (-2, 1 << 21):
        with pytest.raises(api.QcgError) as e:
            eng.set_eri_team_classes(bad)
        assert e.value.code == api.QCG_ERR_ARG
