"""Failure handling through the C ABI: bad inputs come back as status codes, never as a crash.

All faults are injected on the host (bad matrices, bad arguments, a device-memory cap); no GPU fault,
trap or hang is provoked.  The one device-side wait the library has (the team kernels' mbarrier waits for
their bulk copies) is bounded; its give-up path is run on a barrier that nothing completes, with a short
limit, and must come back as a status while the context stays usable.
"""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = api.Engine(B.even_tempered(W.water()))
    e.schwarz(1e-10)
    return e


def _density(n, seed=3):
    Q, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(n, 5)))
    return 2 * Q @ Q.T


def test_nan_density_rejected(eng):
    D = _density(eng.nbf)
    D[3, 4] = D[4, 3] = np.nan
    with pytest.raises(api.QcgError) as e:
        eng.fock_jk(D)
    assert e.value.code == api.QCG_ERR_NONFINITE


def test_inf_density_rejected_on_device_path(eng):
    import torch
    D = torch.tensor(_density(eng.nbf), device="cuda")
    D[0, 0] = float("inf")
    J, K = torch.empty_like(D), torch.empty_like(D)
    with pytest.raises(api.QcgError) as e:
        eng.fock_jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), validate=True)
    assert e.value.code == api.QCG_ERR_NONFINITE


def test_asymmetric_density_rejected(eng):
    D = _density(eng.nbf)
    D[1, 2] += 1e-3
    with pytest.raises(api.QcgError) as e:
        eng.fock_jk(D)
    assert e.value.code == api.QCG_ERR_ASYMMETRIC


def test_wrong_dimension_rejected(eng):
    with pytest.raises(api.QcgError) as e:
        eng.fock_jk(np.eye(eng.nbf + 1))
    assert e.value.code == api.QCG_ERR_ARG


def test_non_canonical_class_rejected(eng):
    with pytest.raises(api.QcgError) as e:
        eng.eri_batch((0, 1, 0, 0), np.zeros((1, 4), dtype=np.int32))
    assert e.value.code == api.QCG_ERR_ARG


def test_shell_class_mismatch_rejected(eng):
    with pytest.raises(api.QcgError) as e:
        eng.eri_batch((1, 0, 0, 0), np.zeros((1, 4), dtype=np.int32))   # shell 0 is an s shell
    assert e.value.code == api.QCG_ERR_ARG


def test_memory_cap_gives_alloc_error():
    e = api.Engine(B.even_tempered(W.water()))
    e.set_memory_limit(1)   # below anything the screening needs
    with pytest.raises(api.QcgError) as ex:
        e.schwarz(1e-10)
    assert ex.value.code == api.QCG_ERR_ALLOC
    e.set_memory_limit(0)   # lifting the cap makes the handle usable again
    e.schwarz(1e-10)
    J, K, _ = e.fock_jk(_density(e.nbf))
    assert np.all(np.isfinite(J))


def test_bad_basis_rejected():
    sh = [B.Shell(3, (0.0, 0.0, 0.0), [1.0], [1.0])]
    with pytest.raises(api.QcgError) as e:
        api.Engine(sh)
    assert e.value.code == api.QCG_ERR_ARG
    sh = [B.Shell(0, (0.0, 0.0, 0.0), [-1.0], [1.0])]
    with pytest.raises(api.QcgError):
        api.Engine(sh)


def test_odd_electron_count_rejected():
    mol = B.Molecule([8, 1], np.array([[0, 0, 0], [0, 0, 1.8]], float))
    with pytest.raises(api.QcgError) as e:
        api.Engine(B.even_tempered(mol)).rhf(mol)
    assert e.value.code == api.QCG_ERR_ARG


def test_bounded_wait_completes_when_the_arrival_comes():
    gave_up, _ = api.selftest_bounded_wait(polls=1000, arrive=True)
    assert not gave_up


def test_bounded_wait_gives_up_and_the_context_stays_usable(eng):
    gave_up, ms = api.selftest_bounded_wait(polls=1000, arrive=False)
    assert gave_up
    assert ms < 1000.0   # 1000 polls, each suspending for at most a few microseconds
    # the GPU still answers: a J/K build right after matches one made before
    D = _density(eng.nbf)
    J1, K1, _ = eng.fock_jk(D)
    gave_up, _ = api.selftest_bounded_wait(polls=1000, arrive=False)
    assert gave_up
    J2, K2, _ = eng.fock_jk(D)
    assert np.abs(J1 - J2).max() < 1e-12 and np.abs(K1 - K2).max() < 1e-12
