"""The FP32 form of the ERI engine and of the J/K build, and the SCF schedule that uses it.

FP32 integrals are reported against the FP64 oracle and gated loosely (relative to the largest integral
of the batch); what must hold exactly is the end result: an SCF that starts in FP32 reaches the plain
all-FP64 energy within 1e-8 Eh, because the build that confirms convergence is all-FP64.
"""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

FP32_ERI_REL = 2e-5     # max |eri32 - eri64| / max |eri64| over a 10^4-quartet batch of one class
FP32_JK_ABS = 2e-5      # max |J32 - J64|, |K32 - K64| for the water density
E_TOL = 1e-8


@pytest.fixture(scope="module")
def pool_engines(oracle_mod):
    shells = W.shell_pool(512, seed=W.SEED0 + 4000)
    return api.Engine(shells), oracle_mod.OracleBasis(shells)


@pytest.mark.parametrize("k", range(21))
def test_fp32_eri_batch_class(k, pool_engines):
    """10^4 quartets per class drawn like the ERI benchmark (contraction 1-3, exponents log-uniform in
    [0.05, 50], centres in a 12-bohr box), FP32 against the oracle's FP64."""
    eng, ob = pool_engines
    cls = W.quartet_classes()[k]
    q = W.eri_class_batch(cls, 10_000, 512, seed=W.SEED0 + 4100 + k)
    got = eng.eri_batch(cls, q, fp32=True)
    assert got.dtype == np.float32 and np.all(np.isfinite(got))
    ref = ob.eri_batch(q)
    rel = np.abs(got.astype(np.float64) - ref).max() / np.abs(ref).max()
    print(f"class {cls}: FP32 max error / max |eri| = {rel:.2e}")
    assert rel <= FP32_ERI_REL


@pytest.fixture(scope="module")
def water_case(oracle_mod):
    mol = W.water()
    sh = B.even_tempered(mol)
    D = oracle_mod.OracleBasis(sh).rhf(mol)["D"]
    return sh, D


def test_fp32_jk_close_to_fp64(water_case):
    sh, D = water_case
    eng = api.Engine(sh)
    J, K, _ = eng.fock_jk(D)
    J32, K32, _ = eng.fock_jk(D, fp32=True)
    dj, dk = np.abs(J32 - J).max(), np.abs(K32 - K).max()
    print(f"FP32 J/K: max |dJ| {dj:.2e}, max |dK| {dk:.2e}")
    assert 0 < max(dj, dk) <= FP32_JK_ABS
    np.testing.assert_allclose(J32, J32.T, atol=1e-14)


def test_mixed_bound_interpolates(water_case):
    """Quartets below the Schwarz bound in FP32: the error shrinks as the bound does, and a zero bound is
    the FP64 build."""
    sh, D = water_case
    eng = api.Engine(sh)
    J, K, _ = eng.fock_jk(D)
    J32, K32, _ = eng.fock_jk(D, fp32=True)
    full = max(np.abs(J32 - J).max(), np.abs(K32 - K).max())
    errs = []
    for bound in (1e-2, 1e-5):
        eng.set_fp32_bound(bound)
        Jm, Km, st = eng.fock_jk(D)
        errs.append(max(np.abs(Jm - J).max(), np.abs(Km - K).max()))
    eng.set_fp32_bound(0.0)
    J0, K0, _ = eng.fock_jk(D)
    assert max(np.abs(J0 - J).max(), np.abs(K0 - K).max()) <= 1e-12
    assert errs[0] <= full * 1.5 and errs[1] <= errs[0]
    assert errs[1] <= 1e-8


def test_fp32_bound_rejects_negative(water_case):
    eng = api.Engine(water_case[0])
    with pytest.raises(api.QcgError) as e:
        eng.set_fp32_bound(-1.0)
    assert e.value.code == api.QCG_ERR_ARG


@pytest.mark.parametrize("incremental", [False, True])
def test_fp32_early_scf_reaches_the_fp64_energy(incremental):
    mol = W.water()
    sh = B.even_tempered(mol)
    plain = api.Engine(sh).rhf(mol)
    chosen = api.Engine(sh).rhf(mol, fp32_early=True, incremental=incremental)
    assert plain["converged"] and chosen["converged"]
    assert chosen["fp32_builds"] > 0
    assert abs(plain["energy"] - chosen["energy"]) <= E_TOL, (plain["energy"], chosen["energy"])


def test_fp32_early_water_dimer():
    mol = W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)
    sh = B.even_tempered(mol)
    plain = api.Engine(sh).rhf(mol)
    chosen = api.Engine(sh).rhf(mol, fp32_early=True, incremental=True, fp32_below=1e-9)
    assert plain["converged"] and chosen["converged"] and chosen["fp32_builds"] > 0
    assert abs(plain["energy"] - chosen["energy"]) <= E_TOL


def test_guess_density_from_a_converged_run():
    mol = W.water()
    sh = B.even_tempered(mol)
    eng = api.Engine(sh)
    ref = eng.rhf(mol, want_density=True)
    again = api.Engine(sh).rhf(mol, guess=ref["D"])
    assert again["converged"] and again["iterations"] <= 3
    assert abs(again["energy"] - ref["energy"]) <= E_TOL
