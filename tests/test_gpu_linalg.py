"""The SCF step's dense linear algebra on the GPU (cuSOLVER eigensolver, cuBLAS products), which qcg_rhf
uses for large bases: forced onto small systems it must reach the host path's energy and iteration count,
and the CPU oracle's energy."""
import os

import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["water", "dimer"])
def test_gpu_linear_algebra_matches_host(which, monkeypatch, oracle_mod):
    mol = W.water() if which == "water" else W.water_cluster(nx=2, ny=1, nz=1, seed=W.SEED0 + 3300)
    sh = B.even_tempered(mol)
    monkeypatch.setenv("QCG_GPU_LINALG_MIN", "1000000")
    host = api.Engine(sh).rhf(mol)
    monkeypatch.setenv("QCG_GPU_LINALG_MIN", "0")
    gpu = api.Engine(sh).rhf(mol)
    assert host["converged"] and gpu["converged"]
    assert abs(host["energy"] - gpu["energy"]) <= 1e-9
    assert abs(host["iterations"] - gpu["iterations"]) <= 1
    orc = oracle_mod.OracleBasis(sh).rhf(mol)
    assert orc["converged"] and abs(gpu["energy"] - orc["energy"]) <= 1e-8
