"""Host-side logic that needs no GPU: the C ABI library, basis construction, workloads, the SCF
eigensolver, and the multi-process plumbing (gloo, world size 2)."""
import os
import re
import socket

import numpy as np
import pytest

from qchem_b200 import api, basis as B, parallel, workloads as W
from tests.conftest import REPO, molecule_from


def _header_symbols():
    text = open(os.path.join(REPO, "include", "qchem_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(qcg_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    import ctypes
    L = ctypes.CDLL(api.library_path())
    syms = _header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), s


def test_no_silent_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(api.QcgError) as e:
        api.Engine(B.even_tempered(W.water()))
    assert e.value.code == api.QCG_ERR_CUDA


def test_syev_matches_numpy():
    rng = np.random.default_rng(4)
    for n in (1, 2, 5, 57, 120):
        A = rng.normal(size=(n, n))
        A = A + A.T
        w, V = api.syev(A)
        np.testing.assert_allclose(w, np.linalg.eigvalsh(A), atol=1e-11 * max(1, np.abs(w).max()))
        np.testing.assert_allclose(V @ np.diag(w) @ V.T, A, atol=1e-11 * n)
        np.testing.assert_allclose(V.T @ V, np.eye(n), atol=1e-12 * n)


def test_syev_degenerate_and_diagonal():
    w, V = api.syev(np.diag([3.0, 1.0, 2.0, 1.0]))
    np.testing.assert_allclose(w, [1, 1, 2, 3])
    w, _ = api.syev(np.ones((4, 4)))
    np.testing.assert_allclose(w, [0, 0, 0, 4], atol=1e-14)


def _check_lowest(A, k):
    w, V = api.syev_lowest(A, k)
    wr, Vr = np.linalg.eigh(A)
    scale = max(1.0, np.abs(wr).max())
    np.testing.assert_allclose(w, wr[:k], atol=1e-11 * scale)
    assert V.shape == (A.shape[0], k)
    np.testing.assert_allclose(V.T @ V, np.eye(k), atol=1e-11)
    np.testing.assert_allclose(A @ V, V * w[:k], atol=1e-10 * scale)
    # the occupied-subspace projector, which is what the SCF density uses, where the spectrum has a gap
    if k < A.shape[0] and wr[k] - wr[k - 1] > 1e-6 * scale:
        np.testing.assert_allclose(V @ V.T, Vr[:, :k] @ Vr[:, :k].T, atol=1e-10)


def test_syev_lowest_matches_numpy():
    rng = np.random.default_rng(7)
    for n, k in ((3, 1), (5, 2), (57, 5), (120, 17), (225, 60), (57, 56), (57, 57)):
        A = rng.normal(size=(n, n))
        _check_lowest(A + A.T, k)


def test_syev_lowest_degenerate_spectra():
    rng = np.random.default_rng(8)
    n = 40
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    # exactly repeated lowest eigenvalues (a 3-fold and a 2-fold level), then a gap
    lam = np.concatenate([[-5.0] * 3, [-2.0] * 2, np.linspace(1, 30, n - 5)])
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    for k in (3, 5, 7):
        _check_lowest(A, k)
    # diagonal and block-diagonal inputs (the reduction is the identity), and the zero matrix
    _check_lowest(np.diag([3.0, 1.0, 2.0, 1.0, 0.5]), 2)
    _check_lowest(np.kron(np.eye(4), np.array([[2.0, 1.0], [1.0, 2.0]])), 4)
    w, V = api.syev_lowest(np.zeros((6, 6)), 2)
    assert w.shape == (2,)
    np.testing.assert_allclose(w, 0.0)
    np.testing.assert_allclose(V.T @ V, np.eye(2), atol=1e-12)


def test_orthogonaliser_is_upper_triangular_and_orthonormalising():
    rng = np.random.default_rng(9)
    for n in (1, 5, 57, 120):
        M = rng.normal(size=(n, n))
        S = M @ M.T + n * np.eye(n)
        X = api.orthogonaliser(S)
        assert X is not None
        np.testing.assert_allclose(X.T @ S @ X, np.eye(n), atol=1e-12 * n)
        np.testing.assert_array_equal(np.tril(X, -1), 0.0)
    # the overlap of the config-1 water basis (diffuse, condition number ~1e4 and above)
    sh = B.even_tempered(W.water())
    from oracle.oracle import OracleBasis
    S = OracleBasis(sh).one_electron(W.water())[0]
    X = api.orthogonaliser(S)
    np.testing.assert_allclose(X.T @ S @ X, np.eye(len(S)), atol=1e-10)
    # not positive definite: refused, so that the SCF falls back to the eigendecomposition
    assert api.orthogonaliser(np.diag([1.0, -1.0, 2.0])) is None


def test_even_tempered_layout():
    mol = W.water()
    sh = B.even_tempered(mol)
    assert len(sh) == 29 and B.nbf(sh) == 57
    assert [s.L for s in sh[:15]] == [0] * 8 + [1] * 5 + [2] * 2
    assert sh[7].exps[0] == pytest.approx(0.1 * 2.5 ** 7)
    assert B.components(2) == [(2, 0, 0), (1, 1, 0), (0, 2, 0), (1, 0, 1), (0, 1, 1), (0, 0, 2)]
    assert B.components(1) == [(1, 0, 0), (0, 1, 0), (0, 0, 1)]


def test_cluster_size_and_determinism():
    m1, m2 = W.water_cluster(), W.water_cluster()
    np.testing.assert_array_equal(m1.R, m2.R)
    sh = B.even_tempered(m1)
    assert len(sh) == 928 and B.nbf(sh) == 1824
    # molecules keep their internal geometry under the random rotations
    for k in range(0, 96, 3):
        assert np.linalg.norm(m1.R[k + 1] - m1.R[k]) == pytest.approx(np.hypot(1.43, 1.11))
    D = W.cluster_density(60, nocc=10)
    np.testing.assert_allclose(D @ D, 2 * D, atol=1e-12)   # 2 x projector
    assert np.trace(D) == pytest.approx(20)


def test_dzvp_reader(dzvp_text, anchors):
    mol = molecule_from(anchors["water"])
    sh = B.read_gaussian94(dzvp_text, mol)
    assert [s.L for s in sh] == [0, 0, 0, 1, 1, 2, 0, 0, 0, 0]
    assert B.nbf(sh) == 19
    assert sh[0].nprim == 6 and sh[5].nprim == 1 and sh[5].coefs == [1.0]
    n2 = molecule_from(anchors["n2"])
    assert B.nbf(B.read_gaussian94(dzvp_text, n2)) == 30


def test_reader_merges_duplicate_radials_like_the_reference():
    text = "\n!\nBASIS=\"t\"\n H   0\n S   1  1.00\n  0.5  1.0\n S   1  1.00\n  0.5  1.0\n ****\n"
    mol = B.Molecule([1], np.zeros((1, 3)))
    sh = B.read_gaussian94(text, mol)
    # equal radials on one centre are merged and the merge appends the L that is already present
    # (src/BasisSet/Molecule/PG_Cart/Imp/IrrepBasisSet.C:75-94), so the s function appears twice
    assert [s.L for s in sh] == [0, 0]


def test_quartet_classes_and_batches():
    cls = W.quartet_classes()
    assert len(cls) == 21 and cls[0] == (0, 0, 0, 0) and cls[-1] == (2, 2, 2, 2)
    for la, lb, lc, ld in cls:
        assert la >= lb and lc >= ld
    q = W.eri_class_batch((2, 1, 1, 0), 100, 64, seed=1)
    pool = W.shell_pool(64, seed=2)
    assert [pool[i].L for i in q[0]] == [2, 1, 1, 0]
    np.testing.assert_array_equal(q, W.eri_class_batch((2, 1, 1, 0), 100, 64, seed=1))


def test_random_molecules_are_closed_shell():
    mols = W.random_molecules(40)
    for m in mols:
        assert m.nelec % 2 == 0 and 2 <= len(m.Z) <= 24


def test_shard_range_partitions():
    for n in (0, 1, 7, 100):
        for world in (1, 2, 3, 8):
            ranges = [parallel.shard_range(n, r, world) for r in range(world)]
            covered = [i for lo, hi in ranges for i in range(lo, hi)]
            assert covered == list(range(n))


def test_shard_weighted_balances():
    costs = [10, 1, 1, 1, 9, 2, 8, 3]
    parts = parallel.shard_weighted(costs, 2)
    assert sorted(i for p in parts for i in p) == list(range(8))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, D, out_q):
    """One rank: its share of the bra shell pairs of a direct J/K build (CPU oracle as the stand-in for
    the rank's GPU), then the sum over ranks and the max of the per-rank times over gloo."""
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle.oracle import OracleBasis
    ob = OracleBasis(B.even_tempered(W.water()))
    J, K = ob.jk_direct_shard(D, rank, world)
    Jt, Kt = torch.from_numpy(J), torch.from_numpy(K)
    parallel.reduce_jk(Jt, Kt)
    t = parallel.max_over_ranks(float(rank + 1))
    if rank == 0:
        out_q.put((Jt.numpy().copy(), Kt.numpy().copy(), t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_jk_reduction_matches_single_build(oracle_mod):
    import multiprocessing as mp
    from oracle.oracle import OracleBasis
    ob = OracleBasis(B.even_tempered(W.water()))
    n = ob.nbf
    Q, _ = np.linalg.qr(np.random.default_rng(8).normal(size=(n, 5)))
    D = 2 * Q @ Q.T
    Jr, Kr, _ = ob.jk_direct(D)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, D, q)) for r in range(2)]
    for p in procs:
        p.start()
    J, K, t = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert t == 2.0
    assert np.abs(J - Jr).max() < 1e-12 and np.abs(K - Kr).max() < 1e-12


def test_cpp_adapter_builds_and_fails_loudly_without_a_device(tmp_path):
    """include/qchem_b200.hpp compiles against the C ABI; without a GPU its constructor throws QCG_ERR_CUDA."""
    import shutil
    import subprocess
    import torch
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    src = tmp_path / "t.cpp"
    src.write_text('#include "qchem_b200.hpp"\nint main(){std::vector<qcg::ShellSpec> s{{0,{0,0,0},{1.0},{1.0}}};\n'
                   'int rc;\n'
                   'try { qcg::FockEngine e(s); rc = e.AODimension() == 1 ? 0 : 3; }\n'
                   'catch (const qcg::Error& err) { rc = err.code == QCG_ERR_CUDA ? 10 : 11; }\n'
                   'qcg::release_cache(); return rc; }\n')
    libdir = os.path.dirname(api.library_path())
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "include"), str(src), "-L", libdir, "-lqchem_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    rc = subprocess.run([str(exe)]).returncode
    assert rc == (0 if torch.cuda.is_available() else 10)


def test_hrr_class_selection(monkeypatch):
    """Where an FP64 ERI batch runs thread-per-quartet (the team form switched off for the class), the
    horizontal-recurrence form serves (dp|dp), (dd|pp), (dd|dp) and (dd|dd) by default; QCG_ERI_HRR=1 / =0
    switch every class."""
    from qchem_b200 import build as qb
    monkeypatch.delenv("QCG_ERI_HRR", raising=False)
    picked = [W.quartet_classes()[k] for k in range(21) if qb._eri_hrr(k)]
    assert picked == [(2, 1, 2, 1), (2, 2, 1, 1), (2, 2, 2, 1), (2, 2, 2, 2)]
    monkeypatch.setenv("QCG_ERI_HRR", "1")
    assert all(qb._eri_hrr(k) for k in range(21))
    monkeypatch.setenv("QCG_ERI_HRR", "0")
    assert not any(qb._eri_hrr(k) for k in range(21))


def test_bench_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the CPU oracle's rate on the ERI microbenchmark's class mix) runs without
    a GPU and prints one JSON line with the keys the benchmark contract needs, the same metric and unit as the
    GPU arm, and a cpu_baseline and e2e block describing itself."""
    import json
    import subprocess
    import sys
    from tests.conftest import REPO
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--ref-sample", "40"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["unit"] == "quartets/s" and line["metric"].startswith("ERI quartets/s")
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0


def test_cpp_salc_block_compiles_and_links(tmp_path):
    """qcg::SalcBlock (the symmetry-adapted faces) compiles against include/qchem_b200.hpp and links against
    qcg_salc_fold / qcg_salc_slice; without a GPU the AO engine's constructor throws QCG_ERR_CUDA first."""
    import shutil
    import subprocess
    import torch
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    src = tmp_path / "s.cpp"
    src.write_text('#include "qchem_b200.hpp"\nint main(){std::vector<qcg::ShellSpec> s{{0,{0,0,0},{1.0},{1.0}}};\n'
                   'int rc;\n'
                   'try { qcg::FockEngine e(s); qcg::SalcBlock b(e, std::vector<double>{1.0}, 1);\n'
                   '  double D[1] = {1.0}, Dao[1] = {0.0}, F[1] = {0.0}, J[1] = {0.0};\n'
                   '  b.AddAODensity(Dao, D); b.SliceAOFock(F, Dao); b.AccumulateDirect(J, D, &b);\n'
                   '  rc = (Dao[0] == 1.0 && F[0] == 1.0 && J[0] > 0.0) ? 0 : 3; }\n'
                   'catch (const qcg::Error& err) { rc = err.code == QCG_ERR_CUDA ? 10 : 11; }\n'
                   'qcg::release_cache(); return rc; }\n')
    libdir = os.path.dirname(api.library_path())
    exe = tmp_path / "s"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "include"), str(src), "-L", libdir, "-lqchem_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    rc = subprocess.run([str(exe)]).returncode
    assert rc == (0 if torch.cuda.is_available() else 10)


def test_default_jk_forms_do_not_overlap():
    """The build's default J/K class sets: the team form for the high-L classes, the warp-shared form for
    twelve others; no class is in both (the team form would take precedence), and (ss|ss), (pp|pp) and
    (dd|ss) stay thread-per-quartet."""
    from qchem_b200 import build as qb
    team, warp = set(qb.JK_TEAM_CLASSES), set(qb.JK_WARP_CLASSES)
    assert not team & warp
    assert len(team) == 6 and len(warp) == 12
    names = ["".join("spd"[l] for l in c) for c in W.quartet_classes()]
    assert {names[k] for k in set(range(21)) - team - warp} == {"ssss", "pppp", "ddss"}
    assert qb._jk_team_mask() & qb._jk_warp_mask() == 0
