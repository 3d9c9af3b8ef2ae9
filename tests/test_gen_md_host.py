"""The generated McMurchie-Davidson code without a GPU: gen_md.py's per-class headers (the code the CUDA
kernels run) are compiled for the host with tests/host_md/host_md.cpp and checked against the CPU oracle
at the GPU parity bar, 1e-12 absolute, for every (s,p,d) class on contracted random shells.  This pins the
code generator, the Boys function, the R recursion and the Hermite transforms on the CPU; the GPU tests
pin the kernels that run them.  The generator's horizontal-recurrence form (gen_md.main_hrr, not yet used
by the kernels) is held to the same bar."""
import concurrent.futures as cf
import ctypes
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from qchem_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "qchem_b200", "csrc")
ERI_ABS = 1e-12
NQ = 24   # quartets per class


@pytest.fixture(scope="session")
def host_classes(tmp_path_factory):
    """{class index: ctypes library} for the 21 classes, built in a temporary directory."""
    if shutil.which("g++") is None:
        pytest.skip("g++ is not available")
    tmp = str(tmp_path_factory.mktemp("host_md"))
    sys.path.insert(0, CSRC)
    try:
        import gen_md
    finally:
        sys.path.pop(0)
    gen_md.main(os.path.join(tmp, "gen"))
    gen_md.main_hrr(os.path.join(tmp, "gen_hrr"))
    for name in ("md_core.cuh", "boys_table.h"):
        shutil.copy(os.path.join(CSRC, name), tmp)
    src = os.path.join(HERE, "host_md", "host_md.cpp")

    def compile_class(k):
        out = os.path.join(tmp, f"host_md_{k}.so")
        r = subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", f"-DQCG_CLASS={k}", "-DHM_HRR", "-I", tmp,
                            src, "-o", out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        lib = ctypes.CDLL(out)
        lib.host_md_eri.restype = ctypes.c_int
        lib.host_md_eri_f32.restype = ctypes.c_int
        lib.host_md_eri_hrr.restype = ctypes.c_int
        lib.host_md_eri_hrr_inplace.restype = ctypes.c_int
        assert lib.host_md_class() == k
        return k, lib

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        return dict(ex.map(compile_class, range(len(W.quartet_classes()))))


def _pack(pool, q):
    """Per-shell rows of the quartets in the harness's layout (8 primitive slots per shell)."""
    n = len(q)
    L = np.zeros(4 * n, dtype=np.int32)
    npr = np.zeros(4 * n, dtype=np.int32)
    ex = np.zeros((4 * n, 8))
    co = np.zeros((4 * n, 8))
    cen = np.zeros((n, 12))
    for i, quartet in enumerate(q):
        for s, idx in enumerate(quartet):
            sh = pool[int(idx)]
            r = 4 * i + s
            L[r], npr[r] = sh.L, len(sh.exps)
            ex[r, :len(sh.exps)] = sh.exps
            co[r, :len(sh.coefs)] = sh.coefs
            cen[i, 3 * s:3 * s + 3] = sh.centre
    return L, npr, ex, co, cen


@pytest.mark.parametrize("k", range(21))
def test_generated_class_matches_oracle(k, host_classes, oracle_mod):
    cls = W.quartet_classes()[k]
    # shells in a 3-bohr box: overlapping distributions give integrals of order 1, so the absolute bar is
    # also a relative one
    pool = W.shell_pool(16, seed=W.SEED0 + 2100, box=3.0)
    q = W.eri_class_batch(cls, NQ, 16, seed=W.SEED0 + 2100 + k)
    L, npr, ex, co, cen = _pack(pool, q)
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.zeros(NQ * blk)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rc = host_classes[k].host_md_eri(ctypes.c_longlong(NQ), p(L, ctypes.c_int), p(npr, ctypes.c_int),
                                     p(ex, ctypes.c_double), p(co, ctypes.c_double), p(cen, ctypes.c_double),
                                     p(out, ctypes.c_double))
    assert rc == 0
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    err = np.abs(out - ref).max()
    assert err <= ERI_ABS, (cls, err)
    assert err <= 1e-12 * np.abs(ref).max(), (cls, err, np.abs(ref).max())
    assert np.abs(ref).max() > 1e-2   # the batch is not trivially small


@pytest.mark.parametrize("k", range(21))
def test_generated_class_fp32_form(k, host_classes, oracle_mod):
    """The FP32 instantiation of the same code: error relative to the batch's largest integral within the
    bar the GPU FP32 tests use (2e-5)."""
    cls = W.quartet_classes()[k]
    pool = W.shell_pool(16, seed=W.SEED0 + 2100, box=3.0)
    q = W.eri_class_batch(cls, NQ, 16, seed=W.SEED0 + 2100 + k)
    L, npr, ex, co, cen = _pack(pool, q)
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.zeros(NQ * blk, dtype=np.float32)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rc = host_classes[k].host_md_eri_f32(ctypes.c_longlong(NQ), p(L, ctypes.c_int), p(npr, ctypes.c_int),
                                         p(ex, ctypes.c_double), p(co, ctypes.c_double), p(cen, ctypes.c_double),
                                         p(out, ctypes.c_float))
    assert rc == 0
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    rel = np.abs(out.astype(np.float64) - ref).max() / np.abs(ref).max()
    assert 0 < rel <= 2e-5, (cls, rel)


@pytest.mark.parametrize("k", range(21))
def test_generated_class_hrr_form(k, host_classes, oracle_mod):
    """[e0|f0] accumulated over the primitives, then the ket and bra horizontal recurrences: the same
    integrals as the direct form, to 1e-12 absolute and relative to the largest integral."""
    cls = W.quartet_classes()[k]
    pool = W.shell_pool(16, seed=W.SEED0 + 2100, box=3.0)
    q = W.eri_class_batch(cls, NQ, 16, seed=W.SEED0 + 2100 + k)
    L, npr, ex, co, cen = _pack(pool, q)
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.zeros(NQ * blk)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    # separate buffers, and in place in each quartet's output block (the planned kernel data flow)
    for fn in (host_classes[k].host_md_eri_hrr, host_classes[k].host_md_eri_hrr_inplace):
        out[:] = np.nan
        rc = fn(ctypes.c_longlong(NQ), p(L, ctypes.c_int), p(npr, ctypes.c_int), p(ex, ctypes.c_double),
                p(co, ctypes.c_double), p(cen, ctypes.c_double), p(out, ctypes.c_double))
        assert rc == 0
        err = np.abs(out - ref).max()
        assert err <= ERI_ABS and err <= 1e-12 * np.abs(ref).max(), (cls, fn.__name__, err, np.abs(ref).max())
