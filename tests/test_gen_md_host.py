"""The generated McMurchie-Davidson code without a GPU: gen_md.py's per-class headers (the code the CUDA
kernels run) are compiled for the host with tests/host_md/host_md.cpp and checked against the CPU oracle
at the GPU parity bar, 1e-12 absolute, for every (s,p,d) class on contracted random shells.  This pins the
code generator, the Boys function, the R recursion and the Hermite transforms on the CPU; the GPU tests
pin the kernels that run them.  The generator's horizontal-recurrence form (gen_md.main_hrr, not yet used
by the kernels) is held to the same bar, and the library's J/K digestion sink (eri_kernels.cuh, compiled
with the CUDA stand-in in tests/host_md/shim) is checked against its digestion formulas, as one quartet and
chunk by chunk as the few-quartet J/K kernel runs it."""
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
    gen_md.main_team(os.path.join(tmp, "gen_team"))
    for name in ("md_core.cuh", "boys_table.h"):
        shutil.copy(os.path.join(CSRC, name), tmp)
    src = os.path.join(HERE, "host_md", "host_md.cpp")

    def compile_class(k):
        out = os.path.join(tmp, f"host_md_{k}.so")
        r = subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", f"-DQCG_CLASS={k}", "-DHM_HRR", "-DHM_TEAM", "-I",
                            tmp, src, "-o", out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        lib = ctypes.CDLL(out)
        lib.host_md_eri.restype = ctypes.c_int
        lib.host_md_eri_f32.restype = ctypes.c_int
        lib.host_md_eri_hrr.restype = ctypes.c_int
        lib.host_md_eri_hrr_inplace.restype = ctypes.c_int
        lib.host_md_eri_hrr_f32.restype = ctypes.c_int
        lib.host_md_eri_team.restype = ctypes.c_int
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


@pytest.mark.parametrize("box", [3.0, 12.0])
@pytest.mark.parametrize("k", range(21))
def test_generated_class_hrr_form(k, box, host_classes, oracle_mod):
    """[e0|f0] accumulated over the primitives, then the ket and bra horizontal recurrences: the same
    integrals as the direct form, to 1e-12 absolute and relative to the largest integral, on compact shells
    and on the benchmark's 12-bohr box (large A - B, C - D)."""
    cls = W.quartet_classes()[k]
    pool = W.shell_pool(16, seed=W.SEED0 + 2100, box=box)
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


@pytest.mark.parametrize("box", [3.0, 12.0])
@pytest.mark.parametrize("k", range(21))
def test_generated_class_team_form(k, box, host_classes, oracle_mod):
    """The team form's arithmetic (producer stage, ket step per component f into Y_f summed over the ket
    primitives, bra step once per bra primitive pair, then both recurrences in place in the output block):
    the integrals of the direct form, to 1e-12 absolute and relative to the largest integral."""
    cls = W.quartet_classes()[k]
    pool = W.shell_pool(16, seed=W.SEED0 + 2100, box=box)
    q = W.eri_class_batch(cls, NQ, 16, seed=W.SEED0 + 2100 + k)
    L, npr, ex, co, cen = _pack(pool, q)
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.full(NQ * blk, np.nan)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rc = host_classes[k].host_md_eri_team(ctypes.c_longlong(NQ), p(L, ctypes.c_int), p(npr, ctypes.c_int),
                                          p(ex, ctypes.c_double), p(co, ctypes.c_double), p(cen, ctypes.c_double),
                                          p(out, ctypes.c_double))
    assert rc == 0
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    err = np.abs(out - ref).max()
    assert err <= ERI_ABS and err <= 1e-12 * np.abs(ref).max(), (cls, err, np.abs(ref).max())


@pytest.fixture(scope="session")
def host_jk(tmp_path_factory):
    """{class index: ctypes library} of tests/host_md/host_jk.cpp (the J/K digestion sink on the host)."""
    if shutil.which("g++") is None:
        pytest.skip("g++ is not available")
    tmp = str(tmp_path_factory.mktemp("host_jk"))
    sys.path.insert(0, CSRC)
    try:
        import gen_md
    finally:
        sys.path.pop(0)
    gen_md.main(os.path.join(tmp, "gen"))
    gen_md.main_hrr(os.path.join(tmp, "gen_hrr"))
    for name in ("md_core.cuh", "boys_table.h", "eri_kernels.cuh", "qcg_internal.h"):
        shutil.copy(os.path.join(CSRC, name), tmp)
    src = os.path.join(HERE, "host_md", "host_jk.cpp")
    shim = os.path.join(HERE, "host_md", "shim")

    def compile_class(k):
        out = os.path.join(tmp, f"host_jk_{k}.so")
        r = subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", f"-DQCG_CLASS={k}", "-DHJ_HRR", "-I", shim,
                            "-I", tmp, src, "-o", out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        lib = ctypes.CDLL(out)
        lib.host_jk_quartet.restype = ctypes.c_int
        lib.host_jk_nchunk.restype = ctypes.c_int
        lib.host_jk_kernel.restype = ctypes.c_int
        lib.host_jk_kernel_batch.restype = ctypes.c_int
        lib.host_jk_kernel_band.restype = ctypes.c_int
        lib.host_eri_hrr_kernel.restype = ctypes.c_int
        lib.host_schwarz_kernel.restype = ctypes.c_int
        lib.host_eri_batch_kernel.restype = ctypes.c_int
        return k, lib

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        return dict(ex.map(compile_class, range(len(W.quartet_classes()))))


def _norm_coefs(sh):
    """The library's contraction preprocessing: (L,0,0) primitive norms folded in, unit radial self-overlap."""
    a = np.asarray(sh.exps, dtype=float)
    L = sh.L
    dfact = float(np.prod(np.arange(2 * L - 1, 0, -2))) if L > 0 else 1.0
    w = np.asarray(sh.coefs, dtype=float) * np.sqrt((4 * a) ** L / ((np.pi / (2 * a)) ** 1.5 * dfact))
    p = a[:, None] + a[None, :]
    ss = (w[:, None] * w[None, :] * (np.pi / p) ** 1.5 / (2 * p) ** L).sum()
    return w / np.sqrt(ss)


@pytest.mark.parametrize("k", range(21))
def test_jk_sink_digests_like_its_formulas(k, host_classes, host_jk):
    """For one shell quartet of each class: J' and K' from the library's digestion sink, both as one
    quartet (jk_kernel) and chunk by chunk with a row flush after every primitive quartet
    (jk_split_kernel), against the digestion formulas applied to the quartet's ERI block."""
    cls = W.quartet_classes()[k]
    pool = W.shell_pool(16, seed=W.SEED0 + 2200, box=3.0)
    q = W.eri_class_batch(cls, 40, 16, seed=W.SEED0 + 2200 + k)
    quartet = next(x for x in q if len(set(int(s) for s in x)) == 4)   # four distinct shells
    shells = [pool[int(s)] for s in quartet]
    nf = [(s.L + 1) * (s.L + 2) // 2 for s in shells]
    f0 = np.concatenate([[0], np.cumsum(nf)[:-1]]).astype(int)
    n = int(sum(nf))
    # the quartet's ERI block from the generated code (checked against the oracle above)
    L, npr, ex, co, cen = _pack(pool, np.asarray([quartet]))
    eri = np.zeros(int(np.prod(nf)))
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    assert host_classes[k].host_md_eri(ctypes.c_longlong(1), p(L, ctypes.c_int), p(npr, ctypes.c_int),
                                       p(ex, ctypes.c_double), p(co, ctypes.c_double), p(cen, ctypes.c_double),
                                       p(eri, ctypes.c_double)) == 0
    eri = eri.reshape(nf)
    rng = np.random.default_rng(k)
    D = rng.normal(size=(n, n))
    D = D + D.T
    s = 0.75   # a symmetry weight as the kernels pass it
    # the sink's formulas: w = s (mu nu|la si); J'[mu nu] += 2 w D[la si], J'[la si] += 2 w D[mu nu],
    # K'[mu la] += w D[nu si], K'[nu la] += w D[mu si], K'[mu si] += w D[nu la], K'[nu si] += w D[mu la]
    Jr, Kr = np.zeros((n, n)), np.zeros((n, n))
    for a in range(nf[0]):
        for b in range(nf[1]):
            for c in range(nf[2]):
                for d in range(nf[3]):
                    mu, nu, la, si = f0[0] + a, f0[1] + b, f0[2] + c, f0[3] + d
                    wv = s * eri[a, b, c, d]
                    Jr[mu, nu] += 2 * wv * D[la, si]
                    Jr[la, si] += 2 * wv * D[mu, nu]
                    Kr[mu, la] += wv * D[nu, si]
                    Kr[nu, la] += wv * D[mu, si]
                    Kr[mu, si] += wv * D[nu, la]
                    Kr[nu, si] += wv * D[mu, la]
    # primitive pairs as the library forms them
    def pairs(s1, s2):
        w1, w2 = _norm_coefs(s1), _norm_coefs(s2)
        rows = []
        for i, a in enumerate(s1.exps):
            for j, b in enumerate(s2.exps):
                row = np.zeros(11)
                host_jk[k].host_prim_pair(ctypes.c_double(a), p(np.asarray(s1.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(w1[i]), ctypes.c_double(b),
                                          p(np.asarray(s2.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(w2[j]), p(row, ctypes.c_double))
                rows.append(row)
        return np.ascontiguousarray(np.array(rows))
    pab, pcd = pairs(shells[0], shells[1]), pairs(shells[2], shells[3])
    scale = max(np.abs(Jr).max(), np.abs(Kr).max())
    for split in (0, 1):
        J, K = np.zeros((n, n)), np.zeros((n, n))
        assert host_jk[k].host_jk_quartet(len(pab), p(pab, ctypes.c_double), len(pcd), p(pcd, ctypes.c_double),
                                          int(f0[0]), int(f0[1]), int(f0[2]), int(f0[3]), ctypes.c_double(s),
                                          p(D, ctypes.c_double), p(J, ctypes.c_double), p(K, ctypes.c_double), n,
                                          split) == 0
        assert np.abs(J - Jr).max() <= 1e-12 * scale and np.abs(K - Kr).max() <= 1e-12 * scale, (cls, split)
    assert host_jk[k].host_jk_nchunk() >= 1


@pytest.mark.parametrize("k", range(21))
def test_jk_kernels_on_a_work_list(k, host_classes, host_jk):
    """The library's jk_kernel (1 and 3 quartets per lane, one and two blocks) and jk_split_kernel run on
    the host over every canonical quartet of one class in a six-shell basis (two s, two p, two d, contracted):
    J' and K' equal the digestion of each quartet's ERI block with its symmetry weight."""
    X = next(x for x in range(6) if (x + 1) * (x + 2) // 2 > k)
    Y = k - X * (X + 1) // 2
    pair_L = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
    npool = 16
    pool = W.shell_pool(npool, seed=W.SEED0 + 2300, box=3.0)
    basis = [L * npool + i for L in range(3) for i in range(2)]          # pool indices, s s p p d d
    Ls = [pool[b].L for b in basis]
    nf = [(L + 1) * (L + 2) // 2 for L in Ls]
    f0 = np.concatenate([[0], np.cumsum(nf)[:-1]]).astype(np.int32)
    n = int(sum(nf))

    def pairs_of(cls_idx):
        la, lb = pair_L[cls_idx]
        return [(a, b) for a in range(6) for b in range(6)
                if Ls[a] == la and Ls[b] == lb and (la > lb or a >= b)]

    bra_pairs, ket_pairs = pairs_of(X), pairs_of(Y)
    same = X == Y
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    # primitive pairs of every bra and ket pair in one table
    rows, ppo, npp = [], {}, {}
    for (a, b) in sorted(set(bra_pairs) | set(ket_pairs)):
        sa, sb = pool[basis[a]], pool[basis[b]]
        wa, wb = _norm_coefs(sa), _norm_coefs(sb)
        ppo[(a, b)] = len(rows)
        for i, ea in enumerate(sa.exps):
            for j, eb in enumerate(sb.exps):
                row = np.zeros(11)
                host_jk[k].host_prim_pair(ctypes.c_double(ea), p(np.asarray(sa.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wa[i]), ctypes.c_double(eb),
                                          p(np.asarray(sb.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wb[j]), p(row, ctypes.c_double))
                rows.append(row)
        npp[(a, b)] = len(rows) - ppo[(a, b)]
    P = np.ascontiguousarray(np.array(rows).T)                            # 11 arrays of np entries

    def lists(prs):
        return (np.array([a for a, _ in prs], dtype=np.int32), np.array([b for _, b in prs], dtype=np.int32),
                np.array([ppo[x] for x in prs], dtype=np.int32), np.array([npp[x] for x in prs], dtype=np.int32),
                np.ones(len(prs)))

    bra, ket = lists(bra_pairs), lists(ket_pairs)
    counts = [i + 1 if same else len(ket_pairs) for i in range(len(bra_pairs))]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    rng = np.random.default_rng(100 + k)
    D = rng.normal(size=(n, n))
    D = D + D.T
    # reference: every canonical quartet's ERI block, digested with its weight
    Jr, Kr = np.zeros((n, n)), np.zeros((n, n))
    for i, (a, b) in enumerate(bra_pairs):
        for j in range(counts[i]):
            c, d = ket_pairs[j]
            L4, npr, ex, co, cen = _pack(pool, np.asarray([[basis[a], basis[b], basis[c], basis[d]]]))
            blk = np.zeros(nf[a] * nf[b] * nf[c] * nf[d])
            assert host_classes[k].host_md_eri(ctypes.c_longlong(1), p(L4, ctypes.c_int), p(npr, ctypes.c_int),
                                               p(ex, ctypes.c_double), p(co, ctypes.c_double),
                                               p(cen, ctypes.c_double), p(blk, ctypes.c_double)) == 0
            blk = blk.reshape(nf[a], nf[b], nf[c], nf[d])
            s = (0.5 if a == b else 1.0) * (0.5 if c == d else 1.0) * (0.5 if same and i == j else 1.0)
            for x in range(nf[a]):
                for y in range(nf[b]):
                    for z in range(nf[c]):
                        for t in range(nf[d]):
                            mu, nu, la, si = f0[a] + x, f0[b] + y, f0[c] + z, f0[d] + t
                            wv = s * blk[x, y, z, t]
                            Jr[mu, nu] += 2 * wv * D[la, si]
                            Jr[la, si] += 2 * wv * D[mu, nu]
                            Kr[mu, la] += wv * D[nu, si]
                            Kr[nu, la] += wv * D[mu, si]
                            Kr[mu, si] += wv * D[nu, la]
                            Kr[nu, si] += wv * D[mu, la]
    scale = max(np.abs(Jr).max(), np.abs(Kr).max())
    for split, run, grid in ((0, 1, 1), (0, 3, 2), (1, 1, 2)):
        J, K = np.zeros((n, n)), np.zeros((n, n))
        rc = host_jk[k].host_jk_kernel(split, run, grid, len(bra_pairs), *(p(x, ctypes.c_int) for x in bra[:4]),
                                       p(bra[4], ctypes.c_double), len(ket_pairs),
                                       *(p(x, ctypes.c_int) for x in ket[:4]), p(ket[4], ctypes.c_double),
                                       p(P, ctypes.c_double), P.shape[1], p(offs, ctypes.c_longlong), int(same),
                                       p(f0, ctypes.c_int), p(D, ctypes.c_double), p(J, ctypes.c_double),
                                       p(K, ctypes.c_double), n)
        assert rc == 0
        assert np.abs(J - Jr).max() <= 1e-12 * scale and np.abs(K - Kr).max() <= 1e-12 * scale, (k, split, run, grid)


def _device_basis(pool):
    """The pool as the library's device basis holds it (normalised coefficients)."""
    L = np.array([sh.L for sh in pool], dtype=np.int32)
    nprim = np.array([len(sh.exps) for sh in pool], dtype=np.int32)
    prim0 = np.concatenate([[0], np.cumsum(nprim)[:-1]]).astype(np.int32)
    cen = np.ascontiguousarray(np.array([sh.centre for sh in pool], dtype=float).reshape(-1))
    alpha = np.concatenate([np.asarray(sh.exps, dtype=float) for sh in pool])
    coef = np.concatenate([_norm_coefs(sh) for sh in pool])
    return L, nprim, prim0, cen, alpha, coef


@pytest.mark.parametrize("k", range(21))
def test_eri_batch_kernel(k, host_jk, oracle_mod):
    """eri_batch_kernel, the library's direct ERI-batch kernel, run on the host over a contracted batch on
    two blocks: the oracle's integrals to 1e-12."""
    cls = W.quartet_classes()[k]
    npool = 16
    pool = W.shell_pool(npool, seed=W.SEED0 + 2500, box=3.0)
    q = np.ascontiguousarray(W.eri_class_batch(cls, 300, npool, seed=W.SEED0 + 2500 + k), dtype=np.int32)
    L, nprim, prim0, cen, alpha, coef = _device_basis(pool)
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.full(len(q) * blk, np.nan)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    assert host_jk[k].host_eri_batch_kernel(2, len(pool), p(L, ctypes.c_int), p(nprim, ctypes.c_int),
                                            p(prim0, ctypes.c_int), p(cen, ctypes.c_double),
                                            p(alpha, ctypes.c_double), p(coef, ctypes.c_double),
                                            ctypes.c_longlong(len(q)), p(q, ctypes.c_int), p(out, ctypes.c_double)) == 0
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    err = np.abs(out - ref).max()
    assert err <= ERI_ABS and err <= 1e-12 * np.abs(ref).max(), (cls, err)


@pytest.mark.parametrize("k", [0, 2, 5, 9, 14, 20])
def test_schwarz_kernels(k, host_jk, oracle_mod):
    """schwarz_kernel and schwarz_split_kernel (per-chunk maxima merged with an atomic max on the bit
    pattern) give the same Schwarz bounds, equal to sqrt(max |(ab|ab)|) of the oracle's diagonal quartets."""
    X = next(x for x in range(6) if (x + 1) * (x + 2) // 2 > k)
    la, lb = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)][X]
    npool = 16
    pool = W.shell_pool(npool, seed=W.SEED0 + 2600, box=3.0)
    pairs = [(la * npool + a, lb * npool + b) for a in range(4) for b in range(4) if la > lb or a >= b]
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rows, ppo, npp = [], [], []
    for (a, b) in pairs:
        sa, sb = pool[a], pool[b]
        wa, wb = _norm_coefs(sa), _norm_coefs(sb)
        ppo.append(len(rows))
        for i, ea in enumerate(sa.exps):
            for j, eb in enumerate(sb.exps):
                row = np.zeros(11)
                host_jk[k].host_prim_pair(ctypes.c_double(ea), p(np.asarray(sa.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wa[i]), ctypes.c_double(eb),
                                          p(np.asarray(sb.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wb[j]), p(row, ctypes.c_double))
                rows.append(row)
        npp.append(len(rows) - ppo[-1])
    P = np.ascontiguousarray(np.array(rows).T)
    sa_ = np.array([a for a, _ in pairs], dtype=np.int32)
    sb_ = np.array([b for _, b in pairs], dtype=np.int32)
    ppo, npp = np.array(ppo, dtype=np.int32), np.array(npp, dtype=np.int32)
    Qs = []
    for split in (0, 1):
        Q = np.full(len(pairs), np.nan)
        assert host_jk[k].host_schwarz_kernel(split, 2, len(pairs), p(sa_, ctypes.c_int), p(sb_, ctypes.c_int),
                                              p(ppo, ctypes.c_int), p(npp, ctypes.c_int), p(P, ctypes.c_double),
                                              P.shape[1], p(Q, ctypes.c_double)) == 0
        Qs.append(Q)
    q = np.array([[a, b, a, b] for a, b in pairs], dtype=np.int32)
    na, nb = (la + 1) * (la + 2) // 2, (lb + 1) * (lb + 2) // 2
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(len(pairs), na, nb, na, nb)
    Qref = np.sqrt(np.abs(np.einsum("iabab->iab", ref)).reshape(len(pairs), -1).max(axis=1))
    np.testing.assert_allclose(Qs[0], Qref, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(Qs[1], Qs[0], rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("k", range(21))
def test_eri_batch_hrr_kernel(k, host_jk, oracle_mod):
    """eri_batch_hrr_kernel (the HRR form of the ERI-batch kernel, not yet instantiated by the library) run on
    the host over a batch of contracted quartets on two blocks: the oracle's integrals to 1e-12."""
    cls = W.quartet_classes()[k]
    npool = 16
    pool = W.shell_pool(npool, seed=W.SEED0 + 2400, box=3.0)
    q = np.ascontiguousarray(W.eri_class_batch(cls, 150, npool, seed=W.SEED0 + 2400 + k), dtype=np.int32)
    L = np.array([sh.L for sh in pool], dtype=np.int32)
    nprim = np.array([len(sh.exps) for sh in pool], dtype=np.int32)
    prim0 = np.concatenate([[0], np.cumsum(nprim)[:-1]]).astype(np.int32)
    cen = np.ascontiguousarray(np.array([sh.centre for sh in pool], dtype=float).reshape(-1))
    alpha = np.concatenate([np.asarray(sh.exps, dtype=float) for sh in pool])
    coef = np.concatenate([_norm_coefs(sh) for sh in pool])
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.full(len(q) * blk, np.nan)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    assert host_jk[k].host_eri_hrr_kernel(2, len(pool), p(L, ctypes.c_int), p(nprim, ctypes.c_int),
                                          p(prim0, ctypes.c_int), p(cen, ctypes.c_double), p(alpha, ctypes.c_double),
                                          p(coef, ctypes.c_double), ctypes.c_longlong(len(q)), p(q, ctypes.c_int),
                                          p(out, ctypes.c_double)) == 0
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    err = np.abs(out - ref).max()
    assert err <= ERI_ABS and err <= 1e-12 * np.abs(ref).max(), (cls, err)


@pytest.mark.parametrize("k", [0, 4, 8, 13, 17, 20])
def test_jk_kernels_on_a_batch_work_list(k, host_classes, host_jk):
    """The J/K kernels on two molecules packed in one work list (per-pair molecules, kets from the bra's
    molecule segment, packed D/J'/K'), with both molecules active and with one switched off as a batched
    SCF does when it converges: each molecule's block equals its own quartets' digestion, and a switched-off
    molecule's block stays zero."""
    X = next(x for x in range(6) if (x + 1) * (x + 2) // 2 > k)
    Y = k - X * (X + 1) // 2
    pair_L = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
    npool = 16
    pool = W.shell_pool(npool, seed=W.SEED0 + 2700, box=3.0)
    mols = [[L * npool + 2 * m + i for L in range(3) for i in range(2)] for m in range(2)]   # pool indices
    Ls = [pool[b].L for b in mols[0]]
    nf = [(L + 1) * (L + 2) // 2 for L in Ls]
    f0_local = np.concatenate([[0], np.cumsum(nf)[:-1]]).astype(int)
    nm = int(sum(nf))
    shells = [b for m in mols for b in m]                 # global shell order: molecule 0, then 1
    f0 = np.array([f0_local[i % 6] for i in range(12)], dtype=np.int32)
    mol_of = [i // 6 for i in range(12)]
    mol_off = np.array([0, nm * nm, 2 * nm * nm], dtype=np.int64)
    mol_n = np.array([nm, nm], dtype=np.int32)

    def pairs_of(cls_idx):
        la, lb = pair_L[cls_idx]
        out = []
        for m in range(2):
            loc = range(6 * m, 6 * m + 6)
            out += [(a, b) for a in loc for b in loc if Ls[a % 6] == la and Ls[b % 6] == lb and (la > lb or a >= b)]
        return out

    bra_pairs, ket_pairs = pairs_of(X), pairs_of(Y)
    same = X == Y
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rows, ppo, npp = [], {}, {}
    for (a, b) in sorted(set(bra_pairs) | set(ket_pairs)):
        sa, sb = pool[shells[a]], pool[shells[b]]
        wa, wb = _norm_coefs(sa), _norm_coefs(sb)
        ppo[(a, b)] = len(rows)
        for i, ea in enumerate(sa.exps):
            for j, eb in enumerate(sb.exps):
                row = np.zeros(11)
                host_jk[k].host_prim_pair(ctypes.c_double(ea), p(np.asarray(sa.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wa[i]), ctypes.c_double(eb),
                                          p(np.asarray(sb.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wb[j]), p(row, ctypes.c_double))
                rows.append(row)
        npp[(a, b)] = len(rows) - ppo[(a, b)]
    P = np.ascontiguousarray(np.array(rows).T)

    def lists(prs):
        return (np.array([a for a, _ in prs], dtype=np.int32), np.array([b for _, b in prs], dtype=np.int32),
                np.array([ppo[x] for x in prs], dtype=np.int32), np.array([npp[x] for x in prs], dtype=np.int32),
                np.ones(len(prs)), np.array([mol_of[a] for a, _ in prs], dtype=np.int32))

    bra, ket = lists(bra_pairs), lists(ket_pairs)
    seg = {m: [j for j, (a, _) in enumerate(ket_pairs) if mol_of[a] == m] for m in range(2)}
    kbase = np.array([seg[mol_of[a]][0] for a, _ in bra_pairs], dtype=np.int32)
    counts = [(i - kbase[i] + 1) if same else len(seg[mol_of[a]]) for i, (a, _) in enumerate(bra_pairs)]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    rng = np.random.default_rng(200 + k)
    Dm = []
    for m in range(2):
        x = rng.normal(size=(nm, nm))
        Dm.append(x + x.T)
    D = np.concatenate([d.reshape(-1) for d in Dm])
    refs = [(np.zeros((nm, nm)), np.zeros((nm, nm))) for _ in range(2)]
    for i, (a, b) in enumerate(bra_pairs):
        m = mol_of[a]
        Jr, Kr = refs[m]
        Dl = Dm[m]
        for jj in range(counts[i]):
            j = kbase[i] + jj
            c, d = ket_pairs[j]
            L4, npr, ex, co, cen = _pack(pool, np.asarray([[shells[a], shells[b], shells[c], shells[d]]]))
            na, nb, nc, nd = (nf[a % 6], nf[b % 6], nf[c % 6], nf[d % 6])
            blk = np.zeros(na * nb * nc * nd)
            assert host_classes[k].host_md_eri(ctypes.c_longlong(1), p(L4, ctypes.c_int), p(npr, ctypes.c_int),
                                               p(ex, ctypes.c_double), p(co, ctypes.c_double),
                                               p(cen, ctypes.c_double), p(blk, ctypes.c_double)) == 0
            blk = blk.reshape(na, nb, nc, nd)
            s_ = (0.5 if a == b else 1.0) * (0.5 if c == d else 1.0) * (0.5 if same and i == j else 1.0)
            for x in range(na):
                for y in range(nb):
                    for z in range(nc):
                        for t in range(nd):
                            mu, nu, la, si = f0[a] + x, f0[b] + y, f0[c] + z, f0[d] + t
                            wv = s_ * blk[x, y, z, t]
                            Jr[mu, nu] += 2 * wv * Dl[la, si]
                            Jr[la, si] += 2 * wv * Dl[mu, nu]
                            Kr[mu, la] += wv * Dl[nu, si]
                            Kr[nu, la] += wv * Dl[mu, si]
                            Kr[mu, si] += wv * Dl[nu, la]
                            Kr[nu, si] += wv * Dl[mu, la]
    scale = max(max(np.abs(r).max() for r in pair) for pair in refs)
    for active in (None, (1, 1), (1, 0), (0, 1)):
        act = None if active is None else np.array(active, dtype=np.int32)
        for split, run, grid in ((0, 1, 1), (0, 3, 2), (1, 1, 2)):
            J, K = np.zeros_like(D), np.zeros_like(D)
            rc = host_jk[k].host_jk_kernel_batch(
                split, run, grid, len(bra_pairs), *(p(x, ctypes.c_int) for x in bra[:4]), p(bra[4], ctypes.c_double),
                p(bra[5], ctypes.c_int), len(ket_pairs), *(p(x, ctypes.c_int) for x in ket[:4]),
                p(ket[4], ctypes.c_double), p(ket[5], ctypes.c_int), p(P, ctypes.c_double), P.shape[1],
                p(offs, ctypes.c_longlong), p(kbase, ctypes.c_int), int(same), p(f0, ctypes.c_int), 2,
                p(mol_off, ctypes.c_longlong), p(mol_n, ctypes.c_int),
                p(act, ctypes.c_int) if act is not None else None, p(D, ctypes.c_double), p(J, ctypes.c_double),
                p(K, ctypes.c_double))
            assert rc == 0
            for m in range(2):
                Jm = J[mol_off[m]:mol_off[m + 1]].reshape(nm, nm)
                Km = K[mol_off[m]:mol_off[m + 1]].reshape(nm, nm)
                on = active is None or active[m] == 1
                Jr, Kr = refs[m] if on else (np.zeros((nm, nm)), np.zeros((nm, nm)))
                assert np.abs(Jm - Jr).max() <= 1e-12 * scale and np.abs(Km - Kr).max() <= 1e-12 * scale, \
                    (k, active, split, run, m)


@pytest.mark.parametrize("k", range(21))
def test_generated_class_hrr_form_fp32(k, host_classes, oracle_mod):
    """The HRR form in FP32 (recurrences included), on the 12-bohr box of the benchmark's shells, where the
    displacements A - B and C - D that the recurrences multiply by are largest.  The recurrences amplify
    FP32 rounding: (dd|pp) and (dd|dd) reach 2.6e-5 and 3.2e-5 of the batch's largest integral, above the
    2e-5 bar the direct FP32 form meets (it stays within 3.3e-7), so the FP32 form keeps the direct
    evaluation; this test records the bound (1e-4) that the FP32 HRR numbers stay within."""
    cls = W.quartet_classes()[k]
    pool = W.shell_pool(16, seed=W.SEED0 + 2800)
    q = W.eri_class_batch(cls, NQ, 16, seed=W.SEED0 + 2800 + k)
    L, npr, ex, co, cen = _pack(pool, q)
    blk = int(np.prod([(l + 1) * (l + 2) // 2 for l in cls]))
    out = np.zeros(NQ * blk, dtype=np.float32)
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    assert host_classes[k].host_md_eri_hrr_f32(ctypes.c_longlong(NQ), p(L, ctypes.c_int), p(npr, ctypes.c_int),
                                               p(ex, ctypes.c_double), p(co, ctypes.c_double),
                                               p(cen, ctypes.c_double), p(out, ctypes.c_float)) == 0
    ref = oracle_mod.OracleBasis(pool).eri_batch(q).reshape(-1)
    rel = np.abs(out.astype(np.float64) - ref).max() / np.abs(ref).max()
    assert rel <= 1e-4, (cls, rel)


@pytest.mark.parametrize("k", [2, 5, 12, 14, 20])
def test_jk_precision_bands_partition_the_build(k, host_jk):
    """A mixed-precision build is two launches per class: FP64 over the quartets with bound Q_ab Q_cd in
    [t, inf) and FP32 over [0, t).  With unequal Schwarz bounds, the two FP64 halves add up to the whole FP64
    build (every quartet in exactly one band), and the mixed and the all-FP32 builds stay within the FP32
    bar of it."""
    X = next(x for x in range(6) if (x + 1) * (x + 2) // 2 > k)
    Y = k - X * (X + 1) // 2
    pair_L = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
    npool = 16
    pool = W.shell_pool(npool, seed=W.SEED0 + 2900, box=3.0)
    basis = [L * npool + i for L in range(3) for i in range(2)]
    Ls = [pool[b].L for b in basis]
    nf = [(L + 1) * (L + 2) // 2 for L in Ls]
    f0 = np.concatenate([[0], np.cumsum(nf)[:-1]]).astype(np.int32)
    n = int(sum(nf))

    def pairs_of(c):
        la, lb = pair_L[c]
        return [(a, b) for a in range(6) for b in range(6) if Ls[a] == la and Ls[b] == lb and (la > lb or a >= b)]

    bra_pairs, ket_pairs = pairs_of(X), pairs_of(Y)
    same = X == Y
    p = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    rows, ppo, npp = [], {}, {}
    for (a, b) in sorted(set(bra_pairs) | set(ket_pairs)):
        sa, sb = pool[basis[a]], pool[basis[b]]
        wa, wb = _norm_coefs(sa), _norm_coefs(sb)
        ppo[(a, b)] = len(rows)
        for i, ea in enumerate(sa.exps):
            for j, eb in enumerate(sb.exps):
                row = np.zeros(11)
                host_jk[k].host_prim_pair(ctypes.c_double(ea), p(np.asarray(sa.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wa[i]), ctypes.c_double(eb),
                                          p(np.asarray(sb.centre, dtype=float), ctypes.c_double),
                                          ctypes.c_double(wb[j]), p(row, ctypes.c_double))
                rows.append(row)
        npp[(a, b)] = len(rows) - ppo[(a, b)]
    P = np.ascontiguousarray(np.array(rows).T)
    rng = np.random.default_rng(300 + k)
    Qof = {x: float(rng.uniform(0.1, 10.0)) for x in set(bra_pairs) | set(ket_pairs)}

    def lists(prs):
        return (np.array([a for a, _ in prs], dtype=np.int32), np.array([b for _, b in prs], dtype=np.int32),
                np.array([ppo[x] for x in prs], dtype=np.int32), np.array([npp[x] for x in prs], dtype=np.int32),
                np.array([Qof[x] for x in prs]))

    bra, ket = lists(bra_pairs), lists(ket_pairs)
    counts = [i + 1 if same else len(ket_pairs) for i in range(len(bra_pairs))]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    bounds = [bra[4][i] * ket[4][j] for i in range(len(bra_pairs)) for j in range(counts[i])]
    t = float(np.median(bounds))
    D = rng.normal(size=(n, n))
    D = D + D.T

    def build(fp32, lo, hi):
        J, K = np.zeros((n, n)), np.zeros((n, n))
        assert host_jk[k].host_jk_kernel_band(fp32, ctypes.c_double(lo), ctypes.c_double(hi), len(bra_pairs),
                                              *(p(x, ctypes.c_int) for x in bra[:4]), p(bra[4], ctypes.c_double),
                                              len(ket_pairs), *(p(x, ctypes.c_int) for x in ket[:4]),
                                              p(ket[4], ctypes.c_double), p(P, ctypes.c_double), P.shape[1],
                                              p(offs, ctypes.c_longlong), int(same), p(f0, ctypes.c_int),
                                              p(D, ctypes.c_double), p(J, ctypes.c_double), p(K, ctypes.c_double),
                                              n) == 0
        return J, K

    inf = float("inf")
    J, K = build(0, 0.0, inf)
    scale = max(np.abs(J).max(), np.abs(K).max())
    lo64, hi64 = build(0, 0.0, t), build(0, t, inf)
    assert np.abs(lo64[0]).max() > 0 and np.abs(hi64[0]).max() > 0           # both bands hold quartets
    assert np.abs(lo64[0] + hi64[0] - J).max() <= 1e-13 * scale
    assert np.abs(lo64[1] + hi64[1] - K).max() <= 1e-13 * scale
    lo32 = build(1, 0.0, t)
    for Jm, Km in ((lo32[0] + hi64[0], lo32[1] + hi64[1]), build(1, 0.0, inf)):
        assert 0 < max(np.abs(Jm - J).max(), np.abs(Km - K).max()) <= 2e-5 * scale
