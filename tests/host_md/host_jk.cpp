// host_jk.cpp -- test harness: the library's J/K digestion sink (JKSink in qchem_b200/csrc/eri_kernels.cuh)
// driven by the generated code of ONE quartet class on the host, for one shell quartet at a time.  It
// digests either the whole quartet (as jk_kernel does) or chunk by chunk, each chunk with its own sink and
// a row flush after every primitive quartet (as jk_split_kernel does).  Build with the CUDA stand-in first
// on the include path:
//   g++ -std=c++17 -O1 -fPIC -shared -DQCG_CLASS=<k> -I tests/host_md/shim -I <csrc> host_jk.cpp -o ...
#include <cmath>
#include <vector>

#include <cuda_runtime.h>   // the stand-in from tests/host_md/shim, before any library header
#include "eri_kernels.cuh"
#include "boys_table.h"

HostDim3 blockIdx, threadIdx, blockDim, gridDim;
namespace qcg {
// the kernels' shared-memory window: per-thread R slices of up to 165 entries at a stride of the block size
double qcg_smem[128 * 165];
}

#define HJ_STR2(x) #x
#define HJ_STR(x) HJ_STR2(x)
#define HJ_CAT2(a, b) a##b
#define HJ_CAT(a, b) HJ_CAT2(a, b)
#include HJ_STR(gen/HJ_CAT(md_class_, QCG_CLASS).cuh)

namespace {
constexpr int kPairLAh[6] = {0, 1, 1, 2, 2, 2}, kPairLBh[6] = {0, 0, 1, 0, 1, 2};
constexpr int cls_X()
{
    int X = 0;
    while ((X + 1) * (X + 2) / 2 <= QCG_CLASS) ++X;
    return X;
}
constexpr int kX = cls_X(), kY = QCG_CLASS - kX * (kX + 1) / 2;
constexpr int LA = kPairLAh[kX], LB = kPairLBh[kX], LC = kPairLAh[kY], LD = kPairLBh[kY];
using Sink = qcg::JKSink<double, LA, LB, LC, LD>;
}   // namespace

extern "C" int host_jk_nchunk() { return HJ_CAT(qcg::gen::kNChunk, QCG_CLASS); }

// One quartet of primitive pairs: npa x npc primitive pairs given as PrimPairData rows (11 doubles each:
// p, P, PA, PB, K), function offsets fa fb fc fd into the n x n matrices, symmetry weight s.  Adds the
// quartet's contributions to J' and K' (row-major n x n).  split = 0: the whole quartet through one sink;
// split = 1: every ket-component chunk through its own sink, with a row flush after each primitive quartet.
extern "C" int host_jk_quartet(int npa, const double* pa, int npc, const double* pc, int fa, int fb, int fc, int fd,
                               double s, const double* D, double* J, double* K, int n, int split)
{
    auto load = [](const double* r) {
        qcg::PrimPairData d;
        d.p = r[0];
        d.Px = r[1]; d.Py = r[2]; d.Pz = r[3];
        d.PAx = r[4]; d.PAy = r[5]; d.PAz = r[6];
        d.PBx = r[7]; d.PBy = r[8]; d.PBz = r[9];
        d.K = r[10];
        return d;
    };
    std::vector<double> rs(qcg::nherm(16));
    const int nchunk = split ? HJ_CAT(qcg::gen::kNChunk, QCG_CLASS) : 1;
    for (int c = 0; c < nchunk; ++c)
    {
        Sink sink;
        sink.D = D;
        sink.J = J;
        sink.K = K;
        sink.n = n;
        sink.set_bra(fa, fb);
        sink.fc = fc;
        sink.fd = fd;
        sink.s = s;
        for (int x = 0; x < npa; ++x)
            for (int y = 0; y < npc; ++y)
            {
                const qcg::PrimPairData ab = load(pa + 11 * x), cd = load(pc + 11 * y);
                if (split)
                {
                    HJ_CAT(qcg::gen::prim_quartet_chunk_, QCG_CLASS)<double, Sink>(c, ab, cd, kBoysTable, rs.data(),
                                                                                  1, sink);
                    sink.flush_k_row();
                }
                else
                    HJ_CAT(qcg::gen::prim_quartet_, QCG_CLASS)<double, Sink>(ab, cd, kBoysTable, rs.data(), 1, sink);
            }
        sink.flush_bra();
    }
    return 0;
}

// the primitive-pair row of two primitives, as the library forms it (make_prim_pair)
extern "C" void host_prim_pair(double a, const double* A, double ca, double b, const double* B, double cb,
                               double* row)
{
    const qcg::PrimPairData d = qcg::make_prim_pair(a, A[0], A[1], A[2], ca, b, B[0], B[1], B[2], cb);
    const double v[11] = {d.p, d.Px, d.Py, d.Pz, d.PAx, d.PAy, d.PAz, d.PBx, d.PBy, d.PBz, d.K};
    for (int k = 0; k < 11; ++k) row[k] = v[k];
}

namespace {
// the class wrapper the kernels expect (as qchem_b200/csrc/eri_class.cu defines it)
struct Cls
{
    static constexpr int LA = ::LA, LB = ::LB, LC = ::LC, LD = ::LD;
    static constexpr bool kRShared = HJ_CAT(qcg::gen::kRShared, QCG_CLASS);
    static constexpr bool kChunked = HJ_CAT(qcg::gen::kChunked, QCG_CLASS);
    static constexpr int kRSize = HJ_CAT(qcg::gen::kRSize, QCG_CLASS);
    static constexpr int kNChunk = HJ_CAT(qcg::gen::kNChunk, QCG_CLASS);
    template <class RT, class S, bool LOCKSTEP = false>
    static void quartet(const qcg::PrimPairData& ab, const qcg::PrimPairData& cd, const double* bt, RT* rs,
                        int stride, S& sink)
    {
        HJ_CAT(qcg::gen::prim_quartet_, QCG_CLASS)<RT, S, LOCKSTEP>(ab, cd, bt, rs, stride, sink);
    }
    template <class RT, class S>
    static void quartet_chunk(int c, const qcg::PrimPairData& ab, const qcg::PrimPairData& cd, const double* bt,
                              RT* rs, int stride, S& sink)
    {
        HJ_CAT(qcg::gen::prim_quartet_chunk_, QCG_CLASS)<RT, S>(c, ab, cd, bt, rs, stride, sink);
    }
};
constexpr int kThreads = Cls::kRShared ? 64 : 128;   // the library's block size for the class
}   // namespace

// The library's J/K kernels over a hand-made work list, every (block, thread) of the grid run in turn:
// split = 0 runs jk_kernel with `run` quartets per lane, split = 1 runs jk_split_kernel.  Pair lists are
// (sa, sb, ppo, npp, Q) per pair; P holds the primitive pairs as 11 arrays of np entries (p, P, PA, PB, K);
// offs[i] .. offs[i+1] are bra pair i's quartets (kets from 0).  No density screening, no precision band.
extern "C" int host_jk_kernel(int split, int run, int grid, int nbra, const int* bsa, const int* bsb,
                              const int* bppo, const int* bnpp, const double* bQ, int nket, const int* ksa,
                              const int* ksb, const int* kppo, const int* knpp, const double* kQ, const double* P,
                              int np, const long long* offs, int same_class, const int* f0, const double* D, double* J,
                              double* K, int n)
{
    if (kThreads * Cls::kRSize > 128 * 165) return 1;
    qcg::PairListDev bra{nbra, bsa, bsb, bppo, bnpp, bQ, nullptr}, ket{nket, ksa, ksb, kppo, knpp, kQ, nullptr};
    qcg::PrimPairsDev pp{P, P + np, P + 2 * np, P + 3 * np, P + 4 * np, P + 5 * np, P + 6 * np, P + 7 * np,
                         P + 8 * np, P + 9 * np, P + 10 * np};
    qcg::JKWorkDev w{};
    w.total = offs[nbra];
    w.gbeg = 0;
    w.gend = w.total;
    w.offs = offs;
    w.same_class = same_class;
    w.lo = 0.0;
    w.hi = HUGE_VAL;
    w.mols = qcg::MolLayoutDev{1, nullptr, nullptr};
    blockDim.x = kThreads;
    gridDim.x = grid;
    for (int b = 0; b < grid; ++b)
        for (int t = 0; t < kThreads; ++t)
        {
            blockIdx.x = b;
            threadIdx.x = t;
            if (split)
                qcg::jk_split_kernel<Cls, kThreads, double>(w, bra, ket, pp, f0, D, J, K, n, kBoysTable);
            else
                qcg::jk_kernel<Cls, kThreads, double>(w, bra, ket, pp, f0, D, J, K, n, kBoysTable, run);
        }
    return 0;
}

// jk_kernel over the quartets whose bound Q_ab Q_cd lies in [lo, hi) (one launch of a mixed-precision
// build), in FP64 (fp32 = 0) or FP32 (fp32 = 1) arithmetic; one block-sized grid, runs of one quartet
extern "C" int host_jk_kernel_band(int fp32, double lo, double hi, int nbra, const int* bsa, const int* bsb,
                                   const int* bppo, const int* bnpp, const double* bQ, int nket, const int* ksa,
                                   const int* ksb, const int* kppo, const int* knpp, const double* kQ,
                                   const double* P, int np, const long long* offs, int same_class, const int* f0,
                                   const double* D, double* J, double* K, int n)
{
    if (kThreads * Cls::kRSize > 128 * 165) return 1;
    qcg::PairListDev bra{nbra, bsa, bsb, bppo, bnpp, bQ, nullptr}, ket{nket, ksa, ksb, kppo, knpp, kQ, nullptr};
    qcg::PrimPairsDev pp{P, P + np, P + 2 * np, P + 3 * np, P + 4 * np, P + 5 * np, P + 6 * np, P + 7 * np,
                         P + 8 * np, P + 9 * np, P + 10 * np};
    qcg::JKWorkDev w{};
    w.total = offs[nbra];
    w.gbeg = 0;
    w.gend = w.total;
    w.offs = offs;
    w.same_class = same_class;
    w.lo = lo;
    w.hi = hi;
    w.mols = qcg::MolLayoutDev{1, nullptr, nullptr};
    const int grid = (int)((w.total + kThreads - 1) / kThreads);
    blockDim.x = kThreads;
    gridDim.x = grid;
    for (int b = 0; b < grid; ++b)
        for (int t = 0; t < kThreads; ++t)
        {
            blockIdx.x = b;
            threadIdx.x = t;
            if (fp32)
                qcg::jk_kernel<Cls, kThreads, float>(w, bra, ket, pp, f0, D, J, K, n, kBoysTable, 1);
            else
                qcg::jk_kernel<Cls, kThreads, double>(w, bra, ket, pp, f0, D, J, K, n, kBoysTable, 1);
        }
    return 0;
}

// The same kernels on several molecules packed in one work list (as a batch handle builds it): bmol/kmol
// give each pair's molecule, kbase[i] the first ket of bra pair i's molecule, mol_off/mol_n the packed
// layout of D, J', K', and mol_active (or null) the molecules still iterating.
extern "C" int host_jk_kernel_batch(int split, int run, int grid, int nbra, const int* bsa, const int* bsb,
                                    const int* bppo, const int* bnpp, const double* bQ, const int* bmol, int nket,
                                    const int* ksa, const int* ksb, const int* kppo, const int* knpp,
                                    const double* kQ, const int* kmol, const double* P, int np,
                                    const long long* offs, const int* kbase, int same_class, const int* f0,
                                    int nmol, const long long* mol_off, const int* mol_n, const int* mol_active,
                                    const double* D, double* J, double* K)
{
    if (kThreads * Cls::kRSize > 128 * 165) return 1;
    qcg::PairListDev bra{nbra, bsa, bsb, bppo, bnpp, bQ, bmol}, ket{nket, ksa, ksb, kppo, knpp, kQ, kmol};
    qcg::PrimPairsDev pp{P, P + np, P + 2 * np, P + 3 * np, P + 4 * np, P + 5 * np, P + 6 * np, P + 7 * np,
                         P + 8 * np, P + 9 * np, P + 10 * np};
    qcg::JKWorkDev w{};
    w.total = offs[nbra];
    w.gbeg = 0;
    w.gend = w.total;
    w.offs = offs;
    w.kbase = kbase;
    w.same_class = same_class;
    w.lo = 0.0;
    w.hi = HUGE_VAL;
    w.mols = qcg::MolLayoutDev{nmol, mol_off, mol_n};
    w.mol_active = mol_active;
    blockDim.x = kThreads;
    gridDim.x = grid;
    for (int b = 0; b < grid; ++b)
        for (int t = 0; t < kThreads; ++t)
        {
            blockIdx.x = b;
            threadIdx.x = t;
            if (split)
                qcg::jk_split_kernel<Cls, kThreads, double>(w, bra, ket, pp, f0, D, J, K, 0, kBoysTable);
            else
                qcg::jk_kernel<Cls, kThreads, double>(w, bra, ket, pp, f0, D, J, K, 0, kBoysTable, run);
        }
    return 0;
}

// Schwarz diagonals of a pair list of a diagonal class (Q_i = sqrt(max |(ab|ab)|)): split = 0 runs
// schwarz_kernel, split = 1 schwarz_split_kernel (Q zeroed first, as the launcher does)
extern "C" int host_schwarz_kernel(int split, int grid, int npair, const int* sa, const int* sb, const int* ppo,
                                   const int* npp, const double* P, int np, double* Q)
{
    if (kX != kY) return 1;
    qcg::PairListDev pl{npair, sa, sb, ppo, npp, nullptr, nullptr};
    qcg::PrimPairsDev pp{P, P + np, P + 2 * np, P + 3 * np, P + 4 * np, P + 5 * np, P + 6 * np, P + 7 * np,
                         P + 8 * np, P + 9 * np, P + 10 * np};
    if (split)
        for (int i = 0; i < npair; ++i) Q[i] = 0.0;
    blockDim.x = kThreads;
    gridDim.x = grid;
    for (int b = 0; b < grid; ++b)
        for (int t = 0; t < kThreads; ++t)
        {
            blockIdx.x = b;
            threadIdx.x = t;
            if (split) qcg::schwarz_split_kernel<Cls, kThreads>(pl, pp, Q, kBoysTable);
            else qcg::schwarz_kernel<Cls, kThreads>(pl, pp, Q, kBoysTable);
        }
    return 0;
}

// the library's direct ERI-batch kernel (eri_batch_kernel) over a batch of quartets, in input order
extern "C" int host_eri_batch_kernel(int grid, int nshell, const int* L, const int* nprim, const int* prim0,
                                     const double* cen, const double* alpha, const double* coef, long long nq,
                                     const int* quartets, double* out)
{
    qcg::BasisDev bs{nshell, L, nprim, prim0, cen, alpha, coef};
    blockDim.x = kThreads;
    gridDim.x = grid;
    for (int b = 0; b < grid; ++b)
        for (int t = 0; t < kThreads; ++t)
        {
            blockIdx.x = b;
            threadIdx.x = t;
            qcg::eri_batch_kernel<Cls, kThreads, double>(bs, reinterpret_cast<const int4*>(quartets), nullptr, nq, out,
                                                        kBoysTable);
        }
    return 0;
}

#ifdef HJ_HRR
// the HRR form of the class (gen_md.main_hrr) and the library's eri_batch_hrr_kernel over a batch of quartets
#include HJ_STR(gen_hrr/HJ_CAT(md_hrr_, QCG_CLASS).cuh)

namespace {
struct ClsH
{
    static constexpr int LA = ::LA, LB = ::LB, LC = ::LC, LD = ::LD;
    static constexpr int kHrrE = HJ_CAT(qcg::gen::kHrrE, QCG_CLASS), kHrrF = HJ_CAT(qcg::gen::kHrrF, QCG_CLASS);
    template <class RT, class S>
    static void quartet_hrr(const qcg::PrimPairData& ab, const qcg::PrimPairData& cd, const double* bt, RT* rs,
                            int stride, S& sink)
    {
        HJ_CAT(qcg::gen::prim_quartet_hrr_, QCG_CLASS)<RT, S>(ab, cd, bt, rs, stride, sink);
    }
    template <class RT>
    static void hrr_ket(const RT* p, RT* y, RT CDx, RT CDy, RT CDz)
    {
        HJ_CAT(qcg::gen::hrr_ket_, QCG_CLASS)<RT>(p, y, CDx, CDy, CDz);
    }
    template <class RT>
    static void hrr_bra(const RT* y, int ys, RT* o, int os, RT ABx, RT ABy, RT ABz)
    {
        HJ_CAT(qcg::gen::hrr_bra_, QCG_CLASS)<RT>(y, ys, o, os, ABx, ABy, ABz);
    }
};
}   // namespace

// basis arrays as the library's device basis holds them (coefficients already normalised), nq quartets of
// shell indices; every (block, thread) of a grid of `grid` blocks of 64 threads run in turn
extern "C" int host_eri_hrr_kernel(int grid, int nshell, const int* L, const int* nprim, const int* prim0,
                                   const double* cen, const double* alpha, const double* coef, long long nq,
                                   const int* quartets, double* out)
{
    qcg::BasisDev bs{nshell, L, nprim, prim0, cen, alpha, coef};
    constexpr int T = 64;
    blockDim.x = T;
    gridDim.x = grid;
    for (int b = 0; b < grid; ++b)
        for (int t = 0; t < T; ++t)
        {
            blockIdx.x = b;
            threadIdx.x = t;
            qcg::eri_batch_hrr_kernel<ClsH, T, double>(bs, reinterpret_cast<const int4*>(quartets), nullptr, nq, out,
                                                      kBoysTable);
        }
    return 0;
}
#endif
