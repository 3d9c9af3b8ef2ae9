// eri_class.cu -- instantiates the kernels of ONE quartet class in ONE arithmetic type; compiled with
// -DQCG_CLASS=k (k = X(X+1)/2 + Y for pair classes X >= Y) and -DQCG_PREC=64 or 32, so that the 21 classes
// of both forms build in parallel.  The FP64 objects define launch_eri_batch_k, launch_jk_k and
// launch_schwarz_k; the FP32 objects launch_eri_batch32_k and launch_jk32_k.
#include <atomic>
#include <type_traits>

#include "eri_kernels.cuh"
#include "smem_attr.h"

#ifndef QCG_CLASS
#error "compile with -DQCG_CLASS=<0..20>"
#endif
#ifndef QCG_PREC
#define QCG_PREC 64
#endif

#define QCG_STR2(x) #x
#define QCG_STR(x) QCG_STR2(x)
#define QCG_CAT2(a, b) a##b
#define QCG_CAT(a, b) QCG_CAT2(a, b)
#include QCG_STR(gen/QCG_CAT(md_class_, QCG_CLASS).cuh)
// QCG_ERI_HRR=1 (FP64 objects only; build.py sets it for the classes where it measured faster): the ERI
// batches use the horizontal-recurrence form (gen/md_hrr_<k>.cuh, eri_batch_hrr_kernel).
#ifndef QCG_ERI_HRR
#define QCG_ERI_HRR 0
#endif
#if QCG_ERI_HRR && QCG_PREC == 64
#include QCG_STR(gen/QCG_CAT(md_hrr_, QCG_CLASS).cuh)
#endif
#if QCG_PREC == 64
#define QCG_NAME(base) QCG_CAT(QCG_CAT(base, _), QCG_CLASS)
#elif QCG_PREC == 32
#define QCG_NAME(base) QCG_CAT(QCG_CAT(base, 32_), QCG_CLASS)
#else
#error "QCG_PREC must be 64 or 32"
#endif

namespace qcg {

namespace {
constexpr int cls_X()
{
    int X = 0;
    while ((X + 1) * (X + 2) / 2 <= QCG_CLASS) ++X;
    return X;
}
constexpr int kX = cls_X();
constexpr int kY = QCG_CLASS - kX * (kX + 1) / 2;
using Real = std::conditional_t<QCG_PREC == 64, double, float>;

struct Cls
{
    static constexpr int LA = kPairLA[kX], LB = kPairLB[kX], LC = kPairLA[kY], LD = kPairLB[kY];
    static constexpr bool kRShared = gen::QCG_CAT(kRShared, QCG_CLASS);
    static constexpr bool kChunked = gen::QCG_CAT(kChunked, QCG_CLASS);
    static constexpr int kRSize = gen::QCG_CAT(kRSize, QCG_CLASS);
    static constexpr int kNChunk = gen::QCG_CAT(kNChunk, QCG_CLASS);
    template <class RT, class Sink, bool LOCKSTEP = false>
    static __device__ __forceinline__ void quartet(const PrimPairData& ab, const PrimPairData& cd,
                                                   const double* __restrict__ bt, RT* __restrict__ rs, int stride,
                                                   Sink& sink)
    {
        gen::QCG_CAT(prim_quartet_, QCG_CLASS)<RT, Sink, LOCKSTEP>(ab, cd, bt, rs, stride, sink);
    }
    // ket-component chunk c of the quartet alone, after rebuilding Boys and R (chunked classes)
    template <class RT, class Sink>
    static __device__ __forceinline__ void quartet_chunk(int c, const PrimPairData& ab, const PrimPairData& cd,
                                                         const double* __restrict__ bt, RT* __restrict__ rs,
                                                         int stride, Sink& sink)
    {
        gen::QCG_CAT(prim_quartet_chunk_, QCG_CLASS)<RT, Sink>(c, ab, cd, bt, rs, stride, sink);
    }
#if QCG_ERI_HRR && QCG_PREC == 64
    // the horizontal-recurrence form (eri_batch_hrr_kernel)
    static constexpr int kHrrE = gen::QCG_CAT(kHrrE, QCG_CLASS), kHrrF = gen::QCG_CAT(kHrrF, QCG_CLASS);
    template <class RT, class Sink>
    static __device__ __forceinline__ void quartet_hrr(const PrimPairData& ab, const PrimPairData& cd,
                                                       const double* __restrict__ bt, RT* __restrict__ rs, int stride,
                                                       Sink& sink)
    {
        gen::QCG_CAT(prim_quartet_hrr_, QCG_CLASS)<RT, Sink>(ab, cd, bt, rs, stride, sink);
    }
    template <class RT>
    static __device__ __forceinline__ void hrr_ket(const RT* p, RT* y, RT CDx, RT CDy, RT CDz)
    {
        gen::QCG_CAT(hrr_ket_, QCG_CLASS)<RT>(p, y, CDx, CDy, CDz);
    }
    template <class RT>
    static __device__ __forceinline__ void hrr_bra(const RT* y, int ys, RT* o, int os, RT ABx, RT ABy, RT ABz)
    {
        gen::QCG_CAT(hrr_bra_, QCG_CLASS)<RT>(y, ys, o, os, ABx, ABy, ABz);
    }
    // the HRR code keeps R in the per-thread shared-memory slice only where the direct code does too, so the
    // direct form's block size and shared memory serve both
    static_assert(!gen::QCG_CAT(kHrrRShared, QCG_CLASS) || kRShared, "HRR R slice needs shared memory");
#endif
};

// classes whose R table lives in shared memory run 64-thread blocks (per-thread R slice); the others 128
constexpr int kThreads = Cls::kRShared ? 64 : 128;
constexpr size_t kSmem = Cls::kRShared ? (size_t)kThreads * Cls::kRSize * sizeof(Real) : 0;
// the Schwarz diagonals are always FP64
constexpr size_t kSmem64 = Cls::kRShared ? (size_t)kThreads * Cls::kRSize * sizeof(double) : 0;

// keyed on the kernel itself: instantiations that differ only in a template flag share a pointer TYPE, and
// each needs its own attribute
template <auto Kernel>
void prepare(size_t smem = kSmem)
{
    static std::atomic<unsigned long long> ready{0};
    ensure_smem(Kernel, smem, ready);
}

long long grid_for(long long work, int nsm)
{
    long long blocks = (work + kThreads - 1) / kThreads;
    const long long cap = (long long)nsm * (Cls::kRShared ? 8 : 16);
    return blocks > cap ? cap : blocks;
}
}   // namespace

// chunked classes: 128-thread blocks in lock step (one chunk of code in flight per block)
constexpr int kLockThreads = 128;
constexpr size_t kLockSmem = (size_t)kLockThreads * Cls::kRSize * sizeof(Real);

// lock step measured faster for every chunked class except FP64 (dd|dd), whose 169 KB per 128-thread
// block leaves no room for a second block (ERI microbenchmark, 10^6 quartets per class); the FP32 form
// needs half of that
constexpr bool kUseLockstep = Cls::kChunked && (QCG_CLASS != 20 || QCG_PREC == 32);

void QCG_NAME(launch_eri_batch)(const BasisDev& bs, const int4* q, const int* order, long long nq, Real* out,
                                const double* boys, cudaStream_t st, int nsm)
{
    if (nq <= 0) return;
#if QCG_ERI_HRR && QCG_PREC == 64
    {
        auto k = eri_batch_hrr_kernel<Cls, kThreads, Real>;
        static std::atomic<unsigned long long> hrr_ready{0};
        ensure_smem(k, kSmem, hrr_ready);
        k<<<(unsigned)grid_for(nq, nsm), kThreads, kSmem, st>>>(bs, q, order, nq, out, boys);
        return;
    }
#endif
    if constexpr (kUseLockstep)
    {
        auto k = eri_batch_lockstep_kernel<Cls, kLockThreads, Real>;
        static std::atomic<unsigned long long> lock_ready{0};
        ensure_smem(k, kLockSmem, lock_ready);
        long long blocks = (nq + kLockThreads - 1) / kLockThreads;
        const long long cap = (long long)nsm * 2;
        if (blocks > cap) blocks = cap;
        k<<<(unsigned)blocks, kLockThreads, kLockSmem, st>>>(bs, q, order, nq, out, boys);
    }
    else
    {
        auto k = eri_batch_kernel<Cls, kThreads, Real>;
        prepare<eri_batch_kernel<Cls, kThreads, Real>>();
        k<<<(unsigned)grid_for(nq, nsm), kThreads, kSmem, st>>>(bs, q, order, nq, out, boys);
    }
}

namespace {
// DET: the deterministic accumulation (JKWorkDev::det_lo, FP64 objects only)
template <bool DET>
void launch_jk_form(const JKWorkDev& w, const PairListDev& bra, const PairListDev& ket, const PrimPairsDev& P,
                    const int* f0, const double* D, double* J, double* K, int n, const double* boys,
                    cudaStream_t st, int nsm)
{
    const long long span = w.gend - w.gbeg;
    if constexpr (Cls::kChunked)
    {
        // at most one block of quartets per SM: a plain launch would leave most of the GPU idle while each
        // lane runs a whole quartet's code, so the quartets' ket-component chunks go to separate warps
        if (span <= (long long)nsm * kThreads)
        {
            auto ks = jk_split_kernel<Cls, kThreads, Real, DET>;
            static std::atomic<unsigned long long> split_ready{0};
            ensure_smem(ks, kSmem, split_ready);
            const long long items = ((span + 31) & ~31LL) * Cls::kNChunk;
            const long long blocks = (items + kThreads - 1) / kThreads;
            ks<<<(unsigned)blocks, kThreads, kSmem, st>>>(w, bra, ket, P, f0, D, J, K, n, boys);
            return;
        }
    }
    auto k = jk_kernel<Cls, kThreads, Real, DET>;
    prepare<jk_kernel<Cls, kThreads, Real, DET>>();
    // quartets per lane run: enough threads for the whole GPU first, longer runs only for large builds
    // (unless the autotuner chose the run and the grid cap)
    long long run = span / ((long long)nsm * 1024);
    run = run < 1 ? 1 : (run > 8 ? 8 : run);
    if (w.run > 0) run = w.run;
    const long long work = (span + run - 1) / run;
    long long blocks = grid_for(work, nsm);
    if (w.cap > 0)
    {
        blocks = (work + kThreads - 1) / kThreads;
        if (blocks > (long long)nsm * w.cap) blocks = (long long)nsm * w.cap;
    }
    k<<<(unsigned)blocks, kThreads, kSmem, st>>>(w, bra, ket, P, f0, D, J, K, n, boys, (int)run);
}
}   // namespace

void QCG_NAME(launch_jk)(const JKWorkDev& w, const PairListDev& bra, const PairListDev& ket, const PrimPairsDev& P,
                         const int* f0, const double* D, double* J, double* K, int n, const double* boys,
                         cudaStream_t st, int nsm)
{
    if (w.gend - w.gbeg <= 0) return;
#if QCG_PREC == 64
    if (w.det_lo)
    {
        launch_jk_form<true>(w, bra, ket, P, f0, D, J, K, n, boys, st, nsm);
        return;
    }
#endif
    launch_jk_form<false>(w, bra, ket, P, f0, D, J, K, n, boys, st, nsm);
}

#if QCG_PREC == 64
// the warp-shared form of the J/K build (jk_warp_kernel): one warp per work item, grid-stride
void QCG_CAT(launch_jk_warp_, QCG_CLASS)(const JKWorkDev& w, const PairListDev& bra, const PairListDev& ket,
                                          const PrimPairsDev& P, const int* f0, const double* D, double* J, double* K,
                                          int n, const double* boys, const int* gbra, const int4* items,
                                          long long nitems, cudaStream_t st, int nsm)
{
    if (nitems <= 0) return;
    auto k = jk_warp_kernel<Cls, kThreads>;
    prepare<jk_warp_kernel<Cls, kThreads>>();
    k<<<(unsigned)grid_for(nitems * 32, nsm), kThreads, kSmem, st>>>(w, bra, ket, P, f0, D, J, K, n, boys, gbra,
                                                                      items, nitems);
}

// Schwarz diagonals exist only for the diagonal classes (X == Y)
void QCG_CAT(launch_schwarz_, QCG_CLASS)(const PairListDev& pl, const PrimPairsDev& P, double* Q, const double* boys,
                                         cudaStream_t st, int nsm)
{
    if constexpr (kX == kY)
    {
        if (pl.n <= 0) return;
        if constexpr (Cls::kChunked)
        {
            // few pairs: their diagonal quartets' chunks on separate warps (see jk_split_kernel)
            if ((long long)pl.n <= (long long)nsm * kThreads)
            {
                auto ks = schwarz_split_kernel<Cls, kThreads>;
                static std::atomic<unsigned long long> split_ready{0};
                ensure_smem(ks, kSmem64, split_ready);
                cudaMemsetAsync(Q, 0, (size_t)pl.n * sizeof(double), st);
                const long long items = (((long long)pl.n + 31) & ~31LL) * Cls::kNChunk;
                ks<<<(unsigned)((items + kThreads - 1) / kThreads), kThreads, kSmem64, st>>>(pl, P, Q, boys);
                return;
            }
        }
        auto k = schwarz_kernel<Cls, kThreads>;
        prepare<schwarz_kernel<Cls, kThreads>>(kSmem64);
        k<<<(pl.n + kThreads - 1) / kThreads, kThreads, kSmem64, st>>>(pl, P, Q, boys);
    }
}
#endif

}   // namespace qcg
