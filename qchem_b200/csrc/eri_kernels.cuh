// eri_kernels.cuh -- class-specialised ERI kernels: Cartesian-ERI batches, Schwarz diagonals and the
// fused ERI + J/K digestion.  Included by eri_class.cu, which is compiled once per quartet class and
// supplies Cls::quartet (the generated straight-line primitive-quartet evaluation of that class).
#pragma once
#include "md_core.cuh"
#include "qcg_internal.h"

namespace qcg {

// ------------------------------------------------------------------------------------------------
// Cartesian ERI batch: out[q][a][b][c][d] = (ab|cd) for quartet q (shell indices), contracted and
// normalised like qchem's NR_Evaluator::FourC (PG_Cart_MnD/Evaluator.C:1912-1920).
// ------------------------------------------------------------------------------------------------
// accumulates every primitive quartet into the (zeroed) output block with fire-and-forget L2 reductions:
// the thread never reads the block back, so no loads are hoisted into registers around the ERI code
template <class RT, int LB, int LC, int LD>
struct StoreSink
{
    static constexpr bool kByValue = true;
    RT* o;
    static constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    __device__ __forceinline__ void ket_begin(int, int) {}
    __device__ __forceinline__ void ket_end(int, int) {}
    __device__ __forceinline__ void operator()(int ia, int ib, int ic, int id, RT v)
    {
        atomicAdd(o + ((ia * NB + ib) * NC + ic) * ND + id, v);
    }
};

__device__ __forceinline__ PrimPairData shell_prim_pair(const BasisDev& bs, int sa, int i, int sb, int j)
{
    const int pa = bs.prim0[sa] + i, pb = bs.prim0[sb] + j;
    return make_prim_pair(bs.alpha[pa], bs.cen[3 * sa], bs.cen[3 * sa + 1], bs.cen[3 * sa + 2], bs.coef[pa],
                          bs.alpha[pb], bs.cen[3 * sb], bs.cen[3 * sb + 1], bs.cen[3 * sb + 2], bs.coef[pb]);
}

// the same with a per-thread switch: lanes that only keep a block in step write nothing
template <class RT, int LB, int LC, int LD>
struct MaskedStoreSink
{
    static constexpr bool kByValue = true;
    RT* o;
    bool active;
    static constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    __device__ __forceinline__ void ket_begin(int, int) {}
    __device__ __forceinline__ void ket_end(int, int) {}
    __device__ __forceinline__ void operator()(int ia, int ib, int ic, int id, RT v)
    {
        if (active) atomicAdd(o + ((ia * NB + ib) * NC + ic) * ND + id, v);
    }
};

// dynamic shared memory holding the per-thread R tables of classes with L >= 6 or chunked code
extern __shared__ double qcg_smem[];

// per-thread R slice in dynamic shared memory, in the arithmetic type of the kernel
template <class RT>
__device__ __forceinline__ RT* r_slice()
{
    return reinterpret_cast<RT*>(qcg_smem) + threadIdx.x;
}

// Quartets are visited through `order` (a permutation grouping equal contraction patterns, so that the
// lanes of a warp run the same primitive loops); each writes its own output block.  RT is the arithmetic
// and output type (double, or float for the FP32 form).
template <class Cls, int THREADS, class RT>
__global__ void __launch_bounds__(THREADS) eri_batch_kernel(BasisDev bs, const int4* __restrict__ quartets,
                                                            const int* __restrict__ order, long long nq,
                                                            RT* __restrict__ out,
                                                            const double* __restrict__ boys_table)
{
    constexpr long long BLK = (long long)ncart(Cls::LA) * ncart(Cls::LB) * ncart(Cls::LC) * ncart(Cls::LD);
    RT* rs = r_slice<RT>();
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nq; g += (long long)gridDim.x * blockDim.x)
    {
        const long long q = order ? order[g] : g;
        const int4 s = quartets[q];
        RT* o = out + q * BLK;
        for (int k = 0; k < (int)BLK; ++k) o[k] = RT(0);
        StoreSink<RT, Cls::LB, Cls::LC, Cls::LD> sink{o};
        const int ni = bs.nprim[s.x], nj = bs.nprim[s.y], nk = bs.nprim[s.z], nl = bs.nprim[s.w];
        const int nket = nk * nl, ntot = ni * nj * nket;
        for (int x = 0; x < ntot; ++x)
        {
            const int ij = x / nket, kl = x - ij * nket;
            const PrimPairData ab = shell_prim_pair(bs, s.x, ij / nj, s.y, ij % nj);
            const PrimPairData cd = shell_prim_pair(bs, s.z, kl / nl, s.w, kl % nl);
            Cls::template quartet<RT>(ab, cd, boys_table, rs, THREADS, sink);
        }
    }
}

// Block-synchronous variant for the classes whose code is split into chunks: the block takes the sorted
// quartets in rounds of THREADS, every thread runs the block's largest primitive count (surplus
// iterations are masked), so all threads reach every barrier inside Cls::quartet<..., true> and the
// block's warps walk the chunk code together.
template <class Cls, int THREADS, class RT>
__global__ void __launch_bounds__(THREADS) eri_batch_lockstep_kernel(BasisDev bs, const int4* __restrict__ quartets,
                                                                     const int* __restrict__ order, long long nq,
                                                                     RT* __restrict__ out,
                                                                     const double* __restrict__ boys_table)
{
    constexpr long long BLK = (long long)ncart(Cls::LA) * ncart(Cls::LB) * ncart(Cls::LC) * ncart(Cls::LD);
    __shared__ int s_nmax;
    RT* rs = r_slice<RT>();
    for (long long base = (long long)blockIdx.x * THREADS; base < nq; base += (long long)gridDim.x * THREADS)
    {
        const long long g = base + threadIdx.x;
        const bool valid = g < nq;
        const long long gq = valid ? g : base;   // idle lanes shadow the round's first quartet
        const long long q = order ? order[gq] : gq;
        const int4 s = quartets[q];
        RT* o = out + q * BLK;
        if (valid)
            for (int k = 0; k < (int)BLK; ++k) o[k] = RT(0);
        const int ni = bs.nprim[s.x], nj = bs.nprim[s.y], nk = bs.nprim[s.z], nl = bs.nprim[s.w];
        const int nket = nk * nl, ntot = ni * nj * nket;
        if (threadIdx.x == 0) s_nmax = 0;
        __syncthreads();
        atomicMax(&s_nmax, ntot);
        __syncthreads();
        const int nmax = s_nmax;
        __syncthreads();
        MaskedStoreSink<RT, Cls::LB, Cls::LC, Cls::LD> sink{o, false};
        for (int x = 0; x < nmax; ++x)
        {
            const int xx = x < ntot ? x : 0;
            sink.active = valid && x < ntot;
            const int ij = xx / nket, kl = xx - ij * nket;
            const PrimPairData ab = shell_prim_pair(bs, s.x, ij / nj, s.y, ij % nj);
            const PrimPairData cd = shell_prim_pair(bs, s.z, kl / nl, s.w, kl % nl);
            Cls::template quartet<RT, MaskedStoreSink<RT, Cls::LB, Cls::LC, Cls::LD>, true>(ab, cd, boys_table, rs,
                                                                                           THREADS, sink);
        }
    }
}

// Cartesian ERI batch in horizontal-recurrence form (the thread-per-quartet form of the classes build.py
// lists in HRR_CLASSES, used when the team form is not; the host tests run it too).  Cls provides the generated HRR functions (gen_md.main_hrr): quartet_hrr adds a
// primitive quartet's [e0|f0] block (e over L = LA..LA+LB on centre A, f over L = LC..LC+LD on centre C)
// into the zeroed output block at row stride n_c n_d with red.global.  After the primitives, hrr_ket
// carries each e row to [e0|cd] in place, and hrr_bra carries each (c d) column to (ab|cd) in place.  The
// recurrences read back through L2 (ld_l2), where the red.global updates are.  The block always has room:
// |E| <= n_a n_b and |F| <= n_c n_d.
template <class RT, int NCD>
struct HrrRowSink
{
    RT* o;
    __device__ __forceinline__ void operator()(int ie, int jf, RT v) { atomicAdd(o + ie * NCD + jf, v); }
};

template <class Cls, int THREADS, class RT>
__global__ void __launch_bounds__(THREADS) eri_batch_hrr_kernel(BasisDev bs, const int4* __restrict__ quartets,
                                                                const int* __restrict__ order, long long nq,
                                                                RT* __restrict__ out,
                                                                const double* __restrict__ boys_table)
{
    constexpr int NCD = ncart(Cls::LC) * ncart(Cls::LD);
    constexpr long long BLK = (long long)ncart(Cls::LA) * ncart(Cls::LB) * NCD;
    static_assert(Cls::kHrrE <= ncart(Cls::LA) * ncart(Cls::LB) && Cls::kHrrF <= NCD, "[e0|f0] fits the block");
    RT* rs = r_slice<RT>();
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nq; g += (long long)gridDim.x * blockDim.x)
    {
        const long long q = order ? order[g] : g;
        const int4 s = quartets[q];
        RT* o = out + q * BLK;
        for (int k = 0; k < (int)BLK; ++k) o[k] = RT(0);
        HrrRowSink<RT, NCD> sink{o};
        const int ni = bs.nprim[s.x], nj = bs.nprim[s.y], nk = bs.nprim[s.z], nl = bs.nprim[s.w];
        const int nket = nk * nl, ntot = ni * nj * nket;
        for (int x = 0; x < ntot; ++x)
        {
            const int ij = x / nket, kl = x - ij * nket;
            const PrimPairData ab = shell_prim_pair(bs, s.x, ij / nj, s.y, ij % nj);
            const PrimPairData cd = shell_prim_pair(bs, s.z, kl / nl, s.w, kl % nl);
            Cls::template quartet_hrr<RT>(ab, cd, boys_table, rs, THREADS, sink);
        }
        const double* A = bs.cen + 3 * s.x;
        const double* B = bs.cen + 3 * s.y;
        const double* C = bs.cen + 3 * s.z;
        const double* D = bs.cen + 3 * s.w;
        const RT CDx = RT(C[0] - D[0]), CDy = RT(C[1] - D[1]), CDz = RT(C[2] - D[2]);
        const RT ABx = RT(A[0] - B[0]), ABy = RT(A[1] - B[1]), ABz = RT(A[2] - B[2]);
        for (int e = 0; e < Cls::kHrrE; ++e) Cls::template hrr_ket<RT>(o + e * NCD, o + e * NCD, CDx, CDy, CDz);
        for (int cd = 0; cd < NCD; ++cd) Cls::template hrr_bra<RT>(o + cd, NCD, o + cd, NCD, ABx, ABy, ABz);
    }
}

// ------------------------------------------------------------------------------------------------
// Pair lists: pair class X holds shell pairs (a,b) with L_a >= L_b, sorted by Schwarz bound
// descending; the primitive pairs of pair i are P[ppo[i] .. ppo[i]+npp[i]).
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ PrimPairData load_pp(const PrimPairsDev& P, int k)
{
    PrimPairData d;
    d.p = P.p[k];
    d.Px = P.Px[k]; d.Py = P.Py[k]; d.Pz = P.Pz[k];
    d.PAx = P.PAx[k]; d.PAy = P.PAy[k]; d.PAz = P.PAz[k];
    d.PBx = P.PBx[k]; d.PBy = P.PBy[k]; d.PBz = P.PBz[k];
    d.K = P.K[k];
    return d;
}

// Schwarz diagonal: Q_i = sqrt(max_{mu nu} |(mu nu|mu nu)|) for every pair of one diagonal class
template <int LA, int LB>
struct DiagSink
{
    static constexpr int NB = ncart(LB), NAB = ncart(LA) * ncart(LB);
    double acc[NAB];
    __device__ __forceinline__ void ket_begin(int, int) {}
    __device__ __forceinline__ void ket_end(int, int) {}
    __device__ __forceinline__ void operator()(int ia, int ib, int ic, int id, double v)
    {
        if (ia == ic && ib == id) acc[ia * NB + ib] += v;
    }
};

template <class Cls, int THREADS>
__global__ void __launch_bounds__(THREADS) schwarz_kernel(PairListDev pl, PrimPairsDev P, double* __restrict__ Q,
                                                          const double* __restrict__ boys_table)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pl.n) return;
    double* rs = r_slice<double>();
    DiagSink<Cls::LA, Cls::LB> sink;
#pragma unroll
    for (int k = 0; k < DiagSink<Cls::LA, Cls::LB>::NAB; ++k) sink.acc[k] = 0.0;
    const int o = pl.ppo[i], n = pl.npp[i];
    for (int x = 0; x < n; ++x)
    {
        const PrimPairData ab = load_pp(P, o + x);
        for (int y = 0; y < n; ++y)
        {
            const PrimPairData cd = load_pp(P, o + y);
            Cls::template quartet<double>(ab, cd, boys_table, rs, THREADS, sink);
        }
    }
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < DiagSink<Cls::LA, Cls::LB>::NAB; ++k) m = fmax(m, fabs(sink.acc[k]));
    Q[i] = sqrt(m);
}

// The same for the chunked classes when they have few pairs: work item t = c * n32 + i (n32 = the pair
// count rounded up to a multiple of 32) evaluates ket-component chunk c of pair i's diagonal quartet, whose
// diagonal elements are exactly the chunk's (c d) = (a b) components, and merges its maximum into Q[i]
// (zeroed by the launcher) with an atomic maximum on the bit pattern, which orders non-negative doubles.
template <class Cls, int THREADS>
__global__ void __launch_bounds__(THREADS) schwarz_split_kernel(PairListDev pl, PrimPairsDev P,
                                                                double* __restrict__ Q,
                                                                const double* __restrict__ boys_table)
{
    const long long n32 = ((long long)pl.n + 31) & ~31LL;
    const long long nitem = n32 * Cls::kNChunk;
    double* rs = r_slice<double>();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nitem;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int c = (int)(t / n32);
        const long long i = t - c * n32;
        if (i >= pl.n) continue;
        DiagSink<Cls::LA, Cls::LB> sink;
#pragma unroll
        for (int k = 0; k < DiagSink<Cls::LA, Cls::LB>::NAB; ++k) sink.acc[k] = 0.0;
        const int o = pl.ppo[i], n = pl.npp[i];
        for (int x = 0; x < n; ++x)
        {
            const PrimPairData ab = load_pp(P, o + x);
            for (int y = 0; y < n; ++y)
            {
                const PrimPairData cd = load_pp(P, o + y);
                Cls::template quartet_chunk<double>(c, ab, cd, boys_table, rs, THREADS, sink);
            }
        }
        double m = 0.0;
#pragma unroll
        for (int k = 0; k < DiagSink<Cls::LA, Cls::LB>::NAB; ++k) m = fmax(m, fabs(sink.acc[k]));
        atomicMax(reinterpret_cast<unsigned long long*>(Q + i), (unsigned long long)__double_as_longlong(sqrt(m)));
    }
}

// ------------------------------------------------------------------------------------------------
// Fused ERI + J/K digestion.  For a canonical quartet with weight w = s * (mu nu|la si),
// s = 1/2^{[a=b]+[c=d]+[ab=cd]}, the eight permutational images reduce to
//   J'[mu nu] += 2 w D[la si]      J'[la si] += 2 w D[mu nu]
//   K'[mu la] += w D[nu si]        K'[nu la] += w D[mu si]
//   K'[mu si] += w D[nu la]        K'[nu si] += w D[mu la]
// and J = J' + J'^T, K = K' + K'^T afterwards.  Partial sums are kept in registers along the
// component loops; what leaves the thread goes to the L2-resident J'/K' with red.global.add.f64.
// ------------------------------------------------------------------------------------------------
template <class RT, int LA, int LB, int LC, int LD, bool DET = false>
struct JKSink
{
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NAB = NA * NB;
    const double* __restrict__ D;
    double* __restrict__ J;
    double* __restrict__ K;
    int n, fa, fb, fc, fd;
    double s;
    long long det_lo = 0;   // DET: offset of the accumulator pairs' low words (JKWorkDev::det_lo)
    // DET: exact integer accumulator pairs (fixed_add); else FP64 atomics.  A template parameter, so that the
    // FP64 kernels carry no trace of the deterministic mode.
    __device__ __forceinline__ void acc(double* M, size_t k, double v)
    {
        if constexpr (DET) fixed_add(M, k, det_lo, v);
        else atomicAdd(M + k, v);
    }
    double jab[NAB];
    double kac[NA], kbc[NB], kad[NA], kbd[NB];
    double dls, jcd;
    double dbs[NB], das[NA], dbl[NB], dal[NA];
    int row_la = -1;   // ket row (c component) whose K'[., la] sums are still in registers

    // a new bra pair: J'[a b] partial sums start from zero
    __device__ __forceinline__ void set_bra(int fa_, int fb_)
    {
        fa = fa_;
        fb = fb_;
#pragma unroll
        for (int k = 0; k < NAB; ++k) jab[k] = 0.0;
#pragma unroll
        for (int k = 0; k < NA; ++k) kac[k] = 0.0;
#pragma unroll
        for (int k = 0; k < NB; ++k) kbc[k] = 0.0;
    }
    __device__ __forceinline__ void ket_begin(int ic, int id)
    {
        const int la = fc + ic, si = fd + id;
        row_la = la;
        dls = __ldg(D + (size_t)la * n + si);
        jcd = 0.0;
#pragma unroll
        for (int k = 0; k < NA; ++k)
        {
            das[k] = __ldg(D + (size_t)(fa + k) * n + si);
            dal[k] = __ldg(D + (size_t)(fa + k) * n + la);
            kad[k] = 0.0;
        }
#pragma unroll
        for (int k = 0; k < NB; ++k)
        {
            dbs[k] = __ldg(D + (size_t)(fb + k) * n + si);
            dbl[k] = __ldg(D + (size_t)(fb + k) * n + la);
            kbd[k] = 0.0;
        }
    }
    __device__ __forceinline__ void operator()(int ia, int ib, int, int, RT v)
    {
        const double w = s * (double)v;   // FP64 accumulation in either arithmetic type
        jab[ia * NB + ib] += w * dls;
        jcd += w * __ldg(D + (size_t)(fa + ia) * n + fb + ib);
        kac[ia] += w * dbs[ib];
        kbc[ib] += w * das[ia];
        kad[ia] += w * dbl[ib];
        kbd[ib] += w * dal[ia];
    }
    __device__ __forceinline__ void ket_end(int ic, int id)
    {
        const int la = fc + ic, si = fd + id;
        acc(J, (size_t)la * n + si, 2.0 * jcd);
#pragma unroll
        for (int k = 0; k < NA; ++k) acc(K, (size_t)(fa + k) * n + si, kad[k]);
#pragma unroll
        for (int k = 0; k < NB; ++k) acc(K, (size_t)(fb + k) * n + si, kbd[k]);
        if (id == ND - 1)
        {
#pragma unroll
            for (int k = 0; k < NA; ++k) { acc(K, (size_t)(fa + k) * n + la, kac[k]); kac[k] = 0.0; }
#pragma unroll
            for (int k = 0; k < NB; ++k) { acc(K, (size_t)(fb + k) * n + la, kbc[k]); kbc[k] = 0.0; }
            row_la = -1;
        }
    }
    // a chunk of ket components that ends inside a ket row leaves that row's K'[., la] sums in registers
    __device__ __forceinline__ void flush_k_row()
    {
        if (row_la < 0) return;
#pragma unroll
        for (int k = 0; k < NA; ++k) { acc(K, (size_t)(fa + k) * n + row_la, kac[k]); kac[k] = 0.0; }
#pragma unroll
        for (int k = 0; k < NB; ++k) { acc(K, (size_t)(fb + k) * n + row_la, kbc[k]); kbc[k] = 0.0; }
        row_la = -1;
    }
    // the end of one quartet: in the deterministic mode J'[a b] leaves the registers after every quartet, so
    // that each quartet's contribution is rounded alone and the integer sums do not depend on how many
    // quartets a lane runs (the launch shape); the FP64 mode keeps summing over the lane's run
    __device__ __forceinline__ void quartet_end()
    {
        if constexpr (DET)
        {
            flush_bra();
#pragma unroll
            for (int k = 0; k < NAB; ++k) jab[k] = 0.0;
        }
    }
    // the bra pair is done (or the lane's run ends): flush J'[a b]
    __device__ __forceinline__ void flush_bra()
    {
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
            {
                const double x = jab[ia * NB + ib];
                if (x != 0.0) acc(J, (size_t)(fa + ia) * n + fb + ib, 2.0 * x);
            }
    }
};

// true when quartet (bra pair i, ket pair j) is skipped: one of its shell pairs is outside the pair subset,
// its density-weighted bound is below the density threshold, or its bound lies outside this launch's
// precision band [w.lo, w.hi)
__device__ __forceinline__ bool jk_skip(const JKWorkDev& w, const PairListDev& bra, const PairListDev& ket, int i,
                                        int j, int sa, int sb, int sc, int sd)
{
    if (w.pmask && !(w.pmask[sa * w.nshell + sb] && w.pmask[sc * w.nshell + sd])) return true;
    const bool banded = w.lo > 0.0 || w.hi < 1e300;
    if (w.dmax)
    {
        const double* M = w.dmax;
        const int ns = w.nshell;
        double m = fmax(M[sa * ns + sb], M[sc * ns + sd]);
        m = fmax(m, fmax(M[sa * ns + sc], M[sa * ns + sd]));
        m = fmax(m, fmax(M[sb * ns + sc], M[sb * ns + sd]));
        const double bnd = bra.Q[i] * ket.Q[j] * m;
        return bnd < w.dthr || (banded && (bnd < w.lo || bnd >= w.hi));
    }
    if (banded)
    {
        const double bnd = bra.Q[i] * ket.Q[j];
        return bnd < w.lo || bnd >= w.hi;
    }
    return false;
}

// Each lane walks RUN quartets spaced one warp apart (g = base + lane + 32 k), so consecutive quartets of a
// lane usually share the bra pair: the bra pair is found by one binary search per run and then advanced,
// and the bra-side J' sums stay in registers until the bra pair changes.  RUN is chosen by the launcher
// from the class's quartet count (1 for small molecules, where parallelism matters more).
// RT is the arithmetic type of the ERI evaluation; a launch takes the quartets whose bound (Q_ab Q_cd, times
// the density maximum when density screening is on) lies in [w.lo, w.hi), so that an FP64 and an FP32
// launch split one build between them.
template <class Cls, int THREADS, class RT, bool DET = false>
__global__ void __launch_bounds__(THREADS) jk_kernel(JKWorkDev w, PairListDev bra, PairListDev ket, PrimPairsDev P,
                                                     const int* __restrict__ shell_f0, const double* __restrict__ D,
                                                     double* __restrict__ J, double* __restrict__ K, int n,
                                                     const double* __restrict__ boys_table, int RUN)
{
    RT* rs = r_slice<RT>();
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = w.gbeg + warp * 32 * RUN; base < w.gend; base += nwarp * 32 * RUN)
    {
        long long g = base + lane;
        if (g >= w.gend) continue;
        // bra pair i: offs[i] <= g < offs[i+1]
        int lo = 0, hi = bra.n;
        while (hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if (w.offs[mid] <= g) lo = mid;
            else hi = mid;
        }
        int i = lo;
        long long next = w.offs[i + 1];
        JKSink<RT, Cls::LA, Cls::LB, Cls::LC, Cls::LD, DET> sink;
        sink.D = D; sink.J = J; sink.K = K; sink.n = n;
        if constexpr (DET) sink.det_lo = w.det_lo;
        // several molecules: the bra pair's molecule selects the packed blocks and their dimension
        auto bind = [&](int ii) {
            if (bra.mol)
            {
                const int m = bra.mol[ii];
                const long long o = w.mols.off[m];
                sink.D = D + o;
                sink.J = J + o;
                sink.K = K + o;
                sink.n = w.mols.n[m];
            }
        };
        int sa = bra.sa[i], sb = bra.sb[i];
        bind(i);
        sink.set_bra(shell_f0[sa], shell_f0[sb]);
        for (int r = 0; r < RUN && g < w.gend; ++r, g += 32)
        {
            if (g >= next)
            {
                sink.flush_bra();
                do
                {
                    ++i;
                    next = w.offs[i + 1];
                } while (g >= next);
                sa = bra.sa[i];
                sb = bra.sb[i];
                bind(i);
                sink.set_bra(shell_f0[sa], shell_f0[sb]);
            }
            if (w.mol_active && bra.mol && !w.mol_active[bra.mol[i]]) continue;
            const int j = (w.kbase ? w.kbase[i] : 0) + (int)(g - w.offs[i]);
            const int sc = ket.sa[j], sd = ket.sb[j];
            if (jk_skip(w, bra, ket, i, j, sa, sb, sc, sd)) continue;
            sink.fc = shell_f0[sc];
            sink.fd = shell_f0[sd];
            sink.s = (sa == sb ? 0.5 : 1.0) * (sc == sd ? 0.5 : 1.0) * ((w.same_class && i == j) ? 0.5 : 1.0);
            const int oi = bra.ppo[i], ni = bra.npp[i], oj = ket.ppo[j], nj = ket.npp[j];
            for (int x = 0; x < ni; ++x)
            {
                const PrimPairData ab = load_pp(P, oi + x);
                for (int y = 0; y < nj; ++y)
                {
                    const PrimPairData cd = load_pp(P, oj + y);
                    Cls::template quartet<RT>(ab, cd, boys_table, rs, THREADS, sink);
                }
            }
            sink.quartet_end();
        }
        sink.flush_bra();
    }
}

// ------------------------------------------------------------------------------------------------
// The warp-shared form of the direct J/K build.  Each half of a warp takes up to 16 bra pairs (a b_l) that
// share their first shell a -- lane l holds (a b_l) -- against one ket pair (c d) at a time.  Of the six
// digestion targets of a quartet, three are then the same for every lane of a half: J'(c d), K'(a c) and
// K'(a d).  Their lane partial sums are added across the half by shuffles and written by one lane each, so
// an L2 atomic per lane becomes one per half warp; only K'(b c) and K'(b d) stay per lane, and J'(a b)
// stays in registers over the whole run of kets.  The ket's pair data and its density rows D(a, .) are the
// same for every lane of a half (one broadcast load each).  Lanes whose quartet is absent (past their bra
// pair's screened ket prefix, skipped by jk_skip, past the end of a short set, or past a shorter primitive
// loop) evaluate a valid quartet with weight 0, so that every lane reaches the shuffles.  Half-warp sets
// rather than whole-warp ones keep more lanes busy: a shell's partner list rarely fills a multiple of 32,
// and 16 neighbours in Q order have closer ket prefixes.  This replaces the same arithmetic as JKSink
// (qchem's MakeDirect / MakeExchange, Molecule/IrrepBasisSet.C:138-183) with fewer memory operations.
// ------------------------------------------------------------------------------------------------

// Sum P values (P a power of two, <= 16) over the 16 lanes of each half of a warp (lanes 0-15 and 16-31
// are separate sets): in log2 P exchange steps each lane keeps half of its values and adds its partner's
// copy of them, then the rest is a plain butterfly, every shuffle within the half.  On return every lane
// holds its half's total of value ((lane & 15) >> (4 - log2 P)); the lanes with lane % (16 / P) == 0 are one
// writer per value and half.
template <int P>
__device__ __forceinline__ double half_warp_transpose_sum(double (&v)[P], int lane)
{
#pragma unroll
    for (int m = P, o = 8; m > 1; m >>= 1, o >>= 1)
    {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < m / 2; ++k)
        {
            const double send = up ? v[k] : v[k + m / 2];
            const double keep = up ? v[k + m / 2] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    double x = v[0];
#pragma unroll
    for (int o = 8 / P; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

constexpr int pow2_at_least(int v) { return v <= 1 ? 1 : 2 * pow2_at_least((v + 1) / 2); }

template <int LA, int LB, int LC, int LD>
struct WarpJKSink
{
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NAB = NA * NB;
    const double* __restrict__ D;
    double* __restrict__ J;
    double* __restrict__ K;
    int n, fa, fb, fc, fd, lane;
    double s;   // symmetry weight of this lane's quartet, 0 for an absent quartet
    double jab[NAB];
    double dls, jcd;
    double das[NA], dal[NA], dbs[NB], dbl[NB];
    double kac[NA], kad[NA], kbc[NB], kbd[NB];

    __device__ __forceinline__ void set_bra(int fa_, int fb_)
    {
        fa = fa_;
        fb = fb_;
#pragma unroll
        for (int k = 0; k < NAB; ++k) jab[k] = 0.0;
    }
    __device__ __forceinline__ void ket_begin(int ic, int id)
    {
        const int la = fc + ic, si = fd + id;
        dls = __ldg(D + (size_t)la * n + si);
        jcd = 0.0;
#pragma unroll
        for (int k = 0; k < NA; ++k)
        {
            das[k] = __ldg(D + (size_t)(fa + k) * n + si);
            dal[k] = __ldg(D + (size_t)(fa + k) * n + la);
            kad[k] = 0.0;
            if (id == 0) kac[k] = 0.0;
        }
#pragma unroll
        for (int k = 0; k < NB; ++k)
        {
            dbs[k] = __ldg(D + (size_t)(fb + k) * n + si);
            dbl[k] = __ldg(D + (size_t)(fb + k) * n + la);
            kbd[k] = 0.0;
            if (id == 0) kbc[k] = 0.0;
        }
    }
    __device__ __forceinline__ void operator()(int ia, int ib, int, int, double v)
    {
        const double w = s * v;
        jab[ia * NB + ib] += w * dls;
        jcd += w * __ldg(D + (size_t)(fa + ia) * n + fb + ib);
        kac[ia] += w * dbs[ib];
        kbc[ib] += w * das[ia];
        kad[ia] += w * dbl[ib];
        kbd[ib] += w * dal[ia];
    }
    // the shared targets of this ket component (and of its ket row at the row's end) across the warp
    template <int V>
    __device__ __forceinline__ void flush_shared(int la, int si)
    {
        constexpr int P = pow2_at_least(V);
        static_assert(P <= 16, "at most 16 shared values per half warp");
        constexpr int SHIFT = (P == 1 ? 4 : P == 2 ? 3 : P == 4 ? 2 : P == 8 ? 1 : 0);
        double v[P];
        v[0] = jcd;
#pragma unroll
        for (int k = 0; k < NA; ++k) v[1 + k] = kad[k];
        if constexpr (V > 1 + NA)
        {
#pragma unroll
            for (int k = 0; k < NA; ++k) v[1 + NA + k] = kac[k];
        }
#pragma unroll
        for (int k = V; k < P; ++k) v[k] = 0.0;
        const double x = half_warp_transpose_sum<P>(v, lane);
        const int idx = (lane & 15) >> SHIFT;
        if ((lane & ((1 << SHIFT) - 1)) != 0 || idx >= V || x == 0.0) return;
        if (idx == 0) atomicAdd(J + (size_t)la * n + si, 2.0 * x);
        else if (idx <= NA) atomicAdd(K + (size_t)(fa + idx - 1) * n + si, x);
        else atomicAdd(K + (size_t)(fa + idx - 1 - NA) * n + la, x);
    }
    __device__ __forceinline__ void ket_end(int ic, int id)
    {
        const int la = fc + ic, si = fd + id;
#pragma unroll
        for (int k = 0; k < NB; ++k)
            if (kbd[k] != 0.0) atomicAdd(K + (size_t)(fb + k) * n + si, kbd[k]);
        if (id == ND - 1)
        {
#pragma unroll
            for (int k = 0; k < NB; ++k)
                if (kbc[k] != 0.0) atomicAdd(K + (size_t)(fb + k) * n + la, kbc[k]);
            flush_shared<1 + 2 * NA>(la, si);
        }
        else
            flush_shared<1 + NA>(la, si);
    }
    __device__ __forceinline__ void flush_bra()
    {
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
            {
                const double x = jab[ia * NB + ib];
                if (x != 0.0) atomicAdd(J + (size_t)(fa + ia) * n + fb + ib, 2.0 * x);
            }
    }
};

// Work item t is two half-warp sets: items[2t] for lanes 0-15 and items[2t + 1] for lanes 16-31, each
// {first entry of its set in gbra, its lane count (<= 16), first ket, end ket}.  A set is gbra[x .. x + y),
// bra pairs sharing their first shell; its kets are positions [z, w) of each lane's ket list (its molecule's
// part of the ket class, from kbase), each lane stopping at its own screened prefix.  The two sets of an
// item have the same first ket, so the warp walks one ket loop for both; the primitive loops run to the
// warp's longest, with weight 0 beyond a lane's own, so that every lane reaches every shuffle.
template <class Cls, int THREADS>
__global__ void __launch_bounds__(THREADS) jk_warp_kernel(JKWorkDev w, PairListDev bra, PairListDev ket,
                                                          PrimPairsDev P, const int* __restrict__ shell_f0,
                                                          const double* __restrict__ D, double* __restrict__ J,
                                                          double* __restrict__ K, int n,
                                                          const double* __restrict__ boys_table,
                                                          const int* __restrict__ gbra, const int4* __restrict__ items,
                                                          long long nitems)
{
    double* rs = r_slice<double>();
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = warp; t < nitems; t += nwarp)
    {
        const int4 it = items[2 * t + (lane >> 4)];
        const int4 other = items[2 * t + 1 - (lane >> 4)];
        const bool real = (lane & 15) < it.y;
        // an empty half (an odd set count) borrows the other half's first bra pair, with weight 0
        const int i = real ? gbra[it.x + (lane & 15)] : gbra[it.y > 0 ? it.x : other.x];
        const int prefix = real ? (int)(w.offs[i + 1] - w.offs[i]) : 0;
        const int jb = w.kbase ? w.kbase[i] : 0;   // the same within a half: one molecule per set
        const int sa = bra.sa[i], sb = bra.sb[i];
        WarpJKSink<Cls::LA, Cls::LB, Cls::LC, Cls::LD> sink;
        sink.D = D;
        sink.J = J;
        sink.K = K;
        sink.n = n;
        sink.lane = lane;
        bool on = true;
        if (bra.mol)
        {
            const int m = bra.mol[i];
            const long long o = w.mols.off[m];
            sink.D = D + o;
            sink.J = J + o;
            sink.K = K + o;
            sink.n = w.mols.n[m];
            on = !(w.mol_active && !w.mol_active[m]);
        }
        sink.set_bra(shell_f0[sa], shell_f0[sb]);
        const int oi = bra.ppo[i], ni = bra.npp[i];
        const int nimax = __reduce_max_sync(0xffffffffu, ni);
        const int jend = it.w > other.w ? it.w : other.w;   // both halves start at it.z == other.z
        for (int jj = it.z; jj < jend; ++jj)
        {
            // a half past its own end repeats its last ket with weight 0
            const int j = jb + (jj < it.w ? jj : (it.w > it.z ? it.w - 1 : it.z));
            const int sc = ket.sa[j], sd = ket.sb[j];
            const bool act = real && on && jj < it.w && jj < prefix && !jk_skip(w, bra, ket, i, j, sa, sb, sc, sd);
            if (!__any_sync(0xffffffffu, act)) continue;
            sink.fc = shell_f0[sc];
            sink.fd = shell_f0[sd];
            const double s =
                (sa == sb ? 0.5 : 1.0) * (sc == sd ? 0.5 : 1.0) * ((w.same_class && i == j) ? 0.5 : 1.0);
            const int oj = ket.ppo[j], nj = ket.npp[j];
            const int njmax = __reduce_max_sync(0xffffffffu, nj);
            for (int x = 0; x < nimax; ++x)
            {
                const PrimPairData ab = load_pp(P, oi + (x < ni ? x : ni - 1));
                for (int y = 0; y < njmax; ++y)
                {
                    const PrimPairData cd = load_pp(P, oj + (y < nj ? y : nj - 1));
                    sink.s = (act && x < ni && y < nj) ? s : 0.0;
                    Cls::template quartet<double>(ab, cd, boys_table, rs, THREADS, sink);
                }
            }
        }
        sink.flush_bra();
    }
}

// Launches of the chunked classes with too few quartets to fill the GPU: work item t = c * span32 + q
// (span32 = the quartet count rounded up to a multiple of 32) runs ket-component chunk c of quartet
// w.gbeg + q.  A warp's lanes share the chunk, and the chunks of one quartet run on different warps at the
// same time, so the launch takes about one chunk's time instead of one whole quartet's.  Each item
// rebuilds Boys and R and digests its chunk's outputs like jk_kernel (the digestion is linear).
template <class Cls, int THREADS, class RT, bool DET = false>
__global__ void __launch_bounds__(THREADS) jk_split_kernel(JKWorkDev w, PairListDev bra, PairListDev ket,
                                                           PrimPairsDev P, const int* __restrict__ shell_f0,
                                                           const double* __restrict__ D, double* __restrict__ J,
                                                           double* __restrict__ K, int n,
                                                           const double* __restrict__ boys_table)
{
    RT* rs = r_slice<RT>();
    const long long span = w.gend - w.gbeg, span32 = (span + 31) & ~31LL;
    const long long nitem = span32 * Cls::kNChunk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nitem;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int c = (int)(t / span32);
        const long long q = t - c * span32;
        if (q >= span) continue;
        const long long g = w.gbeg + q;
        int lo = 0, hi = bra.n;
        while (hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if (w.offs[mid] <= g) lo = mid;
            else hi = mid;
        }
        const int i = lo;
        if (w.mol_active && bra.mol && !w.mol_active[bra.mol[i]]) continue;
        const int j = (w.kbase ? w.kbase[i] : 0) + (int)(g - w.offs[i]);
        const int sa = bra.sa[i], sb = bra.sb[i], sc = ket.sa[j], sd = ket.sb[j];
        if (jk_skip(w, bra, ket, i, j, sa, sb, sc, sd)) continue;
        JKSink<RT, Cls::LA, Cls::LB, Cls::LC, Cls::LD, DET> sink;
        sink.D = D; sink.J = J; sink.K = K; sink.n = n;
        if constexpr (DET) sink.det_lo = w.det_lo;
        if (bra.mol)
        {
            const int m = bra.mol[i];
            const long long o = w.mols.off[m];
            sink.D = D + o;
            sink.J = J + o;
            sink.K = K + o;
            sink.n = w.mols.n[m];
        }
        sink.set_bra(shell_f0[sa], shell_f0[sb]);
        sink.fc = shell_f0[sc];
        sink.fd = shell_f0[sd];
        sink.s = (sa == sb ? 0.5 : 1.0) * (sc == sd ? 0.5 : 1.0) * ((w.same_class && i == j) ? 0.5 : 1.0);
        const int oi = bra.ppo[i], ni = bra.npp[i], oj = ket.ppo[j], nj = ket.npp[j];
        for (int x = 0; x < ni; ++x)
        {
            const PrimPairData ab = load_pp(P, oi + x);
            for (int y = 0; y < nj; ++y)
            {
                const PrimPairData cd = load_pp(P, oj + y);
                Cls::template quartet_chunk<RT>(c, ab, cd, boys_table, rs, THREADS, sink);
                // the next primitive quartet restarts the chunk, possibly inside a different ket row
                sink.flush_k_row();
            }
        }
        sink.flush_bra();
    }
}

}   // namespace qcg
