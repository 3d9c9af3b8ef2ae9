// eri_team.cuh -- warp-specialised ERI-batch kernel for the high-L classes (team form).
//
// A CTA takes 32 contracted quartets at a time (a "group": 32 consecutive entries of the batch's visiting
// order, which groups equal contraction patterns), one per lane, and works through them in three phases.
//
//  1. Stage tables.  For every primitive quartet x of the group (bra primitive pair outer, ket inner) and
//     every lane, a "stage" holds R^0_{tuv} scaled by the prefactor lambda and the single-centre Hermite
//     tables E^{i0}_t of the ket pair (and, after the last ket primitive of a bra primitive pair, of the bra
//     pair) -- generated code, team_produce_<k>.  All warps compute stages, warp w taking x = w, w + nwarps,
//     ..., and write them once to the CTA's slots of the R cache in global memory (entry-major, lane-minor).
//     Two variants were measured slower on a B200 and dropped: rebuilding the Hermite tables in the
//     consumers to halve the stage (1.4x slower on (dd|dd): the contraction is bound by instruction issue),
//     and walking the group one bra primitive pair at a time so that the cache stays in L2 (1.3x slower: a
//     barrier, a pipeline restart and an accumulator save per window cost more than the HBM traffic saved).
//  2. Contraction.  Warp w owns one component f of the ket range of the horizontal-recurrence form (f over
//     L = LC..LC+LD on centre C) per pass; each component has its own straight-line ket code, and the warp
//     count is sized so that the code of the components in flight fits the SM's instruction cache.  It keeps in registers Y_f -- the ket step summed over the ket
//     primitives of the current bra primitive pair -- and acc_f = [e0|f] for every e, adding the bra step
//     of Y_f to acc_f after the bra pair's last ket primitive (team_ket_<k>, team_bra_<k>).  The stages
//     stream from the R cache into shared memory, three deep, by bulk copies (cp.async.bulk, the Tensor
//     Memory Accelerator's untiled form) that one thread issues on an mbarrier; one barrier per primitive
//     quartet.  With more ket components than warps the group is walked in passes, each pass reading the
//     stages again (from L2 or HBM) instead of recomputing them.
//  3. Recurrences.  acc_f goes to the CTA's scratch as [e0|f0] (lane-minor, so every access of a warp is
//     one coalesced line); the ket recurrence per e row gives [e0|cd] there, and the bra recurrence per
//     (c d) column writes (ab|cd) into the quartet's output block (generated team_hrr_ket_<k>,
//     team_hrr_bra_<k>).  No atomics: every output element is written once by one thread.
//
// This is the arithmetic of qchem's PrimGaussian::Repulsion4C (PG_Cart_MnD/Imp/GaussianRF.C:446-483) and
// its contraction (GaussianRF.C:726-752), with the bra and ket transfers done once per contracted quartet
// (horizontal recurrence) and the bra Hermite contraction once per bra primitive pair.
#pragma once
#include <cstdint>

#include "eri_team_iface.h"
#include "md_core.cuh"
#include "team_sync.cuh"

namespace qcg {

extern __shared__ __align__(128) double qcg_team_smem[];

template <class Cls>
__global__ void __launch_bounds__(Cls::kNW * 32, 1)
    eri_batch_team_kernel(BasisDev bs, const int4* __restrict__ quartets, const int* __restrict__ order, long long nq,
                          double* __restrict__ out, const double* __restrict__ boys_table, TeamScratchDev scr)
{
    constexpr int NW = Cls::kNW;                   // warps; warp w owns ket component pass * NW + w
    constexpr int NF = Cls::kNF, NE = Cls::kNE, NH = Cls::kNH;
    constexpr int NPASS = (NF + NW - 1) / NW;
    constexpr int STAGE = Cls::kStage * 32;        // doubles per stage (entry-major, lane-minor)
    constexpr uint32_t STAGE_BYTES = STAGE * sizeof(double);
    constexpr int NCD = ncart(Cls::LC) * ncart(Cls::LD);
    constexpr long long BLK = (long long)ncart(Cls::LA) * ncart(Cls::LB) * NCD;
    static_assert(NE <= ncart(Cls::LA) * ncart(Cls::LB) && NF <= NCD, "[e0|f0] fits the output block");
    __shared__ uint64_t full[3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool leader = threadIdx.x == 0;
    if (leader)
    {
        for (int s = 0; s < 3; ++s) team::mbar_init(&full[s]);
        team::mbar_init_fence();
    }
    __syncthreads();
    double* const rc = scr.rcache + (long long)blockIdx.x * scr.kmax * STAGE;   // this CTA's stage slots
    double* const hA = scr.hrr + (long long)blockIdx.x * (NE * NF + NE * NCD) * 32;
    double* const hB = hA + NE * NF * 32;
    unsigned long long G = 0;   // steps streamed so far: step G uses stage G % 3, phase (G / 3) & 1
    const long long ngroups = (nq + 31) >> 5;
    for (long long g = blockIdx.x; g < ngroups; g += gridDim.x)
    {
        // every warp reads the same 32 quartets: lane l of every warp holds quartet l of the group
        const long long gi = g * 32 + lane;
        const bool valid = gi < nq;
        const long long q = valid ? (order ? (long long)order[gi] : gi) : 0;
        const int4 s = quartets[q];
        int ni = 0, nj = 0, nk = 0, nl = 0;
        if (valid)
        {
            ni = bs.nprim[s.x];
            nj = bs.nprim[s.y];
            nk = bs.nprim[s.z];
            nl = bs.nprim[s.w];
        }
        const int Kcd = nk * nl, K = ni * nj * Kcd;
        const int Kg = __reduce_max_sync(0xffffffffu, K);   // the group's longest primitive loop (CTA-uniform)
        if (Kg > scr.kmax)
        {
            if (leader) atomicOr(scr.err, 2);
            continue;
        }
        // 1. stage tables of every primitive quartet, written once to the R cache
        for (int x = warp; x < Kg; x += NW)
            if (x < K)
            {
                const int ij = x / Kcd, kl = x - ij * Kcd;
                const PrimPairData ab = shell_prim_pair(bs, s.x, ij / nj, s.y, ij % nj);
                const PrimPairData cd = shell_prim_pair(bs, s.z, kl / nl, s.w, kl % nl);
                Cls::produce(rc + (long long)x * STAGE + lane, ab, cd, boys_table, kl == Kcd - 1);
            }
        team::fence_async_global();
        __syncthreads();
        // 2. contraction, the stages streamed back through shared memory three deep
        for (int pass = 0; pass < NPASS; ++pass)
        {
            const int jf = pass * NW + warp;
            auto issue = [&](int x) {
                const unsigned long long gs = G + x;
                team::bulk_load(qcg_team_smem + (gs % 3) * STAGE, rc + (long long)x * STAGE, STAGE_BYTES,
                                &full[gs % 3]);
            };
            if (leader)
            {
                issue(0);
                if (Kg > 1) issue(1);
            }
            double Y[NH], acc[NE];
#pragma unroll
            for (int h = 0; h < NH; ++h) Y[h] = 0.0;
#pragma unroll
            for (int e = 0; e < NE; ++e) acc[e] = 0.0;
            int kl = 0;
            for (int i = 0; i < Kg; ++i)
            {
                const unsigned long long gs = G + i;
                bool late = false;
                if (leader) late = !team::mbar_wait(&full[gs % 3], (uint32_t)((gs / 3) & 1));
                // stage i is in shared memory; every warp has left step i - 1
                if (__syncthreads_or(late))
                {
                    // a copy did not arrive: let the ones in flight land, record it and end the CTA
                    if (leader)
                    {
                        team::drain(full, G, i, Kg);
                        atomicOr(scr.err, 1);
                    }
                    return;
                }
                if (leader && i + 2 < Kg) issue(i + 2);   // into the stage step i - 1 used
                if (jf < NF && i < K)
                {
                    const double* st = qcg_team_smem + (gs % 3) * STAGE + lane;
                    Cls::ket(jf, st, Y);
                    if (kl == Kcd - 1)
                    {
                        Cls::bra(st, Y, acc);
#pragma unroll
                        for (int h = 0; h < NH; ++h) Y[h] = 0.0;
                        kl = 0;
                    }
                    else
                        ++kl;
                }
            }
            G += Kg;
            if (jf < NF)
            {
#pragma unroll
                for (int e = 0; e < NE; ++e) hA[(e * NF + jf) * 32 + lane] = acc[e];
            }
            __syncthreads();   // the pass's stages are no longer read; its [e0|f] columns are written
        }
        // 3. recurrences: ket per e row into [e0|cd], bra per (c d) column into the output block
        const double* A = bs.cen + 3 * s.x;
        const double* B = bs.cen + 3 * s.y;
        const double* C = bs.cen + 3 * s.z;
        const double* D = bs.cen + 3 * s.w;
        if (valid)
        {
            const double CDx = C[0] - D[0], CDy = C[1] - D[1], CDz = C[2] - D[2];
            for (int e = warp; e < NE; e += NW)
                Cls::hrr_ket(hA + e * NF * 32 + lane, hB + e * NCD * 32 + lane, CDx, CDy, CDz);
        }
        __syncthreads();
        if (valid)
        {
            const double ABx = A[0] - B[0], ABy = A[1] - B[1], ABz = A[2] - B[2];
            double* const o = out + q * BLK;
            for (int cd = warp; cd < NCD; cd += NW) Cls::hrr_bra(hB + cd * 32 + lane, o + cd, NCD, ABx, ABy, ABz);
        }
        __syncthreads();   // the scratch and the R cache are free for the next group
    }
}

// ------------------------------------------------------------------------------------------------
// The team form of the direct J/K build.  The same three phases on 32 quartets of a class's screened work
// list at a time (lane l: quartet gbeg + 32 g + l, its bra pair found by binary search, its kets from the
// Q-sorted list), the stages built from the primitive-pair table; the bra recurrence writes (ab|cd) into a
// third lane-minor block of the CTA's scratch, and a fourth phase digests it into J' and K' with the
// thread-per-quartet kernel's sink (JKSink: the eight permutational images, symmetry weights, registers for
// the partial sums, atomics or the deterministic integer pairs), warp w taking ket components w, w + nwarps,
// ....  This replaces qchem's MakeDirect/MakeExchange + ERI4::MatMul (Molecule/IrrepBasisSet.C:138-183,
// Internal/Imp/ERI4.C:10-17) without storing the integrals.
// ------------------------------------------------------------------------------------------------
template <class Cls, bool DET>
__global__ void __launch_bounds__(Cls::kNW * 32, 1)
    jk_team_kernel(JKWorkDev w, PairListDev bra, PairListDev ket, PrimPairsDev P, const int* __restrict__ shell_f0,
                   const double* __restrict__ D, double* __restrict__ J, double* __restrict__ K, int n,
                   const double* __restrict__ boys_table, TeamScratchDev scr)
{
    constexpr int NW = Cls::kNW;
    constexpr int NF = Cls::kNF, NE = Cls::kNE, NH = Cls::kNH;
    constexpr int NPASS = (NF + NW - 1) / NW;
    constexpr int STAGE = Cls::kStage * 32;
    constexpr uint32_t STAGE_BYTES = STAGE * sizeof(double);
    constexpr int NB = ncart(Cls::LB), ND = ncart(Cls::LD);
    constexpr int NAB = ncart(Cls::LA) * NB, NCD = ncart(Cls::LC) * ND;
    static_assert(NE <= NAB && NF <= NCD, "[e0|f0] fits the blocks");
    __shared__ uint64_t full[3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool leader = threadIdx.x == 0;
    if (leader)
    {
        for (int s = 0; s < 3; ++s) team::mbar_init(&full[s]);
        team::mbar_init_fence();
    }
    __syncthreads();
    double* const rc = scr.rcache + (long long)blockIdx.x * scr.kmax * STAGE;
    double* const hA = scr.hrr + (long long)blockIdx.x * (NE * NF + NE * NCD + NAB * NCD) * 32;
    double* const hB = hA + NE * NF * 32;
    double* const hC = hB + NE * NCD * 32;
    unsigned long long G = 0;
    const long long ngroups = (w.gend - w.gbeg + 31) >> 5;
    for (long long g = blockIdx.x; g < ngroups; g += gridDim.x)
    {
        const long long gq = w.gbeg + g * 32 + lane;
        bool valid = gq < w.gend;
        int i = 0, j = 0, sa = 0, sb = 0, sc = 0, sd = 0;
        if (valid)
        {
            int lo = 0, hi = bra.n;   // bra pair i: offs[i] <= gq < offs[i+1]
            while (hi - lo > 1)
            {
                const int mid = (lo + hi) >> 1;
                if (w.offs[mid] <= gq) lo = mid;
                else hi = mid;
            }
            i = lo;
            j = (w.kbase ? w.kbase[i] : 0) + (int)(gq - w.offs[i]);
            sa = bra.sa[i];
            sb = bra.sb[i];
            sc = ket.sa[j];
            sd = ket.sb[j];
            if (w.mol_active && bra.mol && !w.mol_active[bra.mol[i]]) valid = false;
            else if (jk_skip(w, bra, ket, i, j, sa, sb, sc, sd)) valid = false;
        }
        const int Kab = valid ? bra.npp[i] : 0, Kcd = valid ? ket.npp[j] : 0, Kq = Kab * Kcd;
        const int Kg = __reduce_max_sync(0xffffffffu, Kq);   // CTA-uniform: every warp sees the same lanes
        if (Kg == 0) continue;                               // every quartet of the group skipped
        if (Kg > scr.kmax)
        {
            if (leader) atomicOr(scr.err, 2);
            continue;
        }
        // 1. stage tables, from the primitive-pair table
        for (int x = warp; x < Kg; x += NW)
            if (x < Kq)
            {
                const int ij = x / Kcd, kl = x - ij * Kcd;
                const PrimPairData ab = load_pp(P, bra.ppo[i] + ij);
                const PrimPairData cd = load_pp(P, ket.ppo[j] + kl);
                Cls::produce(rc + (long long)x * STAGE + lane, ab, cd, boys_table, kl == Kcd - 1);
            }
        team::fence_async_global();
        __syncthreads();
        // 2. contraction (as in eri_batch_team_kernel)
        for (int pass = 0; pass < NPASS; ++pass)
        {
            const int jf = pass * NW + warp;
            auto issue = [&](int x) {
                const unsigned long long gs = G + x;
                team::bulk_load(qcg_team_smem + (gs % 3) * STAGE, rc + (long long)x * STAGE, STAGE_BYTES,
                                &full[gs % 3]);
            };
            if (leader)
            {
                issue(0);
                if (Kg > 1) issue(1);
            }
            double Y[NH], acc[NE];
#pragma unroll
            for (int h = 0; h < NH; ++h) Y[h] = 0.0;
#pragma unroll
            for (int e = 0; e < NE; ++e) acc[e] = 0.0;
            int kl = 0;
            for (int x = 0; x < Kg; ++x)
            {
                const unsigned long long gs = G + x;
                bool late = false;
                if (leader) late = !team::mbar_wait(&full[gs % 3], (uint32_t)((gs / 3) & 1));
                if (__syncthreads_or(late))
                {
                    if (leader)
                    {
                        team::drain(full, G, x, Kg);
                        atomicOr(scr.err, 1);
                    }
                    return;
                }
                if (leader && x + 2 < Kg) issue(x + 2);
                if (jf < NF && x < Kq)
                {
                    const double* st = qcg_team_smem + (gs % 3) * STAGE + lane;
                    Cls::ket(jf, st, Y);
                    if (kl == Kcd - 1)
                    {
                        Cls::bra(st, Y, acc);
#pragma unroll
                        for (int h = 0; h < NH; ++h) Y[h] = 0.0;
                        kl = 0;
                    }
                    else
                        ++kl;
                }
            }
            G += Kg;
            if (jf < NF)
            {
#pragma unroll
                for (int e = 0; e < NE; ++e) hA[(e * NF + jf) * 32 + lane] = acc[e];
            }
            __syncthreads();
        }
        // 3. recurrences into the scratch: [e0|cd] in hB, (ab|cd) in hC (lane-minor)
        // C - D = (P - D) - (P - C) and A - B = (P - B) - (P - A), from the shell pairs' first primitive pairs
        if (valid)
        {
            const PrimPairData cd0 = load_pp(P, ket.ppo[j]);
            const double CDx = cd0.PBx - cd0.PAx, CDy = cd0.PBy - cd0.PAy, CDz = cd0.PBz - cd0.PAz;
            for (int e = warp; e < NE; e += NW)
                Cls::hrr_ket(hA + e * NF * 32 + lane, hB + e * NCD * 32 + lane, CDx, CDy, CDz);
        }
        __syncthreads();
        if (valid)
        {
            const PrimPairData ab0 = load_pp(P, bra.ppo[i]);
            const double ABx = ab0.PBx - ab0.PAx, ABy = ab0.PBy - ab0.PAy, ABz = ab0.PBz - ab0.PAz;
            for (int cd = warp; cd < NCD; cd += NW)
                Cls::hrr_bra(hB + cd * 32 + lane, hC + cd * 32 + lane, NCD * 32, ABx, ABy, ABz);
        }
        __syncthreads();
        // 4. digestion of this lane's quartet, ket components cd = warp, warp + NW, ...
        if (valid)
        {
            JKSink<double, Cls::LA, Cls::LB, Cls::LC, Cls::LD, DET> sink;
            sink.D = D;
            sink.J = J;
            sink.K = K;
            sink.n = n;
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
            for (int cd = warp; cd < NCD; cd += NW)
            {
                const int ic = cd / ND, id = cd - ic * ND;
                sink.ket_begin(ic, id);
#pragma unroll
                for (int ab = 0; ab < NAB; ++ab) sink(ab / NB, ab % NB, ic, id, hC[(ab * NCD + cd) * 32 + lane]);
                sink.ket_end(ic, id);
                sink.flush_k_row();
            }
            sink.flush_bra();
        }
        __syncthreads();   // the scratch and the R cache are free for the next group
    }
}

}   // namespace qcg
