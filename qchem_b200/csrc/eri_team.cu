// eri_team.cu -- the team form of the FP64 ERI batches (eri_team.cuh) for ONE quartet class; compiled with
// -DQCG_CLASS=k for every class, defining launch_eri_team_k and team_shape_k.  The generated code comes from
// gen/md_team_<k>.cuh (stage tables, ket and bra steps, recurrences).
#include <atomic>

#include "eri_kernels.cuh"
#include "eri_team.cuh"
#include "smem_attr.h"

#ifndef QCG_CLASS
#error "compile with -DQCG_CLASS=<0..20>"
#endif

#define QCG_STR2(x) #x
#define QCG_STR(x) QCG_STR2(x)
#define QCG_CAT2(a, b) a##b
#define QCG_CAT(a, b) QCG_CAT2(a, b)
#include QCG_STR(gen/QCG_CAT(md_team_, QCG_CLASS).cuh)

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

// Warps per CTA, every warp a consumer of its own ket component per pass.  At most 8: the SM's registers are
// split among its four schedulers, and 8 warps (two per scheduler) leave each thread up to 255 registers,
// which the (dd|dd) steps need without spilling (a ninth warp caps every thread at 168).  Each component
// has its own straight-line ket code, and the code of the components in flight must fit the instruction
// cache.  Measured on a B200: on (dd|dd) 8 warps on 8 components ran at half the speed of 4 (and 3.4x slower
// than 8 warps sharing one component's code), 2 warps were slower than 4, and 4 warps also beat 8 on (dd|dp),
// (dd|pp) and (dp|dp), whose largest components have 220-570 instructions.  So: 8 warps where the largest
// component has at most kSmallKet instructions, else 4.
constexpr int kSmallKet = 150;

constexpr int team_warps(int nf, int ket_instr)
{
    const int maxw = ket_instr <= kSmallKet ? 8 : 4;
    const int npass = (nf + maxw - 1) / maxw;
    return (nf + npass - 1) / npass;
}

struct Cls
{
    static constexpr int LA = kPairLA[kX], LB = kPairLB[kX], LC = kPairLA[kY], LD = kPairLB[kY];
    static constexpr int kNF = gen::QCG_CAT(kTeamNF, QCG_CLASS), kNE = gen::QCG_CAT(kTeamNE, QCG_CLASS);
    static constexpr int kNH = gen::QCG_CAT(kTeamNH, QCG_CLASS), kStage = gen::QCG_CAT(kTeamStage, QCG_CLASS);
#ifdef QCG_TEAM_NW
    static constexpr int kNW = QCG_TEAM_NW;
#else
    static constexpr int kNW = team_warps(kNF, gen::QCG_CAT(kTeamKetInstr, QCG_CLASS));
#endif
    static __device__ __forceinline__ void produce(double* st, const PrimPairData& ab, const PrimPairData& cd,
                                                   const double* __restrict__ bt, bool bra_e)
    {
        gen::QCG_CAT(team_produce_, QCG_CLASS)<double>(st, ab, cd, bt, bra_e);
    }
    static __device__ __forceinline__ void ket(int jf, const double* st, double (&Y)[kNH])
    {
        gen::QCG_CAT(team_ket_, QCG_CLASS)<double>(jf, st, Y);
    }
    static __device__ __forceinline__ void bra(const double* st, const double (&Y)[kNH], double (&acc)[kNE])
    {
        gen::QCG_CAT(team_bra_, QCG_CLASS)<double>(st, Y, acc);
    }
    static __device__ __forceinline__ void hrr_ket(const double* p, double* y, double CDx, double CDy, double CDz)
    {
        gen::QCG_CAT(team_hrr_ket_, QCG_CLASS)<double>(p, y, CDx, CDy, CDz);
    }
    static __device__ __forceinline__ void hrr_bra(const double* y, double* o, int os, double ABx, double ABy,
                                                   double ABz)
    {
        gen::QCG_CAT(team_hrr_bra_, QCG_CLASS)<double>(y, o, os, ABx, ABy, ABz);
    }
};

constexpr int kThreads = Cls::kNW * 32;
constexpr int kNCD = ncart(Cls::LC) * ncart(Cls::LD);
constexpr size_t kSmem = 3 * (size_t)Cls::kStage * 32 * sizeof(double);   // three stages
std::atomic<unsigned long long> g_smem_ready{0};
}   // namespace

TeamShape QCG_CAT(team_shape_, QCG_CLASS)(int nsm)
{
    auto k = eri_batch_team_kernel<Cls>;
    ensure_smem(k, kSmem, g_smem_ready);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, kSmem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    TeamShape sh;
    sh.grid = nsm * per_sm;
    sh.threads = kThreads;
    sh.slot_doubles = (long long)Cls::kStage * 32;
    // [e0|f0], [e0|cd] and, for the J/K form, (ab|cd): lane-minor blocks of the group's 32 quartets
    sh.hrr_doubles = (long long)(Cls::kNE * Cls::kNF + Cls::kNE * kNCD + ncart(Cls::LA) * ncart(Cls::LB) * kNCD) * 32;
    return sh;
}

void QCG_CAT(launch_eri_team_, QCG_CLASS)(const BasisDev& bs, const int4* q, const int* order, long long nq,
                                          double* out, const double* boys, const TeamScratchDev& scr,
                                          const TeamShape& sh, cudaStream_t st)
{
    if (nq <= 0) return;
    auto k = eri_batch_team_kernel<Cls>;
    ensure_smem(k, kSmem, g_smem_ready);
    // one wave of CTAs, each walking groups of 32 quartets; the scratch has room for sh.grid CTAs
    const long long ngroups = (nq + 31) / 32;
    const long long blocks = ngroups < sh.grid ? ngroups : sh.grid;
    k<<<(unsigned)blocks, kThreads, kSmem, st>>>(bs, q, order, nq, out, boys, scr);
}

// the team form of the direct J/K build of this class (jk_team_kernel); the scratch has room for sh.grid CTAs
void QCG_CAT(launch_jk_team_, QCG_CLASS)(const JKWorkDev& w, const PairListDev& bra, const PairListDev& ket,
                                         const PrimPairsDev& P, const int* f0, const double* D, double* J,
                                         double* K, int n, const double* boys, const TeamScratchDev& scr,
                                         const TeamShape& sh, cudaStream_t st)
{
    const long long span = w.gend - w.gbeg;
    if (span <= 0) return;
    auto k = w.det_lo ? jk_team_kernel<Cls, true> : jk_team_kernel<Cls, false>;
    static std::atomic<unsigned long long> ready{0}, ready_det{0};
    ensure_smem(k, kSmem, w.det_lo ? ready_det : ready);
    const long long ngroups = (span + 31) / 32;
    const long long blocks = ngroups < sh.grid ? ngroups : sh.grid;
    k<<<(unsigned)blocks, kThreads, kSmem, st>>>(w, bra, ket, P, f0, D, J, K, n, boys, scr);
}

}   // namespace qcg
