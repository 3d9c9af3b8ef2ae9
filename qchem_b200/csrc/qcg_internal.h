// qcg_internal.h -- device-side views and kernel launchers shared by the CUDA translation units.
// Not part of the public ABI (include/qchem_b200.h is).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace qcg {

// pair classes (la >= lb): 0 ss, 1 ps, 2 pp, 3 ds, 4 dp, 5 dd
constexpr int kNumPairClasses = 6;
constexpr int kNumQuartetClasses = 21;   // (X,Y), X >= Y, index X(X+1)/2 + Y
constexpr int kPairLA[6] = {0, 1, 1, 2, 2, 2};
constexpr int kPairLB[6] = {0, 0, 1, 0, 1, 2};

// shells as structure of arrays; coef has the (L,0,0) primitive norm and the radial normalisation folded in
struct BasisDev
{
    int nshell;
    const int* L;
    const int* nprim;
    const int* prim0;
    const double* cen;     // 3 per shell
    const double* alpha;   // per primitive
    const double* coef;    // per primitive
};

// primitive-pair table (all pair classes share one table)
struct PrimPairsDev
{
    const double *p, *Px, *Py, *Pz, *PAx, *PAy, *PAz, *PBx, *PBy, *PBz, *K;
};

// shell pairs of one pair class, sorted by Schwarz bound descending (by molecule, then Schwarz bound
// descending, in a handle that holds several molecules)
struct PairListDev
{
    int n;
    const int* sa;
    const int* sb;
    const int* ppo;
    const int* npp;
    const double* Q;     // Schwarz bound of each pair (same order)
    const int* mol;      // molecule of each pair (null for a single molecule)
};

// Several molecules in one handle: matrices are packed, molecule m's n_m x n_m block (row-major, local
// function indices) starting at element off[m]; nmol == 1 is the plain dense nbf x nbf layout.
struct MolLayoutDev
{
    int nmol;
    const long long* off;   // nmol + 1 entries, off[nmol] = elements of a packed matrix
    const int* n;           // functions of each molecule
};

// flattened canonical quartets of one quartet class: bra pair i owns quartets offs[i] .. offs[i+1)
struct JKWorkDev
{
    long long total;
    // the slice [gbeg, gend) of the class's quartets this build evaluates (a rank's shard; 0 and total
    // for the whole build)
    long long gbeg, gend;
    const long long* offs;
    int same_class;
    // density screening of an incremental build: skip a quartet when
    // Q_ab Q_cd max(|D| over its six digestion blocks) < dthr; dmax[a*nshell+b] = max |D| of block (a,b)
    const double* dmax;
    int nshell;
    double dthr;
    // precision band: this launch evaluates the quartets whose bound lies in [lo, hi) (0 and >= 1e300:
    // every quartet)
    double lo, hi;
    // several molecules: the kets of bra pair i start at kbase[i] (the bra's molecule's part of the ket
    // class); D, J', K' of a quartet are the packed blocks of its molecule
    const int* kbase;
    MolLayoutDev mols;
    // launch shape: quartets per lane and blocks-per-SM cap (0: the launcher's own choice; set by the
    // autotuner, qcg_autotune_jk)
    int run, cap;
    // several molecules: mol_active[m] == 0 skips molecule m's quartets (a batched SCF's converged
    // molecules); null: every molecule
    const int* mol_active;
    // a subset of shell pairs (qcg_set_pair_subset): a quartet is evaluated only when pmask[a * nshell + b]
    // and pmask[c * nshell + d] are both set (the mask is symmetric); null: every quartet
    const unsigned char* pmask;
    // deterministic accumulation (QCG_JK_DETERMINISTIC): J' and K' are pairs of 64-bit integer words, the
    // high word at element k (units of 2^-30) and the low word at k + det_lo (units of 2^-70), summed with
    // integer atomics, so that the result does not depend on their order; 0: FP64 atomics
    long long det_lo;
};

// One contribution v to a deterministic accumulator pair (hi word at p[k], lo word at p[k + lo]).  v is split
// exactly: hi = round(v 2^30), the remainder r = v - hi 2^-30 is exact (|r| <= 2^-31) and lo = round(r 2^70),
// so a contribution is represented to 2^-71 and the two integer sums are exact for |J'|, |K'| < 2^33 and
// fewer than 2^24 contributions per element.
__device__ __forceinline__ void fixed_add(double* p, size_t k, long long lo_off, double v)
{
    const long long hi = __double2ll_rn(v * 0x1p30);
    const double r = v - (double)hi * 0x1p-30;
    const long long lo = __double2ll_rn(r * 0x1p70);
    unsigned long long* w = reinterpret_cast<unsigned long long*>(p);
    atomicAdd(w + k, (unsigned long long)hi);
    atomicAdd(w + k + lo_off, (unsigned long long)lo);
}

void launch_block_max(const double* D, const int* shell_f0, const int* shell_L, int nshell, int n, double* dmax,
                      cudaStream_t st, int nsm);

// launchers, two object files per quartet class (eri_class.cu compiled with -DQCG_CLASS=k and
// -DQCG_PREC=64 or 32)
using EriBatchLauncher = void (*)(const BasisDev&, const int4*, const int*, long long, double*, const double*,
                                  cudaStream_t, int);
using JKLauncher = void (*)(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&, const int*,
                            const double*, double*, double*, int, const double*, cudaStream_t, int);
// the warp-shared J/K form (FP64): gbra = bra pairs grouped by first shell, items = {gbra start, lanes,
// first ket, end ket}
using JKWarpLauncher = void (*)(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&,
                                const int*, const double*, double*, double*, int, const double*, const int*,
                                const int4*, long long, cudaStream_t, int);
extern const JKWarpLauncher kJKWarpLaunchers[kNumQuartetClasses];
using SchwarzLauncher = void (*)(const PairListDev&, const PrimPairsDev&, double*, const double*, cudaStream_t, int);

using EriBatch32Launcher = void (*)(const BasisDev&, const int4*, const int*, long long, float*, const double*,
                                    cudaStream_t, int);

extern const EriBatchLauncher kEriBatchLaunchers[kNumQuartetClasses];
extern const EriBatch32Launcher kEriBatch32Launchers[kNumQuartetClasses];

// counting sort of a quartet batch by contraction pattern -> order (a permutation of 0..nq-1)
void launch_pattern_sort(const BasisDev& bs, const int4* quartets, long long nq, unsigned char* key, int* hist,
                         int* cursor, int* order, cudaStream_t st, int nsm);
extern const JKLauncher kJKLaunchers[kNumQuartetClasses];     // FP64 evaluation
extern const JKLauncher kJK32Launchers[kNumQuartetClasses];   // FP32 evaluation, FP64 accumulation
extern const SchwarzLauncher kSchwarzLaunchers[kNumPairClasses];

}   // namespace qcg
