// eri_team_iface.h -- launch interface of the team form of the FP64 ERI batches (eri_team.cu).
#pragma once
#include <cuda_runtime.h>

#include "qcg_internal.h"

namespace qcg {

// Device memory a team launch works in, beside its inputs and outputs (the handle owns it):
//   rcache -- per CTA, kmax stage slots: the primitive quartets' R tables and Hermite tables, written once
//             per group of quartets and streamed back into shared memory once per pass;
//   hrr    -- per CTA, the [e0|f0], [e0|cd] and (for the J/K form) (ab|cd) blocks of the group's 32 quartets,
//             lane-minor;
//   err    -- bit 0: a wait for a bulk copy gave up (the results of the launch are not valid);
//             bit 1: a group needed more stage slots than kmax.
struct TeamScratchDev
{
    double* rcache;
    int kmax;
    double* hrr;
    int* err;
};

// The launch shape of class k on nsm SMs and the scratch it needs per CTA, in doubles.
struct TeamShape
{
    int grid, threads;
    long long slot_doubles;   // one stage slot of the R cache
    long long hrr_doubles;
};

using EriTeamLauncher = void (*)(const BasisDev&, const int4*, const int*, long long, double*, const double*,
                                 const TeamScratchDev&, const TeamShape&, cudaStream_t);
using EriTeamShapeFn = TeamShape (*)(int nsm);

using JKTeamLauncher = void (*)(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&,
                                const int*, const double*, double*, double*, int, const double*,
                                const TeamScratchDev&, const TeamShape&, cudaStream_t);

extern const EriTeamLauncher kEriTeamLaunchers[kNumQuartetClasses];
extern const JKTeamLauncher kJKTeamLaunchers[kNumQuartetClasses];
extern const EriTeamShapeFn kEriTeamShapes[kNumQuartetClasses];

}   // namespace qcg
