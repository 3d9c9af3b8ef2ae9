// registry.cu -- tables of the per-class launchers compiled in the 42 eri_class objects (21 classes x FP64/FP32)
// and the 21 eri_team objects (the team form of the FP64 ERI batches); the warp-shared J/K form is in the
// FP64 eri_class objects.
#include "eri_team_iface.h"
#include "qcg_internal.h"

namespace qcg {

#define QCG_DECL(k)                                                                                          \
    void launch_eri_batch_##k(const BasisDev&, const int4*, const int*, long long, double*, const double*,          \
                              cudaStream_t, int);                                                                   \
    void launch_jk_##k(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&, const int*,    \
                       const double*, double*, double*, int, const double*, cudaStream_t, int);                      \
    void launch_schwarz_##k(const PairListDev&, const PrimPairsDev&, double*, const double*, cudaStream_t, int);      \
    void launch_eri_batch32_##k(const BasisDev&, const int4*, const int*, long long, float*, const double*,        \
                                cudaStream_t, int);                                                                 \
    void launch_jk32_##k(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&, const int*,  \
                         const double*, double*, double*, int, const double*, cudaStream_t, int);                    \
    void launch_eri_team_##k(const BasisDev&, const int4*, const int*, long long, double*, const double*,            \
                             const TeamScratchDev&, const TeamShape&, cudaStream_t);                                 \
    TeamShape team_shape_##k(int);                                                                                  \
    void launch_jk_team_##k(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&,          \
                            const int*, const double*, double*, double*, int, const double*, const TeamScratchDev&, \
                            const TeamShape&, cudaStream_t);                                                        \
    void launch_jk_warp_##k(const JKWorkDev&, const PairListDev&, const PairListDev&, const PrimPairsDev&,          \
                            const int*, const double*, double*, double*, int, const double*, const int*,            \
                            const int4*, long long, cudaStream_t, int);
QCG_DECL(0) QCG_DECL(1) QCG_DECL(2) QCG_DECL(3) QCG_DECL(4) QCG_DECL(5) QCG_DECL(6) QCG_DECL(7) QCG_DECL(8)
QCG_DECL(9) QCG_DECL(10) QCG_DECL(11) QCG_DECL(12) QCG_DECL(13) QCG_DECL(14) QCG_DECL(15) QCG_DECL(16)
QCG_DECL(17) QCG_DECL(18) QCG_DECL(19) QCG_DECL(20)
#undef QCG_DECL

const EriBatchLauncher kEriBatchLaunchers[kNumQuartetClasses] = {
    launch_eri_batch_0,  launch_eri_batch_1,  launch_eri_batch_2,  launch_eri_batch_3,  launch_eri_batch_4,
    launch_eri_batch_5,  launch_eri_batch_6,  launch_eri_batch_7,  launch_eri_batch_8,  launch_eri_batch_9,
    launch_eri_batch_10, launch_eri_batch_11, launch_eri_batch_12, launch_eri_batch_13, launch_eri_batch_14,
    launch_eri_batch_15, launch_eri_batch_16, launch_eri_batch_17, launch_eri_batch_18, launch_eri_batch_19,
    launch_eri_batch_20};
const EriTeamShapeFn kEriTeamShapes[kNumQuartetClasses] = {
    team_shape_0,  team_shape_1,  team_shape_2,  team_shape_3,  team_shape_4,  team_shape_5,  team_shape_6,
    team_shape_7,  team_shape_8,  team_shape_9,  team_shape_10, team_shape_11, team_shape_12, team_shape_13,
    team_shape_14, team_shape_15, team_shape_16, team_shape_17, team_shape_18, team_shape_19, team_shape_20};
const JKTeamLauncher kJKTeamLaunchers[kNumQuartetClasses] = {
    launch_jk_team_0,  launch_jk_team_1,  launch_jk_team_2,  launch_jk_team_3,  launch_jk_team_4,
    launch_jk_team_5,  launch_jk_team_6,  launch_jk_team_7,  launch_jk_team_8,  launch_jk_team_9,
    launch_jk_team_10, launch_jk_team_11, launch_jk_team_12, launch_jk_team_13, launch_jk_team_14,
    launch_jk_team_15, launch_jk_team_16, launch_jk_team_17, launch_jk_team_18, launch_jk_team_19,
    launch_jk_team_20};
const JKWarpLauncher kJKWarpLaunchers[kNumQuartetClasses] = {
    launch_jk_warp_0,  launch_jk_warp_1,  launch_jk_warp_2,  launch_jk_warp_3,  launch_jk_warp_4,
    launch_jk_warp_5,  launch_jk_warp_6,  launch_jk_warp_7,  launch_jk_warp_8,  launch_jk_warp_9,
    launch_jk_warp_10, launch_jk_warp_11, launch_jk_warp_12, launch_jk_warp_13, launch_jk_warp_14,
    launch_jk_warp_15, launch_jk_warp_16, launch_jk_warp_17, launch_jk_warp_18, launch_jk_warp_19,
    launch_jk_warp_20};
const EriTeamLauncher kEriTeamLaunchers[kNumQuartetClasses] = {
    launch_eri_team_0,  launch_eri_team_1,  launch_eri_team_2,  launch_eri_team_3,  launch_eri_team_4,
    launch_eri_team_5,  launch_eri_team_6,  launch_eri_team_7,  launch_eri_team_8,  launch_eri_team_9,
    launch_eri_team_10, launch_eri_team_11, launch_eri_team_12, launch_eri_team_13, launch_eri_team_14,
    launch_eri_team_15, launch_eri_team_16, launch_eri_team_17, launch_eri_team_18, launch_eri_team_19,
    launch_eri_team_20};
const JKLauncher kJKLaunchers[kNumQuartetClasses] = {
    launch_jk_0,  launch_jk_1,  launch_jk_2,  launch_jk_3,  launch_jk_4,  launch_jk_5,  launch_jk_6,
    launch_jk_7,  launch_jk_8,  launch_jk_9,  launch_jk_10, launch_jk_11, launch_jk_12, launch_jk_13,
    launch_jk_14, launch_jk_15, launch_jk_16, launch_jk_17, launch_jk_18, launch_jk_19, launch_jk_20};
const EriBatch32Launcher kEriBatch32Launchers[kNumQuartetClasses] = {
    launch_eri_batch32_0,  launch_eri_batch32_1,  launch_eri_batch32_2,  launch_eri_batch32_3,  launch_eri_batch32_4,
    launch_eri_batch32_5,  launch_eri_batch32_6,  launch_eri_batch32_7,  launch_eri_batch32_8,  launch_eri_batch32_9,
    launch_eri_batch32_10, launch_eri_batch32_11, launch_eri_batch32_12, launch_eri_batch32_13, launch_eri_batch32_14,
    launch_eri_batch32_15, launch_eri_batch32_16, launch_eri_batch32_17, launch_eri_batch32_18, launch_eri_batch32_19,
    launch_eri_batch32_20};
const JKLauncher kJK32Launchers[kNumQuartetClasses] = {
    launch_jk32_0,  launch_jk32_1,  launch_jk32_2,  launch_jk32_3,  launch_jk32_4,  launch_jk32_5,  launch_jk32_6,
    launch_jk32_7,  launch_jk32_8,  launch_jk32_9,  launch_jk32_10, launch_jk32_11, launch_jk32_12, launch_jk32_13,
    launch_jk32_14, launch_jk32_15, launch_jk32_16, launch_jk32_17, launch_jk32_18, launch_jk32_19, launch_jk32_20};
// diagonal classes X == Y have quartet index X(X+1)/2 + X
const SchwarzLauncher kSchwarzLaunchers[kNumPairClasses] = {launch_schwarz_0, launch_schwarz_2,  launch_schwarz_5,
                                                            launch_schwarz_9, launch_schwarz_14, launch_schwarz_20};

}   // namespace qcg
