/* qchem_b200.h -- C ABI of the B200 McMurchie-Davidson ERI engine and direct J/K Fock build.
 *
 * Drop-in boundary for qchem's molecular Hartree-Fock path (JanReimers/qchem).  Style follows the
 * reference's flat bridge header pybind/qcb_api.h:14-37: extern "C", an opaque handle, caller-owned
 * buffers, int status codes, no C++ types across the boundary.
 *
 * Each entry point names the reference interface it replaces:
 *   qcg_basis_create    PG_Cart IrrepBasisSet + PGData::Init (flattened shells, unit-self-overlap norms)
 *                       src/BasisSet/Molecule/PG_Cart/Imp/IrrepBasisSet.C:60-147,
 *                       src/BasisSet/Molecule/Evaluators/PG_Cart_MnD/Imp/PGData.C:17-33
 *   qcg_eri_batch       NR_Evaluator::FourC for whole shell quartets
 *                       src/BasisSet/Molecule/Evaluators/PG_Cart_MnD/Evaluator.C:1912-1920
 *   qcg_schwarz         (no reference counterpart: the reference stores full ERI4 blocks; this prepares the
 *                       screened direct build that replaces them)
 *   qcg_fock_jk         Orbital_HF_IBS<double>::AccumulateDirect / AccumulateExchange and
 *                       WholeSystemFock_IBS<double>::MakeAOFock(Dao, exchange)
 *                       src/BasisSet/Orbital_HF_IBS.C:33-54,75-87; the ERI4 build + contraction they use
 *                       src/BasisSet/Molecule/IrrepBasisSet.C:138-183, src/BasisSet/Internal/Imp/ERI4.C:10-42
 *   qcg_one_electron    NR_Evaluator::Overlap / Grad2 / Nuclear   (Evaluator.C:71-76)
 *   qcg_rhf             Calculation + SCFIterator::Iterate with DIIS  (src/SCFIterator/Imp/SCFIterator.C:283-398)
 *
 * Matrices are dense, row-major, nbf x nbf doubles; D is the total RHF density (occupation 2).
 * J_ab = sum_cd (ab|cd) D_cd and K_ac = sum_bd (ab|cd) D_bd, both UNSCALED (the caller forms
 * F = H + J - 1/2 K, as HF_HT.C:48-70 does).  The engine is single-stream and not re-entrant per handle.
 */
#ifndef QCHEM_B200_H
#define QCHEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qcg_handle qcg_handle;

enum qcg_status {
    QCG_OK = 0,
    QCG_ERR_ARG = 1,         /* invalid argument (null pointer, bad size, L > 2, non-canonical class...) */
    QCG_ERR_CUDA = 2,        /* a CUDA runtime call failed; see qcg_last_error */
    QCG_ERR_NONFINITE = 3,   /* NaN/Inf in an input matrix or in a result */
    QCG_ERR_ASYMMETRIC = 4,  /* density matrix not symmetric */
    QCG_ERR_ALLOC = 5,       /* device allocation failed or exceeded the handle's memory limit */
    QCG_ERR_STATE = 6,       /* call order violated (e.g. qcg_fock_jk before qcg_schwarz) */
    QCG_ERR_NOCONV = 7       /* SCF did not converge within the iteration limit */
};

/* flags for qcg_fock_jk */
#define QCG_JK_SKIP_VALIDATION 1   /* do not check D for NaN/Inf and symmetry */
#define QCG_JK_J_ONLY 2            /* reserved: both J and K are always built */
#define QCG_JK_FP32 4              /* evaluate every quartet in FP32 (accumulation into J and K stays FP64) */
/* accumulate J and K as exact 64-bit integer pairs (units of 2^-30 and 2^-70) instead of FP64 atomics, each
 * quartet's contribution rounded alone: the result is the same bit for bit from build to build, whatever order
 * the GPU's atomic updates take and whatever launch shapes the autotuner chose (for a given basis and shard);
 * each contribution is represented to 2^-71, and |J|, |K| must stay below 2^32.  Not recorded as a CUDA graph. */
#define QCG_JK_DETERMINISTIC 8

typedef struct qcg_stats {
    double ms_total;          /* device time of the whole J/K build (CUDA events) */
    double ms_eri;            /* device time of the ERI + digestion kernels */
    long long quartets;       /* shell quartets evaluated after screening */
    long long prim_quartets;  /* primitive quartets evaluated */
    double flops;             /* algorithmic FLOPs (fixed per-class formula) of the ERI work */
} qcg_stats;

typedef struct qcg_scf_params {
    int max_iter;             /* default 100 */
    double de_tol;            /* |E_k - E_{k-1}| stop, default 1e-10 Eh */
    double fd_tol;            /* ||[F',D']|| must also be below this, default 1e-5 (SCFParams MinFD) */
    double schwarz_thresh;    /* default 1e-10 */
    int diis_nproj;           /* default 4 */
    double diis_fdmax;        /* <= 0: Z^2 * 0.1 / 32 (Calculation.C default) */
    double diis_svtol;        /* default 5e-9 */
    int incremental;          /* 0 (default): full FP64 J/K every iteration.  1: after a full build, build
                                 J[D_k - D_k-1], K[...] with density-weighted Schwarz screening and add them
                                 to the previous J, K; full rebuild every rebuild_every iterations, for every
                                 iteration once |dE| < 1000 de_tol (each screened build adds its own small
                                 error), and once more on convergence (the reported energy is from a full
                                 build) */
    double inc_thresh;        /* skip a quartet of an incremental build when Q_ab Q_cd max|dD| < inc_thresh
                                 (default 1e-11) */
    int rebuild_every;        /* default 8 */
    int fp32_early;           /* 1: until the DIIS error first falls below fp32_switch, quartets whose density-
                                 weighted bound Q_ab Q_cd max|D| is below fp32_scale * (previous DIIS error) are
                                 evaluated in FP32 (FP64 accumulation, FP64 Boys below T = 12), then a full FP64
                                 rebuild; default 0 */
    double fp32_switch;       /* default 1e-5 */
    double fp32_scale;        /* <= 0 (default): 1e-4 / (3e-7 nbf^2), i.e. the worst-case FP32 error of a Fock
                                 element (nbf^2 quartets of relative error 3e-7) at 1e-4 of the DIIS error */
    double fp32_below;        /* after the switch, quartets whose bound is below this stay FP32; default 0 */
    const double* D_guess;    /* optional initial total density, nbf*nbf (NULL: core-Hamiltonian guess) */
    int autotune;             /* 1: qcg_autotune_jk on the first density before the first build; default 0 */
    int spherical;            /* 1: the SCF in real solid-harmonic functions (qcg_spherical_transform); D_guess
                                 and D_out are then spherical; needs incremental = 0; default 0 */
    int deterministic;        /* 1: every J/K build with QCG_JK_DETERMINISTIC (exact integer accumulation), so
                                 that the trajectory, the iteration count and the energy repeat bit for bit from
                                 run to run -- near-degenerate SCFs otherwise follow the rounding of the FP64
                                 atomics; each build costs about 1.9x; not with fp32_early or fp32_below > 0;
                                 default 0 */
} qcg_scf_params;

typedef struct qcg_scf_result {
    double energy;            /* total energy incl. nuclear repulsion */
    double e_nuc;
    int iterations;
    int converged;
    double fd_error;          /* final ||[F',D']|| */
    double wall_s;            /* host wall time of qcg_rhf */
    double fock_ms;           /* summed device time of the J/K builds */
    int full_builds;          /* J/K builds from the full density */
    int incremental_builds;   /* J/K builds from a density difference */
    int fp32_builds;          /* J/K builds in which quartets below a bound were evaluated in FP32 */
} qcg_scf_result;

/* ---- lifetime -------------------------------------------------------------------------------- */
/* Shells in basis order.  shell_L[i] in {0,1,2}; primitives of shell i are the next shell_nprim[i]
 * entries of exps/coefs (raw contraction coefficients: the engine folds the (L,0,0) primitive norm and
 * renormalises every Cartesian component to unit self-overlap); centres: 3 doubles per shell (bohr). */
int qcg_basis_create(const int* shell_L, const int* shell_nprim, const double* exps, const double* coefs,
                     const double* centres, int nshell, qcg_handle** out);
/* Several molecules in one handle (batched SCF): shells grouped by molecule in molecule order,
 * shell_mol[i] in [0, nmol).  Shell pairs and quartets never mix molecules.  Every matrix argument of the
 * J/K calls is then PACKED: molecule m's n_m x n_m block (row-major, the molecule's own function order)
 * follows molecule m-1's.  qcg_basis_create is the nmol = 1 case.  No reference counterpart: the
 * reference runs one molecule per Calculation. */
int qcg_basis_create_batch(const int* shell_L, const int* shell_nprim, const double* exps, const double* coefs,
                           const double* centres, int nshell, const int* shell_mol, int nmol, qcg_handle** out);
int qcg_nmol(const qcg_handle* h, int* nmol);
int qcg_mol_nbf(const qcg_handle* h, int* nbf_per_molecule);   /* nmol entries */
/* Destroying a handle keeps its idle device slabs, pinned staging buffer, streams and events in a
 * process-wide cache that the next handle on the same device reuses: handle set-up and tear-down then
 * cost no allocation or synchronising free (about 6 ms of a 57-function RHF otherwise).
 * qcg_release_cache frees everything in the cache (resources of live handles are not in it); call it
 * from the thread that owns the CUDA context before cudaDeviceReset or when the memory is wanted back.
 * No reference counterpart (the reference has no device resources). */
void qcg_destroy(qcg_handle* h);
void qcg_release_cache(void);
const char* qcg_last_error(const qcg_handle* h);
/* stream for all later work of this handle; NULL is the CUDA default (legacy) stream.  A new handle
 * starts on its own non-blocking stream. */
int qcg_set_stream(qcg_handle* h, void* cuda_stream);
int qcg_set_memory_limit(qcg_handle* h, long long bytes); /* cap on device bytes this handle allocates; 0 = none */
int qcg_nbf(const qcg_handle* h, int* nbf);
int qcg_nshell(const qcg_handle* h, int* nshell);
/* per-function normalisation constants ns (1/sqrt of the self-overlap of the coefficient-scaled radial) */
int qcg_norms(const qcg_handle* h, double* ns);

/* ---- integrals ------------------------------------------------------------------------------- */
/* Cartesian ERIs of nq shell quartets of ONE canonical class (la>=lb, lc>=ld, (la,lb) >= (lc,ld) in
 * the order ss<ps<pp<ds<dp<dd).  quartets: 4 int32 shell indices per quartet, whose L must match the
 * class.  out: nq blocks of nA*nB*nC*nD doubles, row-major [a][b][c][d].  Host buffers. */
int qcg_eri_batch(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, double* out);
/* same with device pointers (no validation of the shell L's; the stream is the handle's) */
int qcg_eri_batch_device(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* d_quartets,
                         double* d_out);
/* 3-centre Coulomb integrals (ab|c) of nt shell triples (3 int32 each; 2 >= la >= lb, lc <= 2):
 * out[t][a][b][c], contracted and normalised like NR_Evaluator::RepulsionThreeC
 * (src/BasisSet/Molecule/Evaluators/PG_Cart_MnD/Evaluator.C:1905-1908, primitive integral GaussianRF.C:415-444),
 * the integrals of density-fitted Coulomb.  Fitting shells are ordinary shells of the handle.  Host buffers. */
int qcg_eri3_batch(qcg_handle* h, int la, int lb, int lc, long long nt, const int* triples, double* out);
/* FP32 forms of the two batch calls: the same integrals evaluated in FP32 arithmetic (pair data, Boys
 * argument, prefactor and Boys below T = 12 in FP64, rounded once) with float output.  No reference
 * counterpart (the reference is FP64 only). */
int qcg_eri_batch_f32(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, float* out);
int qcg_eri_batch_device_f32(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* d_quartets,
                             float* d_out);

/* Schwarz bounds Q_ab = sqrt(max |(ab|ab)|) for every shell pair and the screened quartet lists used by
 * qcg_fock_jk (quartets with Q_ab Q_cd < thresh are skipped).  Q: optional, nshell*nshell doubles. */
int qcg_schwarz(qcg_handle* h, double thresh, double* Q);

/* J and K for a total density D.  Host buffers (copies inside). */
int qcg_fock_jk(qcg_handle* h, const double* D, double* J, double* K, int flags, qcg_stats* stats);
/* same with device pointers on the handle's stream; results are ready when the stream reaches them */
int qcg_fock_jk_device(qcg_handle* h, const double* d_D, double* d_J, double* d_K, int flags, qcg_stats* stats);
/* Mixed precision for later qcg_fock_jk / qcg_fock_jk_device calls: quartets whose density-weighted
 * Schwarz bound Q_ab Q_cd max|D| (max over the six D blocks the quartet touches) is below `bound` are
 * evaluated in FP32 (accumulated in FP64), the rest in FP64.  0 (the default) keeps every quartet FP64.
 * No reference counterpart. */
int qcg_set_fp32_bound(qcg_handle* h, double bound);
/* 1: J/K builds repeated with the same arguments (device pointers, screening, precision) are captured as
 * a CUDA graph on their second occurrence and replayed afterwards; 0 (default): launched kernel by kernel.
 * Also switched on by the environment variable QCG_GRAPHS=1.  The handle's stream must not be the legacy
 * default stream for capture to happen. */
int qcg_set_graphs(qcg_handle* h, int enable);
/* Which FP64 ERI-batch classes (bit k: class k of qcg_eri_batch*) run in the team form -- a warp-specialised
 * kernel that shares each primitive quartet's R table among the warps of a CTA and transfers to (ab|cd) once
 * per contracted quartet -- rather than the one-thread-per-quartet form.  -1 (default): the library's own
 * choice, or the mask in the environment variable QCG_ERI_TEAM_MASK.  Both forms give the same integrals
 * to rounding.  No reference counterpart. */
int qcg_set_eri_team_classes(qcg_handle* h, long long mask);
/* The same choice for the direct J/K build (bit k: class k of the work lists): the team kernel, whose CTAs
 * digest each group's integral blocks into J and K, or the thread-per-quartet kernel; -1 (default): the
 * library's choice -- the team form for the (dd|xx) classes except (dd|ss), and (dp|dp), of a build with at least
 * 2^20 quartets in the class -- or QCG_JK_TEAM_MASK in the environment (a mask set here or there applies at
 * any size).  Same J and K to rounding (bit for bit under QCG_JK_DETERMINISTIC only within one form).  No
 * reference counterpart. */
int qcg_set_jk_team_classes(qcg_handle* h, long long mask);
/* The warp-shared form of the direct J/K build for the classes in mask (bit k: class k; the team form takes
 * precedence where both are set): each half of a warp takes up to 16 bra pairs sharing their first shell
 * against one ket pair at a time, so that the J'(cd), K'(ac) and K'(ad) contributions of its lanes are added
 * by warp shuffles and written once per half warp instead of once per lane.  FP64 builds of one rank (not
 * with qcg_set_shard or QCG_JK_DETERMINISTIC).  -1 (default): the library's choice -- the (ps|ss), (ps|ps),
 * (pp|ss), (pp|ps), (ds|xx), (dp|ss), (dp|ps), (dp|pp) and (dp|ds) classes of full builds with at least 2^20
 * quartets in the class -- or QCG_JK_WARP_MASK in the environment (a mask set here or there applies to every
 * build).  Same J
 * and K to rounding.  No reference counterpart. */
int qcg_set_jk_warp_classes(qcg_handle* h, long long mask);
/* Restrict later J/K builds to a subset of shell pairs: mask (nshell x nshell bytes, row-major; pair (a,b) is
 * in the subset when mask[a*nshell+b] or mask[b*nshell+a] is non-zero) selects the pairs, and a quartet
 * (ab|cd) is evaluated only when both (a,b) and (c,d) are in it; J and K are then that sub-block's
 * contribution.  NULL restores every quartet.  Single-molecule handles.  Used to check slices of a large
 * build against the CPU oracle; no reference counterpart. */
int qcg_set_pair_subset(qcg_handle* h, const unsigned char* mask);
/* Several GPUs on one J/K build: with (rank, world) set, later qcg_fock_jk* calls evaluate only this rank's
 * contiguous slice of every class's screened quartets (1/world of its primitive quartets, see
 * qcg_shard_work) and return the rank's PARTIAL J and K;
 * the sum over ranks (one all-reduce) is the full J and K.  (0, 1), the default, is the whole build.  The
 * qcg_stats figures still describe the whole build.  No reference counterpart (the reference is one
 * process). */
int qcg_set_shard(qcg_handle* h, int rank, int world);
/* The work of share `rank` of `world` under qcg_set_shard: its screened shell quartets and primitive quartets.
 * The shares are cut at equal fractions of every class's primitive quartets (a contracted quartet costs its
 * primitive-quartet count), so their primitive counts are equal to within one quartet per class while their
 * quartet counts may differ.  Needs qcg_schwarz first.  No reference counterpart. */
int qcg_shard_work(qcg_handle* h, int rank, int world, long long* quartets, long long* prim_quartets);
/* Autotuner of the J/K launch shapes.  For every quartet class it times the class kernel on up to 2^20 of
 * the handle's screened quartets (density d_D, `reps` timed launches per candidate) for each candidate
 * (quartets per lane 1, 2, 4, 8, 16) x (blocks per SM 8, 16) and keeps the fastest for later builds of this
 * handle, until the screening changes.  run_out / cap_out (optional, 21 ints each) receive the choices.
 * No reference counterpart. */
int qcg_autotune_jk(qcg_handle* h, const double* d_D, int reps, int* run_out, int* cap_out);

/* The J/K build of qcg_fock_jk_device for callers that must not allocate device memory once their setup
 * is done -- for example a host program whose device memory is owned by its own pool allocator, or one
 * that runs under a device-memory budget fixed at startup.  This call performs no cudaMalloc, cudaFree or
 * other allocating call: its J'/K' accumulators live in a file-scope device array of the library, sized
 * for at most 512 basis functions (larger bases are rejected with QCG_ERR_ARG).  qcg_basis_create and
 * qcg_schwarz, which do allocate, must have run before.  The first call on a device looks up the array's
 * device address; make that first call before any stream capture (qcg_release_cache forgets the address,
 * so the first call after it looks it up again).  All calls share the one array (it keeps the last call's
 * contents and is cleared at the start of each call), so calls that overlap on the GPU race: issue them in
 * order on one stream.  It evaluates this rank's slice after qcg_set_shard and uses the autotuned launch
 * shape, like qcg_fock_jk_device, but always in FP64 (qcg_set_fp32_bound does not apply).  No validation of
 * D, and no report of non-finite results.  Has no counterpart in the reference. */
int qcg_fock_jk_device_noalloc(qcg_handle* h, const double* d_D, double* d_J, double* d_K);

/* Real solid-harmonic (spherical) functions, the reference's PG_Spherical basis: per shell 2L+1 components
 * ordered m = -L..L (p: y, z, x; d: xy, yz, z^2-(x^2+y^2)/2, xz, x^2-y^2), each normalised to unit
 * self-overlap (src/BasisSet/Molecule/Evaluators/PG_Spherical_MnD/Evaluator.C:84-96, Imp/Evaluator.C:13-24).
 * T (nbf x nbf_spherical, row-major) maps them onto the handle's Cartesian functions, chi_s = sum_t T_ts phi_t;
 * J and K of a spherical density are T^T J[T D T^T] T and T^T K[...] T (host buffers, nbf_spherical^2). */
int qcg_nbf_spherical(const qcg_handle* h, int* n);
int qcg_spherical_transform(qcg_handle* h, double* T);
int qcg_fock_jk_spherical(qcg_handle* h, const double* D, double* J, double* K, int flags, qcg_stats* stats);

/* overlap, kinetic (1/2 <grad|grad>) and nuclear attraction, natom nuclei of charge Z at R (3 per atom) */
int qcg_one_electron(qcg_handle* h, int natom, const double* Z, const double* R, double* S, double* T, double* V);
/* the same for a batch handle: molecule m has mol_natom[m] nuclei (Z, R concatenated in molecule order);
 * S, T, V packed */
int qcg_one_electron_batch(qcg_handle* h, const int* mol_natom, const double* Z, const double* R, double* S,
                           double* T, double* V);

/* ---- RHF ------------------------------------------------------------------------------------- */
void qcg_scf_default_params(qcg_scf_params* p);
/* Closed-shell SCF: core-Hamiltonian guess, Pulay DIIS on the orthonormal-basis Fock matrix, J/K on the
 * GPU every iteration.  D_out (optional, nbf*nbf) receives the final density. */
int qcg_rhf(qcg_handle* h, int natom, const double* Z, const double* R, int nelec, const qcg_scf_params* params,
            qcg_scf_result* result, double* D_out);
/* All molecules of a batch handle to convergence together: each iteration is one J/K build over every
 * molecule, then per-molecule host steps in parallel.  results: nmol entries (wall_s and fock_ms are the
 * batch's); D_out optional, packed.  D_guess (optional) is packed too: one initial density per molecule.
 * The incremental and fp32 parameters are ignored. */
int qcg_rhf_batch(qcg_handle* h, const int* mol_natom, const double* Z, const double* R, const int* nelec,
                  const qcg_scf_params* params, qcg_scf_result* results, double* D_out);

/* ---- learned initial guess ------------------------------------------------------------------ */
/* A multilayer perceptron (SiLU hidden layers, linear output) whose forward and backward passes and Adam
 * updates run on the GPU: matrix-product operands rounded to BF16, FP32 accumulation, FP32 master
 * weights.  It maps per-atom-pair geometry features to density-matrix blocks; the predicted density is
 * handed to qcg_rhf through qcg_scf_params.D_guess.  No reference counterpart: the reference always
 * starts from the core Hamiltonian (src/SCFIterator/Imp/Seed.C:70-80).  Row-major float32 device arrays;
 * parameters are laid out layer by layer as W (out x in) then b (out). */
typedef struct qcg_mlp qcg_mlp;
int qcg_mlp_create(int nlayers, const int* widths /* nlayers+1 */, unsigned long long seed, qcg_mlp** out);
void qcg_mlp_destroy(qcg_mlp* m);
const char* qcg_mlp_last_error(const qcg_mlp* m);
int qcg_mlp_set_stream(qcg_mlp* m, void* cuda_stream);
int qcg_mlp_nparams(const qcg_mlp* m, long long* n);
int qcg_mlp_params(qcg_mlp* m, float* host_params);            /* copy out (nparams floats) */
int qcg_mlp_set_params(qcg_mlp* m, const float* host_params);  /* copy in; resets the Adam moments */
/* y (rows x widths[L]) = network(x (rows x widths[0])) */
int qcg_mlp_forward(qcg_mlp* m, int rows, const float* d_x, float* d_y);
/* masked mean-squared error sum(mask (y - t)^2) / sum(mask) (mask entries 0 or 1) and its gradient with
 * respect to every parameter (kept for qcg_mlp_adam; also copied to grad_host when given) */
int qcg_mlp_loss_grad(qcg_mlp* m, int rows, const float* d_x, const float* d_target, const float* d_mask, float* loss,
                      float* grad_host);
/* one Adam step with decoupled weight decay on the last gradient */
int qcg_mlp_adam(qcg_mlp* m, float lr, float beta1, float beta2, float eps, float weight_decay);

/* ---- symmetry-adapted (SALC) blocks ----------------------------------------------------------- */
/* qchem's WholeSystemFock_IBS face of a symmetry-adapted basis (src/BasisSet/Orbital_HF_IBS.C:75-87,
 * src/BasisSet/Imp/SymmetryAdapted_IBS.C:45-70): one irrep block is m functions, the columns of O (nbf x m,
 * row-major, over the handle's Cartesian AO functions).  J and K are linear in D, so the whole system's J
 * and K come from ONE AO build of the summed density: each block folds its density up (qcg_salc_fold), the
 * AO build runs once (qcg_fock_jk), and each block slices its part out (qcg_salc_slice).  Both products run
 * on the GPU (cuBLAS, the handle's stream); the results are symmetrised, as the reference's SymCopy does.
 * Host buffers, synchronous; single-molecule handles. */
/* Dao (nbf x nbf) += sym(O D O^T), D (m x m) the block's density */
int qcg_salc_fold(qcg_handle* h, int m, const double* O, const double* D, double* Dao);
/* Fab (m x m) += sym(O^T Fao O), Fao (nbf x nbf) an AO matrix (J, K or a Fock matrix) */
int qcg_salc_slice(qcg_handle* h, int m, const double* O, const double* Fao, double* Fab);

/* ---- measurement ----------------------------------------------------------------------------- */
/* FP64 fused-multiply-add throughput of the current device (TFLOP/s) from a pure-DFMA kernel timed over
 * `reps` launches: the roofline denominator of the ERI kernels.  No reference counterpart. */
int qcg_measure_fp64_peak(int reps, double* tflops, double* ms_per_launch);
/* the same for FP32 fused multiply-adds: the roofline denominator of the FP32 ERI kernels */
int qcg_measure_fp32_peak(int reps, double* tflops, double* ms_per_launch);

/* ---- failure handling ------------------------------------------------------------------------ */
/* Runs the team kernels' bounded mbarrier wait on its own, on the current device: one thread waits for the
 * first phase of a barrier that expects one arrival.  arrive != 0: the arrival comes first and the wait
 * completes (*gave_up = 0).  arrive == 0: nothing arrives; the wait gives up after `polls` polls and the
 * kernel reports it (*gave_up = 1), leaving the context usable.  *ms (optional): the launch's duration.
 * No reference counterpart. */
int qcg_selftest_bounded_wait(long long polls, int arrive, int* gave_up, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* QCHEM_B200_H */
