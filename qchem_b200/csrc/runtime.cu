// runtime.cu -- the C ABI (include/qchem_b200.h): handle, basis upload, pair lists and Schwarz screening,
// the direct J/K build, Cartesian ERI batches, one-electron integrals and the RHF driver.
//
// Host-side work here is setup (once per geometry) and the SCF linear algebra; every integral and the
// whole J/K build run in the CUDA kernels.  There is no CPU fallback: without a usable device every
// entry point returns QCG_ERR_CUDA.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include <cublas_v2.h>
#include <cusolverDn.h>

#include "../../include/qchem_b200.h"
#include "eri_team_iface.h"
#include "md_core.cuh"
#include "qcg_internal.h"
#include "boys_table.h"

namespace qcg {
void launch_validate(const double* D, long long total, int n, const MolLayoutDev& ml, double tol, int* flag,
                     cudaStream_t st, int nsm);
void launch_symmetrize(const double* Jp, const double* Kp, double* J, double* K, long long total, int n,
                       const MolLayoutDev& ml, int* flag, cudaStream_t st, int nsm);
void launch_symmetrize_fixed(const double* Jp, const double* Kp, double* J, double* K, long long total, int n,
                             const MolLayoutDev& ml, int* flag, cudaStream_t st, int nsm);
void launch_one_electron(const BasisDev& bs, const int* f0, int n, int natom, const double* Z, const double* R,
                         double* S, double* T, double* V, const double* boys, cudaStream_t st, int nsm,
                         const int2* pairs = nullptr, long long npair_list = 0, const int* shell_mol = nullptr,
                         const MolLayoutDev& ml = MolLayoutDev{1, nullptr, nullptr}, const int* atom0 = nullptr,
                         const int* natoms = nullptr);
void launch_dfma_peak(double* out, int blocks, int threads, int iters, cudaStream_t st);
void launch_bounded_wait_selftest(long long polls, int arrive, int* err, cudaStream_t st);
void launch_ffma_peak(float* out, int blocks, int threads, int iters, cudaStream_t st);
}   // namespace qcg

using namespace qcg;

namespace {

struct Error
{
    int code;
    std::string msg;
};

#define CK(call)                                                                                                  \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) throw Error{QCG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};   \
    } while (0)

constexpr int kMaxL = 2;
const double kPi = 3.14159265358979323846;

int pair_class(int la, int lb)   // la >= lb
{
    return la * (la + 1) / 2 + lb;
}

// algorithmic FLOPs per primitive quartet (fixed per-class formula):
// (20+3L) + 2 sum_{j<=L} H(j) + 2 H(Lab) S(cd) + 2 nc nd S(ab) + 2 na nb nc nd
double class_flops(int la, int lb, int lc, int ld)
{
    auto H = [](int n) { return (n + 1) * (n + 2) * (n + 3) / 6; };
    auto comps = [](int L) {
        std::vector<std::array<int, 3>> c;
        for (int m = 0; m <= L; ++m)
            for (int l = 0; l <= L - m; ++l) c.push_back({L - m - l, l, m});
        return c;
    };
    auto S = [&](int l1, int l2) {
        long t = 0;
        for (auto a : comps(l1))
            for (auto b : comps(l2)) t += (long)(a[0] + b[0] + 1) * (a[1] + b[1] + 1) * (a[2] + b[2] + 1);
        return (double)t;
    };
    const int L = la + lb + lc + ld;
    double f = 20 + 3 * L;
    for (int j = 0; j <= L; ++j) f += 2 * H(j);
    f += 2.0 * H(la + lb) * S(lc, ld) + 2.0 * ncart(lc) * ncart(ld) * S(la, lb) +
         2.0 * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    return f;
}

struct DevBuf
{
    void* p = nullptr;
    size_t bytes = 0;
};

// Idle resources of destroyed handles, kept for the next handle on the same device: device slabs, pinned
// staging buffers, non-blocking streams and events.  Creating and destroying these costs milliseconds per
// handle (cudaFree and cudaFreeHost synchronise the device), which is a third of a 57-function RHF; a
// process that runs many small SCFs pays it once.  A handle hands its resources back only after
// synchronising its streams, so nothing in the cache has work in flight.  qcg_release_cache frees the
// cache; the cache object itself is never destroyed, so nothing is freed after the CUDA runtime is torn
// down at exit.
class ResourceCache
{
public:
    static constexpr size_t kSlab = 8u << 20, kStage = 4u << 20;
    static ResourceCache& get()
    {
        static ResourceCache* c = new ResourceCache;
        return *c;
    }
    void* slab(int dev)
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            auto& v = per_[dev].slabs;
            if (!v.empty())
            {
                void* p = v.back();
                v.pop_back();
                return p;
            }
        }
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, kSlab);
        if (e != cudaSuccess) throw Error{QCG_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
        return p;
    }
    char* stage()
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (!stages_.empty())
            {
                char* p = stages_.back();
                stages_.pop_back();
                return p;
            }
        }
        char* p = nullptr;
        CK(cudaMallocHost(&p, kStage));
        return p;
    }
    cudaStream_t stream(int dev)
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            auto& v = per_[dev].streams;
            if (!v.empty())
            {
                cudaStream_t s = v.back();
                v.pop_back();
                return s;
            }
        }
        cudaStream_t s = nullptr;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        return s;
    }
    // timing: an event that can time (cudaEventElapsedTime); otherwise created with cudaEventDisableTiming
    cudaEvent_t event(int dev, bool timing)
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            auto& v = timing ? per_[dev].tevents : per_[dev].sevents;
            if (!v.empty())
            {
                cudaEvent_t e = v.back();
                v.pop_back();
                return e;
            }
        }
        cudaEvent_t e = nullptr;
        CK(timing ? cudaEventCreate(&e) : cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        return e;
    }
    // pinned host blocks of at least `bytes` (capacities are powers of two from 1 MiB; *cap receives it)
    char* pinned(size_t bytes, size_t* cap)
    {
        size_t c = (size_t)1 << 20;
        while (c < bytes) c <<= 1;
        *cap = c;
        {
            std::lock_guard<std::mutex> g(mu_);
            auto it = pinned_.find(c);
            if (it != pinned_.end())
            {
                char* p = it->second;
                pinned_.erase(it);
                return p;
            }
        }
        char* p = nullptr;
        CK(cudaMallocHost(&p, c));
        return p;
    }
    void give_pinned(char* p, size_t cap)
    {
        std::lock_guard<std::mutex> g(mu_);
        pinned_.emplace(cap, p);
    }
    void give_slab(int dev, void* p)
    {
        std::lock_guard<std::mutex> g(mu_);
        per_[dev].slabs.push_back(p);
    }
    void give_stage(char* p)
    {
        std::lock_guard<std::mutex> g(mu_);
        stages_.push_back(p);
    }
    void give_stream(int dev, cudaStream_t s)
    {
        std::lock_guard<std::mutex> g(mu_);
        per_[dev].streams.push_back(s);
    }
    void give_event(int dev, cudaEvent_t e, bool timing)
    {
        std::lock_guard<std::mutex> g(mu_);
        (timing ? per_[dev].tevents : per_[dev].sevents).push_back(e);
    }
    // frees everything idle (resources of live handles are not in the cache)
    void release_all()
    {
        std::lock_guard<std::mutex> g(mu_);
        int cur = 0;
        cudaGetDevice(&cur);
        for (auto& kv : per_)
        {
            cudaSetDevice(kv.first);
            for (void* p : kv.second.slabs) cudaFree(p);
            for (cudaStream_t s : kv.second.streams) cudaStreamDestroy(s);
            for (cudaEvent_t e : kv.second.tevents) cudaEventDestroy(e);
            for (cudaEvent_t e : kv.second.sevents) cudaEventDestroy(e);
        }
        per_.clear();
        cudaSetDevice(cur);
        for (char* p : stages_) cudaFreeHost(p);
        stages_.clear();
        for (auto& kv : pinned_) cudaFreeHost(kv.second);
        pinned_.clear();
    }

private:
    struct PerDevice
    {
        std::vector<void*> slabs;
        std::vector<cudaStream_t> streams;
        std::vector<cudaEvent_t> tevents, sevents;
    };
    std::mutex mu_;
    std::unordered_map<int, PerDevice> per_;
    std::vector<char*> stages_;
    std::unordered_multimap<size_t, char*> pinned_;
};

// a pinned host array from the resource cache for the lifetime of one call
struct PinnedArray
{
    double* p = nullptr;
    size_t cap = 0;
    explicit PinnedArray(size_t n) { p = (double*)ResourceCache::get().pinned(std::max<size_t>(n, 1) * sizeof(double), &cap); }
    ~PinnedArray() { ResourceCache::get().give_pinned((char*)p, cap); }
    PinnedArray(const PinnedArray&) = delete;
    PinnedArray& operator=(const PinnedArray&) = delete;
};

}   // namespace

// arguments that identify a J/K build for graph replay
struct QcgGraphKey
{
    const void* D = nullptr;
    const void* J = nullptr;
    const void* K = nullptr;
    const void* dmax = nullptr;
    double dthr = -1, band = -1;
    int gen = -1;
    bool operator==(const QcgGraphKey& o) const
    {
        return D == o.D && J == o.J && K == o.K && dmax == o.dmax && dthr == o.dthr && band == o.band && gen == o.gen;
    }
};

struct qcg_handle
{
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    std::string last_error;
    long long mem_limit = 0, mem_used = 0;
    std::vector<DevBuf> allocs;

    // basis (host)
    int nshell = 0, nbf = 0;
    // several molecules in one handle (qcg_basis_create_batch): shells grouped by molecule, f0 local to the
    // molecule, every matrix packed as the molecules' n_m x n_m blocks one after the other
    int nmol = 1;
    std::vector<int> shell_mol, mol_shell0, mol_nbf;
    std::vector<long long> mol_off;
    long long packed = 0;   // elements of one matrix
    int* d_shell_mol = nullptr;
    long long* d_mol_off = nullptr;
    int* d_mol_n = nullptr;
    const int* d_mol_active = nullptr;   // set by the batched SCF while it runs: molecules still iterating
    MolLayoutDev mols() const { return MolLayoutDev{nmol, d_mol_off, d_mol_n}; }
    std::vector<int> L, nprim, prim0, f0;
    std::vector<double> cen, alpha, coef, ns;

    // basis (device)
    BasisDev bs{};
    double* d_boys = nullptr;
    int* d_f0 = nullptr;

    // pair lists and screening
    bool screened = false;
    double thresh = 0;
    std::vector<int> pl_sa[kNumPairClasses], pl_sb[kNumPairClasses], pl_ppo[kNumPairClasses], pl_npp[kNumPairClasses],
        pl_mol[kNumPairClasses];
    std::vector<double> pl_Q[kNumPairClasses];
    PairListDev pl_dev[kNumPairClasses]{};
    PrimPairsDev pp_dev{};
    JKWorkDev work[kNumQuartetClasses]{};
    // host copies of the work lists for the shard boundaries: per class, the quartet offsets and ket bases
    // of the bra pairs and the prefix sums of their primitive quartets; per pair class, the prefix sums of
    // the primitive-pair counts
    std::vector<long long> wh_offs[kNumQuartetClasses], wh_cum[kNumQuartetClasses];
    std::vector<int> wh_kbase[kNumQuartetClasses];
    std::vector<long long> pl_nppsum[kNumPairClasses];
    // the warp-shared J/K form (jk_warp_kernel), per class, built on first use after each screening: bra pairs
    // grouped by first shell and the work items over them
    int* d_wgbra[kNumQuartetClasses] = {};
    int4* d_witems[kNumQuartetClasses] = {};
    long long nwitems[kNumQuartetClasses] = {};
    bool witems_ready[kNumQuartetClasses] = {};
    long long jk_warp_mask = -1;   // qcg_set_jk_warp_classes; -1: the process default
    double fp32_below = 0;   // qcg_set_fp32_bound: quartets with a smaller bound are evaluated in FP32
    int shard_rank = 0, shard_world = 1;   // qcg_set_shard: this handle's slice of every J/K build
    std::shared_ptr<void> sph;             // the spherical map, built on first use
    std::shared_ptr<void> salc;            // cuBLAS handle and buffers of the symmetry-adapted faces
    int tuned_run[kNumQuartetClasses] = {}, tuned_cap[kNumQuartetClasses] = {};   // qcg_autotune_jk (0: default)
    double* d_dmaxD = nullptr;   // per shell-pair max |D| of a full build's density (mixed precision)
    long long work_quartets = 0, work_prim_quartets = 0;
    double work_flops = 0;
    std::vector<double> Qfull;

    // ERI-batch scratch: contraction-pattern keys, bucket counters and the visiting order (grow only)
    long long sort_cap = 0;
    unsigned char* d_key = nullptr;
    int *d_order = nullptr, *d_hist = nullptr, *d_cursor = nullptr;

    // team-form ERI batches (eri_team.cu): per-CTA R cache and recurrence scratch (grow only), error word
    double* d_team = nullptr;
    long long team_cap = 0;   // doubles
    int* d_team_err = nullptr;
    bool team_pending = false;   // a team kernel ran since the error word was last read
    unsigned char* d_pmask = nullptr;   // qcg_set_pair_subset (null: every quartet)
    int maxnp[kMaxL + 1] = {};   // largest contraction length per angular momentum (0: not yet computed)

    // host-buffer ERI batches: two quartet/output buffer pairs (grow only) and a copy-out stream
    void* hb_q[2] = {nullptr, nullptr};
    void* hb_out[2] = {nullptr, nullptr};
    size_t hb_qcap[2] = {0, 0}, hb_ocap[2] = {0, 0};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t hb_done[2] = {nullptr, nullptr}, hb_free[2] = {nullptr, nullptr};

    // J/K buffers
    double *d_D = nullptr, *d_Jp = nullptr, *d_Kp = nullptr, *d_J = nullptr, *d_K = nullptr;
    int* d_flag = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    // side streams for the class kernels of one build (fork after the accumulators are zeroed, join before
    // the symmetrisation), so that classes with few quartets run side by side
    static constexpr int kSide = 6;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr, join[kSide] = {};
    // J/K builds replayed as CUDA graphs, keyed by their arguments and the screening generation
    bool use_graphs = false;
    long long team_mask = -1;      // qcg_set_eri_team_classes; -1: the process default (eri_team_mask)
    long long jk_team_mask = -1;   // qcg_set_jk_team_classes; -1: the process default (jk_team_mask)
    int screen_gen = 0;
    QcgGraphKey last_key{};
    std::vector<std::pair<QcgGraphKey, cudaGraphExec_t>> graphs;
    void drop_graphs()
    {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        graphs.clear();
        last_key = QcgGraphKey{};
    }

    // Small buffers (pair lists, work offsets, basis arrays: a few hundred per handle) are carved out of
    // 8 MiB slabs, so that setting up and destroying a handle costs a handful of cudaMalloc/cudaFree
    // calls instead of hundreds; releasing a slab piece is a no-op until the handle goes.  Larger buffers
    // have their own allocation.
    static constexpr size_t kSlab = ResourceCache::kSlab, kSmallMax = 1u << 20;
    std::vector<DevBuf> slabs;
    size_t slab_used = kSlab;
    // pinned staging for uploads of host vectors (asynchronous copies; reused after a stream sync)
    static constexpr size_t kStage = ResourceCache::kStage;
    char* stage = nullptr;
    size_t stage_used = 0;

    // slab pieces in use (pointer -> bytes) and released pieces kept for reuse by size
    std::unordered_map<void*, size_t> small_live;
    std::unordered_multimap<size_t, void*> small_free;

    void* raw_alloc(size_t bytes)
    {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) throw Error{QCG_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
        return p;
    }
    // mem_used counts the bytes handed out (the limit applies to those, not to slab capacity)
    template <class T>
    T* alloc(size_t count)
    {
        const size_t bytes = (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~(size_t)255;
        if (mem_limit > 0 && mem_used + (long long)bytes > mem_limit)
            throw Error{QCG_ERR_ALLOC, "device memory limit of " + std::to_string(mem_limit) + " bytes exceeded"};
        void* p = nullptr;
        if (bytes <= kSmallMax)
        {
            auto it = small_free.find(bytes);
            if (it != small_free.end())
            {
                p = it->second;
                small_free.erase(it);
            }
            else
            {
                if (slab_used + bytes > kSlab)
                {
                    slabs.push_back({ResourceCache::get().slab(device), kSlab});
                    slab_used = 0;
                }
                p = (char*)slabs.back().p + slab_used;
                slab_used += bytes;
            }
            small_live[p] = bytes;
        }
        else
        {
            p = raw_alloc(bytes);
            allocs.push_back({p, bytes});
        }
        mem_used += bytes;
        return (T*)p;
    }
    void release(void* p)
    {
        auto it = small_live.find(p);
        if (it != small_live.end())
        {
            mem_used -= it->second;
            small_free.emplace(it->second, p);
            small_live.erase(it);
            return;
        }
        for (size_t i = 0; i < allocs.size(); ++i)
            if (allocs[i].p == p)
            {
                cudaFree(p);
                mem_used -= allocs[i].bytes;
                allocs.erase(allocs.begin() + i);
                return;
            }
    }
    // Uploads between begin_uploads() and flush_uploads() are merged: a piece whose device address and
    // staging offset both continue the previous piece (consecutive slab allocations do) extends one pending
    // copy, so a run of small uploads costs one cudaMemcpyAsync.  Nothing queued on the stream may read an
    // uploaded array before the flush.
    bool defer_uploads = false;
    char* pend_dev = nullptr;
    char* pend_stage = nullptr;
    size_t pend_span = 0;
    void begin_uploads() { defer_uploads = true; }
    void flush_uploads()
    {
        if (pend_span) CK(cudaMemcpyAsync(pend_dev, pend_stage, pend_span, cudaMemcpyHostToDevice, stream));
        pend_span = 0;
        defer_uploads = false;
    }
    template <class T>
    T* upload(const std::vector<T>& v)
    {
        T* d = alloc<T>(v.size());
        const size_t bytes = v.size() * sizeof(T);
        if (bytes == 0) return d;
        const size_t span = (bytes + 255) & ~(size_t)255;   // the allocation's extent (alloc rounds to 256)
        if (bytes > kStage)
        {
            if (pend_span) CK(cudaMemcpyAsync(pend_dev, pend_stage, pend_span, cudaMemcpyHostToDevice, stream));
            pend_span = 0;
            CK(cudaMemcpyAsync(d, v.data(), bytes, cudaMemcpyHostToDevice, stream));
            return d;
        }
        if (!stage)
        {
            stage = ResourceCache::get().stage();
            stage_used = 0;
        }
        if (stage_used + span > kStage)
        {
            if (pend_span) CK(cudaMemcpyAsync(pend_dev, pend_stage, pend_span, cudaMemcpyHostToDevice, stream));
            pend_span = 0;
            CK(cudaStreamSynchronize(stream));   // earlier copies out of the staging buffer are done
            stage_used = 0;
        }
        char* src = stage + stage_used;
        std::memcpy(src, v.data(), bytes);
        stage_used += span;
        if (!defer_uploads)
        {
            CK(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, stream));
            return d;
        }
        if (pend_span && (char*)d == pend_dev + pend_span && src == pend_stage + pend_span)
        {
            pend_span += span;
            return d;
        }
        if (pend_span) CK(cudaMemcpyAsync(pend_dev, pend_stage, pend_span, cudaMemcpyHostToDevice, stream));
        pend_dev = (char*)d;
        pend_stage = src;
        pend_span = span;
        return d;
    }
    // streams and events come from the process-wide cache and go back to it, idle, when the handle goes
    cudaStream_t new_stream() { return ResourceCache::get().stream(device); }
    cudaEvent_t new_event(bool timing) { return ResourceCache::get().event(device, timing); }
    ~qcg_handle()
    {
        if (stream) cudaStreamSynchronize(stream);
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        for (int k = 0; k < kSide; ++k)
            if (side[k]) cudaStreamSynchronize(side[k]);
        if (own_stream) cudaStreamSynchronize(own_stream);
        drop_graphs();
        for (auto& a : allocs) cudaFree(a.p);
        // a handle whose context failed gives nothing back: its resources may be unusable
        const bool healthy = cudaGetLastError() == cudaSuccess;
        auto& rc = ResourceCache::get();
        auto give_event = [&](cudaEvent_t e, bool timing) {
            if (!e) return;
            if (healthy) rc.give_event(device, e, timing);
            else cudaEventDestroy(e);
        };
        auto give_stream = [&](cudaStream_t s) {
            if (!s) return;
            if (healthy) rc.give_stream(device, s);
            else cudaStreamDestroy(s);
        };
        for (auto& a : slabs)
        {
            if (healthy) rc.give_slab(device, a.p);
            else cudaFree(a.p);
        }
        if (stage)
        {
            if (healthy) rc.give_stage(stage);
            else cudaFreeHost(stage);
        }
        give_event(ev0, true);
        give_event(ev1, true);
        give_event(ev2, true);
        give_event(fork, false);
        for (int k = 0; k < 2; ++k)
        {
            give_event(hb_done[k], false);
            give_event(hb_free[k], false);
        }
        give_stream(copy_stream);
        for (int k = 0; k < kSide; ++k)
        {
            give_event(join[k], false);
            give_stream(side[k]);
        }
        give_stream(own_stream);
    }
};

namespace {

template <class F>
int guarded(qcg_handle* h, F&& f)
{
    try
    {
        f();
        if (h) h->last_error.clear();
        return QCG_OK;
    }
    catch (const Error& e)
    {
        if (h) h->last_error = e.msg;
        return e.code;
    }
    catch (const std::exception& e)
    {
        if (h) h->last_error = e.what();
        return QCG_ERR_ARG;
    }
}

void require(bool ok, const std::string& msg, int code = QCG_ERR_ARG)
{
    if (!ok) throw Error{code, msg};
}

double dfact(int i)
{
    double r = 1;
    for (int k = i; k > 1; k -= 2) r *= k;
    return r;
}

// GetNormalization(Polarization(L,0,0)) of one primitive (PG_Cart_MnD/Imp/GaussianRF.C:512-521)
double prim_norm(double a, int L)
{
    const double s = std::pow(kPi / (2 * a), 1.5);
    return std::sqrt(std::pow(4 * a, L) / (s * dfact(2 * L - 1)));
}

// ------------------------------------------------------------------------------------------------
// Symmetric eigensolver, A = V diag(w) V^T with ascending w (row-major n x n):
//   1. Householder reduction to tridiagonal T = Q^T A Q, one reflector per column,
//   2. implicit symmetric QR steps with a Wilkinson shift on T (bulge chasing with Givens rotations),
//      rotations accumulated into V = Q G_1^T G_2^T ...
// The accumulated matrix is kept transposed (Qt[k][r] = Q[r][k]) so that both the reflectors and the
// rotations of a sweep update contiguous rows: a sweep is applied to blocks of 32 columns of Qt at a time,
// each block walking the whole rotation chain with its running row in registers.
// ------------------------------------------------------------------------------------------------
void syev(int n, const double* Ain, double* w, double* V)
{
    std::vector<double> T(Ain, Ain + (size_t)n * n), Qt((size_t)n * n, 0.0), v(n), pv(n), wv(n), sr(n);
    auto t = [&](int i, int j) -> double& { return T[(size_t)i * n + j]; };
    auto qt = [&](int k, int r) -> double* { return Qt.data() + (size_t)k * n + r; };
    for (int i = 0; i < n; ++i) *qt(i, i) = 1.0;
    const bool par = n >= 192;
    for (int k = 0; k + 2 < n; ++k)
    {
        // reflector H = I - beta v v^T mapping x = T[k+1:, k] onto alpha e_1
        double xn = 0.0;
        for (int i = k + 1; i < n; ++i) xn += t(i, k) * t(i, k);
        xn = std::sqrt(xn);
        if (xn == 0.0) continue;
        const double alpha = t(k + 1, k) > 0 ? -xn : xn;
        for (int i = k + 1; i < n; ++i) v[i] = t(i, k);
        v[k + 1] -= alpha;
        double vv = 0.0;
        for (int i = k + 1; i < n; ++i) vv += v[i] * v[i];
        if (vv == 0.0) continue;
        const double beta = 2.0 / vv;
        // trailing block update: A <- A - v w^T - w v^T with p = beta A v, w = p - (beta p.v / 2) v
        auto matvec_row = [&](int i) {
            const double* ti = &t(i, 0);
            double s = 0.0;
#pragma omp simd reduction(+ : s)
            for (int j = k + 1; j < n; ++j) s += ti[j] * v[j];
            pv[i] = beta * s;
        };
        // small problems stay out of the OpenMP runtime (entering a region costs about as much as a row)
        if (par && n - k > 96)
        {
#pragma omp parallel for schedule(static)
            for (int i = k + 1; i < n; ++i) matvec_row(i);
        }
        else
            for (int i = k + 1; i < n; ++i) matvec_row(i);
        double pdv = 0.0;
        for (int i = k + 1; i < n; ++i) pdv += pv[i] * v[i];
        for (int i = k + 1; i < n; ++i) wv[i] = pv[i] - 0.5 * beta * pdv * v[i];
        auto update_row = [&](int i) {
            double* ti = &t(i, 0);
            const double vi = v[i], wi = wv[i];
            for (int j = k + 1; j < n; ++j) ti[j] -= vi * wv[j] + wi * v[j];
        };
        if (par && n - k > 96)
        {
#pragma omp parallel for schedule(static)
            for (int i = k + 1; i < n; ++i) update_row(i);
        }
        else
            for (int i = k + 1; i < n; ++i) update_row(i);
        t(k + 1, k) = t(k, k + 1) = alpha;
        for (int i = k + 2; i < n; ++i) t(i, k) = t(k, i) = 0.0;
        // Q <- Q H, i.e. Qt <- H Qt: s_r = sum_i v_i Qt[i][r], Qt[j][r] -= beta v_j s_r
        std::fill(sr.begin(), sr.end(), 0.0);
        for (int i = k + 1; i < n; ++i)
        {
            const double vi = v[i];
            const double* qi = qt(i, 0);
            for (int r = 0; r < n; ++r) sr[r] += vi * qi[r];
        }
        auto q_row = [&](int j) {
            double* qj = qt(j, 0);
            const double f = beta * v[j];
            for (int r = 0; r < n; ++r) qj[r] -= f * sr[r];
        };
        if (par)
        {
#pragma omp parallel for schedule(static)
            for (int j = k + 1; j < n; ++j) q_row(j);
        }
        else
            for (int j = k + 1; j < n; ++j) q_row(j);
    }
    // rotation G on (k,k+1): T <- G T G^T, G = [[c, s], [-s, c]]; the matching Qt <- G Qt updates of one
    // sweep are recorded and applied afterwards
    std::vector<double> rc(n), rs(n);
    auto rotate = [&](int k, double c, double s, int lo, int hi) {
        for (int j = lo; j <= hi; ++j)
        {
            const double a = t(k, j), b = t(k + 1, j);
            t(k, j) = c * a + s * b;
            t(k + 1, j) = -s * a + c * b;
        }
        for (int i = lo; i <= hi; ++i)
        {
            const double a = t(i, k), b = t(i, k + 1);
            t(i, k) = c * a + s * b;
            t(i, k + 1) = -s * a + c * b;
        }
        rc[k] = c;
        rs[k] = s;
    };
    constexpr int RB = 32;
    const int nblk = (n + RB - 1) / RB;
    auto apply_sweep = [&](int l, int m) {
        auto block = [&](int blk) {
            const int r0 = blk * RB, nr = std::min(RB, n - r0);
            double a[RB];
            const double* ql = qt(l, r0);
            for (int r = 0; r < nr; ++r) a[r] = ql[r];
            for (int k = l; k < m; ++k)
            {
                double* qk = qt(k, r0);
                const double* qk1 = qt(k + 1, r0);
                const double c = rc[k], s = rs[k];
                for (int r = 0; r < nr; ++r)
                {
                    const double b = qk1[r];
                    qk[r] = c * a[r] + s * b;
                    a[r] = -s * a[r] + c * b;
                }
            }
            double* qm = qt(m, r0);
            for (int r = 0; r < nr; ++r) qm[r] = a[r];
        };
        if (par && m - l > 32)
        {
#pragma omp parallel for schedule(static)
            for (int blk = 0; blk < nblk; ++blk) block(blk);
        }
        else
            for (int blk = 0; blk < nblk; ++blk) block(blk);
    };
    const double eps = 1e-15;
    int m = n - 1, steps = 0;
    while (m > 0)
    {
        if (std::fabs(t(m, m - 1)) <= eps * (std::fabs(t(m, m)) + std::fabs(t(m - 1, m - 1))))
        {
            t(m, m - 1) = t(m - 1, m) = 0.0;
            --m;
            continue;
        }
        int l = m - 1;
        while (l > 0 && std::fabs(t(l, l - 1)) > eps * (std::fabs(t(l, l)) + std::fabs(t(l - 1, l - 1)))) --l;
        if (++steps > 60 * n) throw Error{QCG_ERR_NOCONV, "eigensolver did not converge"};
        // Wilkinson shift from the trailing 2x2 of the block
        const double a = t(m - 1, m - 1), b = t(m, m - 1), c2 = t(m, m);
        const double delta = 0.5 * (a - c2);
        const double mu = delta == 0.0 ? c2 - std::fabs(b)
                                       : c2 - b * b / (delta + (delta > 0 ? 1.0 : -1.0) * std::hypot(delta, b));
        double x = t(l, l) - mu, z = t(l + 1, l);
        for (int k = l; k < m; ++k)
        {
            const double r = std::sqrt(x * x + z * z);
            const double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : z / r;
            rotate(k, c, s, std::max(l, k - 1), std::min(m, k + 2));
            if (k + 1 < m)
            {
                x = t(k + 1, k);
                z = t(k + 2, k);
            }
        }
        apply_sweep(l, m);
    }
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return t(x, x) < t(y, y); });
    for (int j = 0; j < n; ++j)
    {
        w[j] = t(idx[j], idx[j]);
        const double* qj = qt(idx[j], 0);
        for (int r = 0; r < n; ++r) V[(size_t)r * n + j] = qj[r];
    }
}

// The lowest k eigenpairs of a symmetric n x n matrix: the k lowest eigenvalues in w[0..k) (ascending)
// and their eigenvectors in the first k columns of V (row-major n x n; the other columns are left as they
// are).  The SCF step needs only the occupied orbitals, so this skips the O(n^3) parts of syev that
// produce the rest: forming Q and accumulating the QR rotations into it.
//   1. Householder reduction T = Q^T A Q, Q = H_0 H_1 ... H_{n-3}, keeping the reflectors (v_j, beta_j);
//   2. the k lowest eigenvalues of T by bisection on Sturm counts (negative pivots of T - x I = L D L^T),
//      refined to the Rayleigh quotients of the vectors of step 3;
//   3. eigenvectors x of T by inverse iteration (tridiagonal LU with partial pivoting, three solves from a
//      fixed start vector), re-orthogonalised by modified Gram-Schmidt inside clusters of eigenvalues
//      closer than 1e-3 ||T||, with equal eigenvalues pulled apart by 10 eps ||T|| (the scheme of
//      LAPACK's stein);
//   4. v = H_0 (H_1 (... (H_{n-3} x))).
// Each vector's tridiagonal residual and the vectors' orthonormality are checked; if either is off by
// more than 1e-10 relative, the full solver runs instead.
void syev_lowest(int n, const double* Ain, int k, double* w, double* V)
{
    if (k >= n || n < 3 || k <= 0)
    {
        std::vector<double> wa(n), Va((size_t)n * n);
        syev(n, Ain, wa.data(), Va.data());
        const int kk = std::min(std::max(k, 0), n);
        for (int j = 0; j < kk; ++j) w[j] = wa[j];
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < kk; ++j) V[(size_t)i * n + j] = Va[(size_t)i * n + j];
        return;
    }
    std::vector<double> T(Ain, Ain + (size_t)n * n), R((size_t)n * n, 0.0), beta(n, 0.0), v(n), pv(n), wv(n);
    auto t = [&](int i, int j) -> double& { return T[(size_t)i * n + j]; };
    const bool par = n >= 192;
    for (int j = 0; j + 2 < n; ++j)
    {
        double xn = 0.0;
        for (int i = j + 1; i < n; ++i) xn += t(i, j) * t(i, j);
        xn = std::sqrt(xn);
        if (xn == 0.0) continue;
        const double alpha = t(j + 1, j) > 0 ? -xn : xn;
        for (int i = j + 1; i < n; ++i) v[i] = t(i, j);
        v[j + 1] -= alpha;
        double vv = 0.0;
        for (int i = j + 1; i < n; ++i) vv += v[i] * v[i];
        if (vv == 0.0) continue;
        const double b = 2.0 / vv;
        auto matvec_row = [&](int i) {
            const double* ti = &t(i, 0);
            double s = 0.0;
#pragma omp simd reduction(+ : s)
            for (int c = j + 1; c < n; ++c) s += ti[c] * v[c];
            pv[i] = b * s;
        };
        // small problems stay out of the OpenMP runtime: entering a parallel region, even one whose if
        // clause is false, costs about as much as a row of this size
        if (par && n - j > 96)
        {
#pragma omp parallel for schedule(static)
            for (int i = j + 1; i < n; ++i) matvec_row(i);
        }
        else
            for (int i = j + 1; i < n; ++i) matvec_row(i);
        double pdv = 0.0;
        for (int i = j + 1; i < n; ++i) pdv += pv[i] * v[i];
        for (int i = j + 1; i < n; ++i) wv[i] = pv[i] - 0.5 * b * pdv * v[i];
        auto update_row = [&](int i) {
            double* ti = &t(i, 0);
            const double vi = v[i], wi = wv[i];
            for (int c = j + 1; c < n; ++c) ti[c] -= vi * wv[c] + wi * v[c];
        };
        if (par && n - j > 96)
        {
#pragma omp parallel for schedule(static)
            for (int i = j + 1; i < n; ++i) update_row(i);
        }
        else
            for (int i = j + 1; i < n; ++i) update_row(i);
        t(j + 1, j) = t(j, j + 1) = alpha;
        for (int i = j + 2; i < n; ++i) t(i, j) = t(j, i) = 0.0;
        for (int i = j + 1; i < n; ++i) R[(size_t)j * n + i] = v[i];
        beta[j] = b;
    }
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = t(i, i);
    for (int i = 0; i + 1 < n; ++i) e[i] = t(i + 1, i);
    double tnorm = 0.0, glo = HUGE_VAL, ghi = -HUGE_VAL, emax2 = 0.0;
    for (int i = 0; i < n; ++i)
    {
        const double r = std::fabs(e[i]) + (i > 0 ? std::fabs(e[i - 1]) : 0.0);
        tnorm = std::max(tnorm, std::fabs(d[i]) + r);
        glo = std::min(glo, d[i] - r);
        ghi = std::max(ghi, d[i] + r);
        emax2 = std::max(emax2, e[i] * e[i]);
    }
    const double ulp = 2.220446049250313e-16;
    // the k lowest eigenvalues: bisection inside the Gershgorin interval on the count of eigenvalues below x
    const double pivmin = std::max(1e-300, 4.0 * ulp * ulp * std::max(emax2, 1e-300));
    auto count_below = [&](double x) {
        int cnt = 0;
        double q = d[0] - x;
        if (std::fabs(q) < pivmin) q = -pivmin;
        if (q < 0) ++cnt;
        for (int i = 1; i < n; ++i)
        {
            q = (d[i] - x) - e[i - 1] * e[i - 1] / q;
            if (std::fabs(q) < pivmin) q = -pivmin;
            if (q < 0) ++cnt;
        }
        return cnt;
    };
    const double pad = 2.0 * ulp * std::max(tnorm, 1e-300) + pivmin;
    glo -= pad;
    ghi += pad;
    // all k intervals are bisected together: the Sturm recurrence is a chain of dependent divisions, and k
    // interleaved chains keep the divider busy.  Intervals stop at 1e-12 ||T||; the final eigenvalues are
    // the Rayleigh quotients of the inverse-iteration vectors below.
    {
        std::vector<double> ba(k, glo), bb(k, ghi), mid(k), q(k);
        std::vector<int> cnt(k);
        const double tol = 1e-12 * std::max(tnorm, 1e-300) + pivmin;
        for (int it = 0; it < 200; ++it)
        {
            bool open = false;
            for (int j = 0; j < k; ++j)
            {
                mid[j] = 0.5 * (ba[j] + bb[j]);
                open = open || (bb[j] - ba[j] > tol && mid[j] > ba[j] && mid[j] < bb[j]);
            }
            if (!open) break;
            for (int j = 0; j < k; ++j)
            {
                q[j] = d[0] - mid[j];
                if (std::fabs(q[j]) < pivmin) q[j] = -pivmin;
                cnt[j] = q[j] < 0 ? 1 : 0;
            }
            for (int i = 1; i < n; ++i)
            {
                const double di = d[i], e2 = e[i - 1] * e[i - 1];
                for (int j = 0; j < k; ++j)
                {
                    double qq = (di - mid[j]) - e2 / q[j];
                    if (std::fabs(qq) < pivmin) qq = -pivmin;
                    q[j] = qq;
                    cnt[j] += qq < 0 ? 1 : 0;
                }
            }
            for (int j = 0; j < k; ++j)
            {
                if (cnt[j] > j) bb[j] = mid[j];
                else ba[j] = mid[j];
            }
        }
        for (int j = 0; j < k; ++j) w[j] = 0.5 * (ba[j] + bb[j]);
    }
    // inverse iteration on the tridiagonal (d, e)
    const double sep = 10.0 * ulp * tnorm, ortol = 1e-3 * tnorm;
    std::vector<double> X((size_t)k * n), u0(n), u1(n), u2(n), mult(n), y(n);
    std::vector<char> swp(n);
    double sigma_prev = 0.0;
    int j0 = 0;
    for (int j = 0; j < k; ++j)
    {
        double sigma = w[j];
        if (j == 0 || w[j] - w[j - 1] > ortol) j0 = j;
        else if (sigma - sigma_prev < sep) sigma = sigma_prev + sep;
        sigma_prev = sigma;
        // LU of T - sigma I with partial pivoting: row i of U holds u0 (diagonal), u1, u2 (two above)
        double a = d[0] - sigma, b = e[0], c = 0.0;
        for (int i = 0; i + 1 < n; ++i)
        {
            const double ra = e[i], rb = d[i + 1] - sigma, rc = i + 2 < n ? e[i + 1] : 0.0;
            if (std::fabs(ra) > std::fabs(a))
            {
                swp[i] = 1;
                u0[i] = ra; u1[i] = rb; u2[i] = rc;
                const double f = a / ra;
                mult[i] = f;
                a = b - f * rb;
                b = c - f * rc;
            }
            else
            {
                swp[i] = 0;
                u0[i] = a; u1[i] = b; u2[i] = c;
                const double f = a == 0.0 ? 0.0 : ra / a;
                mult[i] = f;
                a = rb - f * b;
                b = rc - f * c;
            }
            c = 0.0;
        }
        u0[n - 1] = a;
        for (int i = 0; i < n; ++i)
            if (std::fabs(u0[i]) < ulp * tnorm) u0[i] = u0[i] < 0 ? -ulp * tnorm : ulp * tnorm;
        double* xj = &X[(size_t)j * n];
        // fixed start vector with no special structure
        uint64_t st = 0x9E3779B97F4A7C15ULL * (uint64_t)(j + 1);
        for (int i = 0; i < n; ++i)
        {
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            xj[i] = (double)(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        }
        for (int it = 0; it < 3; ++it)
        {
            for (int i = 0; i < n; ++i) y[i] = xj[i];
            for (int i = 0; i + 1 < n; ++i)
            {
                if (swp[i]) std::swap(y[i], y[i + 1]);
                y[i + 1] -= mult[i] * y[i];
            }
            for (int i = n - 1; i >= 0; --i)
            {
                double s = y[i];
                if (i + 1 < n) s -= u1[i] * y[i + 1];
                if (i + 2 < n) s -= u2[i] * y[i + 2];
                y[i] = s / u0[i];
            }
            for (int p = j0; p < j; ++p)
            {
                const double* xp = &X[(size_t)p * n];
                double dot = 0.0;
                for (int i = 0; i < n; ++i) dot += xp[i] * y[i];
                for (int i = 0; i < n; ++i) y[i] -= dot * xp[i];
            }
            double nrm = 0.0;
            for (int i = 0; i < n; ++i) nrm += y[i] * y[i];
            nrm = std::sqrt(nrm);
            if (!(nrm > 0.0) || !std::isfinite(nrm)) break;
            for (int i = 0; i < n; ++i) xj[i] = y[i] / nrm;
        }
    }
    // eigenvalues: Rayleigh quotients x^T T x of the (unit) vectors
    for (int j = 0; j < k; ++j)
    {
        const double* xj = &X[(size_t)j * n];
        double rq = 0.0;
        for (int i = 0; i < n; ++i)
        {
            double tx = d[i] * xj[i];
            if (i > 0) tx += e[i - 1] * xj[i - 1];
            if (i + 1 < n) tx += e[i] * xj[i + 1];
            rq += xj[i] * tx;
        }
        w[j] = rq;
    }
    // self-check: tridiagonal residuals and orthonormality
    bool ok = true;
    for (int j = 0; j < k && ok; ++j)
    {
        const double* xj = &X[(size_t)j * n];
        double res = 0.0, nrm = 0.0;
        for (int i = 0; i < n; ++i)
        {
            double r = (d[i] - w[j]) * xj[i];
            if (i > 0) r += e[i - 1] * xj[i - 1];
            if (i + 1 < n) r += e[i] * xj[i + 1];
            res = std::max(res, std::fabs(r));
            nrm += xj[i] * xj[i];
        }
        ok = std::isfinite(res) && res <= 1e-10 * std::max(tnorm, 1e-300) && std::fabs(nrm - 1.0) <= 1e-10;
        for (int p = 0; p < j && ok; ++p)
        {
            double dot = 0.0;
            for (int i = 0; i < n; ++i) dot += X[(size_t)p * n + i] * xj[i];
            ok = std::fabs(dot) <= 1e-10;
        }
    }
    if (!ok)
    {
        std::vector<double> wa(n), Va((size_t)n * n);
        syev(n, Ain, wa.data(), Va.data());
        for (int j = 0; j < k; ++j) w[j] = wa[j];
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < k; ++j) V[(size_t)i * n + j] = Va[(size_t)i * n + j];
        return;
    }
    // back-transformation v = H_0 (... (H_{n-3} x))
    for (int j = 0; j < k; ++j)
    {
        double* xj = &X[(size_t)j * n];
        for (int q = n - 3; q >= 0; --q)
        {
            if (beta[q] == 0.0) continue;
            const double* rq = &R[(size_t)q * n];
            double s = 0.0;
#pragma omp simd reduction(+ : s)
            for (int i = q + 1; i < n; ++i) s += rq[i] * xj[i];
            s *= beta[q];
            for (int i = q + 1; i < n; ++i) xj[i] -= s * rq[i];
        }
        for (int i = 0; i < n; ++i) V[(size_t)i * n + j] = xj[i];
    }
}

// X = L^{-T} for the Cholesky factor S = L L^T of a symmetric positive definite S (row-major n x n):
// X is upper triangular with X^T S X = 1.  Returns false (X unspecified) if a pivot is not positive.
bool cholesky_orthogonaliser(int n, const double* S, double* X)
{
    std::vector<double> L((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j)
    {
        double dj = S[(size_t)j * n + j];
        const double* lj = &L[(size_t)j * n];
        for (int k = 0; k < j; ++k) dj -= lj[k] * lj[k];
        if (!(dj > 0.0)) return false;
        const double ljj = std::sqrt(dj);
        L[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i)
        {
            const double* li = &L[(size_t)i * n];
            double v = S[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) v -= li[k] * lj[k];
            L[(size_t)i * n + j] = v / ljj;
        }
    }
    // M = L^{-1} (lower triangular) by forward substitution, column by column; X = M^T
    std::vector<double> M((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c)
    {
        M[(size_t)c * n + c] = 1.0 / L[(size_t)c * n + c];
        for (int i = c + 1; i < n; ++i)
        {
            const double* li = &L[(size_t)i * n];
            double v = 0.0;
            for (int k = c; k < i; ++k) v -= li[k] * M[(size_t)k * n + c];
            M[(size_t)i * n + c] = v / li[i];
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) X[(size_t)i * n + j] = M[(size_t)j * n + i];
    return true;
}

// C = op(A) op(B), n x n, row-major
void gemm(int n, const double* A, bool ta, const double* B, bool tb, double* C)
{
    std::vector<double> At, Bt;
    const double* a = A;
    const double* b = B;
    if (ta)
    {
        At.resize((size_t)n * n);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) At[(size_t)i * n + j] = A[(size_t)j * n + i];
        a = At.data();
    }
    if (tb)
    {
        Bt.resize((size_t)n * n);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) Bt[(size_t)i * n + j] = B[(size_t)j * n + i];
        b = Bt.data();
    }
    // row i of C = sum_k a_ik (row k of b): contiguous rows, vectorisable without reassociation
    auto row = [&](int i) {
        double* ci = C + (size_t)i * n;
        const double* ai = a + (size_t)i * n;
        for (int j = 0; j < n; ++j) ci[j] = 0.0;
        for (int k = 0; k < n; ++k)
        {
            const double aik = ai[k];
            const double* bk = b + (size_t)k * n;
            for (int j = 0; j < n; ++j) ci[j] += aik * bk[j];
        }
    };
    if (n > 96)
    {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) row(i);
    }
    else
        for (int i = 0; i < n; ++i) row(i);
}

std::vector<double> solve_dense(int n, std::vector<double> A, std::vector<double> b)
{
    for (int c = 0; c < n; ++c)
    {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (piv != c)
        {
            for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[piv * n + k]);
            std::swap(b[c], b[piv]);
        }
        if (A[c * n + c] == 0.0) throw Error{QCG_ERR_NOCONV, "singular DIIS system"};
        for (int r = c + 1; r < n; ++r)
        {
            const double f = A[r * n + c] / A[c * n + c];
            for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
            b[r] -= f * b[c];
        }
    }
    std::vector<double> x(n);
    for (int r = n - 1; r >= 0; --r)
    {
        double s = b[r];
        for (int k = r + 1; k < n; ++k) s -= A[r * n + k] * x[k];
        x[r] = s / A[r * n + r];
    }
    return x;
}

// ------------------------------------------------------------------------------------------------
// Dense FP64 linear algebra of the SCF step on the GPU for large bases (cuSOLVER syevd, cuBLAS dgemm), in
// place of the host eigensolver and products above, whose O(n^3) cost at n ~ 2000 rivals the Fock build
// itself (LASolverLapack.C:126-145 is the reference's eigensolver call).  Host arrays in and out (row-major);
// device buffers and library handles are kept between calls.  Not thread-safe: one per SCF.
// ------------------------------------------------------------------------------------------------
struct GpuLinalg
{
    cudaStream_t st = nullptr;
    cusolverDnHandle_t sol = nullptr;
    cublasHandle_t blas = nullptr;
    double *dA = nullptr, *dB = nullptr, *dC = nullptr, *dW = nullptr, *dWork = nullptr;
    int* dInfo = nullptr;
    int cap = 0, lwork = 0;

    explicit GpuLinalg(cudaStream_t s) : st(s)
    {
        if (cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS) throw Error{QCG_ERR_CUDA, "cusolverDnCreate failed"};
        if (cublasCreate(&blas) != CUBLAS_STATUS_SUCCESS) throw Error{QCG_ERR_CUDA, "cublasCreate failed"};
        cusolverDnSetStream(sol, st);
        cublasSetStream(blas, st);
    }
    ~GpuLinalg()
    {
        if (st) cudaStreamSynchronize(st);
        for (void* p : {(void*)dA, (void*)dB, (void*)dC, (void*)dW, (void*)dWork, (void*)dInfo}) cudaFree(p);
        if (sol) cusolverDnDestroy(sol);
        if (blas) cublasDestroy(blas);
    }
    void reserve(int n)
    {
        if (n <= cap) return;
        for (double** p : {&dA, &dB, &dC, &dW}) { cudaFree(*p); *p = nullptr; }
        const size_t nn = (size_t)n * n;
        CK(cudaMalloc(&dA, nn * sizeof(double)));
        CK(cudaMalloc(&dB, nn * sizeof(double)));
        CK(cudaMalloc(&dC, nn * sizeof(double)));
        CK(cudaMalloc(&dW, (size_t)n * sizeof(double)));
        if (!dInfo) CK(cudaMalloc(&dInfo, sizeof(int)));
        int lw = 0;
        if (cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dA, n, dW, &lw) !=
            CUSOLVER_STATUS_SUCCESS)
            throw Error{QCG_ERR_CUDA, "cusolverDnDsyevd_bufferSize failed"};
        cudaFree(dWork);
        dWork = nullptr;
        CK(cudaMalloc(&dWork, (size_t)std::max(lw, 1) * sizeof(double)));
        lwork = lw;
        cap = n;
    }
    // A = V diag(w) V^T, w ascending, V row-major with eigenvectors as columns (as syev above)
    void syev(int n, const double* A, double* w, double* V)
    {
        reserve(n);
        const size_t nn = (size_t)n * n;
        CK(cudaMemcpyAsync(dA, A, nn * sizeof(double), cudaMemcpyHostToDevice, st));
        if (cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dA, n, dW, dWork, lwork,
                             dInfo) != CUSOLVER_STATUS_SUCCESS)
            throw Error{QCG_ERR_CUDA, "cusolverDnDsyevd failed"};
        // column-major result: eigenvector j is column j of dA; transpose to the row-major layout on the device
        const double one = 1.0, zero = 0.0;
        if (cublasDgeam(blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, &one, dA, n, &zero, dB, n, dB, n) != CUBLAS_STATUS_SUCCESS)
            throw Error{QCG_ERR_CUDA, "cublasDgeam failed"};
        int info = 0;
        CK(cudaMemcpyAsync(w, dW, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(V, dB, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&info, dInfo, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (info != 0) throw Error{QCG_ERR_NOCONV, "cusolverDnDsyevd did not converge"};
    }
    // C = op(A) op(B), n x n row-major (a row-major array is its transpose column-major, so the product is
    // computed as C^T = op(B)^T op(A)^T)
    void gemm(int n, const double* A, bool ta, const double* B, bool tb, double* C)
    {
        reserve(n);
        const size_t nn = (size_t)n * n;
        CK(cudaMemcpyAsync(dA, A, nn * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(dB, B, nn * sizeof(double), cudaMemcpyHostToDevice, st));
        const double one = 1.0, zero = 0.0;
        if (cublasDgemm(blas, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N, n, n, n, &one, dB, n, dA,
                        n, &zero, dC, n) != CUBLAS_STATUS_SUCCESS)
            throw Error{QCG_ERR_CUDA, "cublasDgemm failed"};
        CK(cudaMemcpyAsync(C, dC, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    // Dp = 2 U_occ U_occ^T from row-major U whose first nocc columns are the occupied orbitals
    void occ_density(int n, int nocc, const double* U, double* Dp)
    {
        reserve(n);
        const size_t nn = (size_t)n * n;
        CK(cudaMemcpyAsync(dA, U, nn * sizeof(double), cudaMemcpyHostToDevice, st));
        // column-major view M = U^T; its first nocc rows (ld n) are U_occ^T; Dp = 2 (U_occ^T)^T (U_occ^T)
        const double two = 2.0, zero = 0.0;
        if (cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, nocc, &two, dA, n, dA, n, &zero, dC, n) !=
            CUBLAS_STATUS_SUCCESS)
            throw Error{QCG_ERR_CUDA, "cublasDgemm failed"};
        CK(cudaMemcpyAsync(Dp, dC, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
};

// bases with at least this many functions take the GPU path in qcg_rhf (QCG_GPU_LINALG_MIN overrides)
int gpu_linalg_min()
{
    const char* e = std::getenv("QCG_GPU_LINALG_MIN");
    return e ? std::atoi(e) : 256;
}

// ------------------------------------------------------------------------------------------------
// Real solid-harmonic (spherical) functions over the Cartesian engine.  A spherical component of a shell
// is a fixed combination of the shell's raw Cartesian monomials, ordered m = -l..+l, normalised by its own
// self-overlap (PG_Spherical_MnD/Imp/Evaluator.C:13-24); l = 1: y, z, x; l = 2: xy, yz, z^2-(x^2+y^2)/2,
// xz, x^2-y^2 (the reference's SphericalShell table, src/Math/Angular.C).  With the Cartesian functions
// normalised by ns, chi_s = sum_t T[t][s] phi_t, T[t][s] = N_s c_t / ns_t, and every spherical matrix is
// T^T M T of the Cartesian one (J and K of D_sph are those of D_cart = T D_sph T^T).  T is block-diagonal
// over shells, so each transform is a sweep over shell-pair blocks.
// ------------------------------------------------------------------------------------------------
struct SphericalMap
{
    int nc = 0, ns = 0;
    std::vector<int> c0, s0, nca, nsa;          // per shell: first Cartesian / spherical function, counts
    std::vector<std::vector<double>> blk;       // per shell: nca x nsa block of T, row-major

    // Cartesian monomial coefficients of the spherical components of shell L (rows: spherical m = -l..l,
    // columns: the shell's Cartesian components in PG order)
    static std::vector<std::vector<double>> harmonics(int L)
    {
        if (L == 0) return {{1.0}};
        if (L == 1) return {{0, 1, 0}, {0, 0, 1}, {1, 0, 0}};   // PG order x, y, z
        // PG order for d: xx, xy, yy, xz, yz, zz
        return {{0, 1, 0, 0, 0, 0}, {0, 0, 0, 0, 1, 0}, {-0.5, 0, -0.5, 0, 0, 1}, {0, 0, 0, 1, 0, 0}, {1, 0, -1, 0, 0, 0}};
    }
    void build(const qcg_handle* h, const std::vector<double>& Scart)
    {
        nc = h->nbf;
        const int nsh = h->nshell;
        c0.resize(nsh);
        s0.resize(nsh);
        nca.resize(nsh);
        nsa.resize(nsh);
        blk.assign(nsh, {});
        ns = 0;
        for (int a = 0; a < nsh; ++a)
        {
            const int L = h->L[a];
            c0[a] = h->f0[a];
            nca[a] = ncart(L);
            nsa[a] = 2 * L + 1;
            s0[a] = ns;
            ns += nsa[a];
            const auto Y = harmonics(L);
            blk[a].assign((size_t)nca[a] * nsa[a], 0.0);
            for (int m = 0; m < nsa[a]; ++m)
            {
                // raw self-overlap of sum_t Y[m][t] raw_t, raw_t = phi_t / ns_t
                double raw = 0.0;
                for (int t = 0; t < nca[a]; ++t)
                    for (int u = 0; u < nca[a]; ++u)
                        raw += Y[m][t] * Y[m][u] * Scart[(size_t)(c0[a] + t) * nc + c0[a] + u] /
                               (h->ns[c0[a] + t] * h->ns[c0[a] + u]);
                require(raw > 0, "spherical component with zero self-overlap");
                const double N = 1.0 / std::sqrt(raw);
                for (int t = 0; t < nca[a]; ++t) blk[a][(size_t)t * nsa[a] + m] = N * Y[m][t] / h->ns[c0[a] + t];
            }
        }
    }
    // D_cart = T D_sph T^T
    void to_cart(const double* Ds, double* Dc) const
    {
        const int nsh = (int)c0.size();
#pragma omp parallel for schedule(dynamic) if (nc > 256)
        for (int a = 0; a < nsh; ++a)
            for (int b = 0; b < nsh; ++b)
                for (int t = 0; t < nca[a]; ++t)
                    for (int u = 0; u < nca[b]; ++u)
                    {
                        double v = 0.0;
                        for (int m = 0; m < nsa[a]; ++m)
                        {
                            const double ta = blk[a][(size_t)t * nsa[a] + m];
                            if (ta == 0.0) continue;
                            for (int k = 0; k < nsa[b]; ++k)
                                v += ta * Ds[(size_t)(s0[a] + m) * ns + s0[b] + k] * blk[b][(size_t)u * nsa[b] + k];
                        }
                        Dc[(size_t)(c0[a] + t) * nc + c0[b] + u] = v;
                    }
    }
    // M_sph = T^T M_cart T
    void to_sph(const double* Mc, double* Ms) const
    {
        const int nsh = (int)c0.size();
#pragma omp parallel for schedule(dynamic) if (nc > 256)
        for (int a = 0; a < nsh; ++a)
            for (int b = 0; b < nsh; ++b)
                for (int m = 0; m < nsa[a]; ++m)
                    for (int k = 0; k < nsa[b]; ++k)
                    {
                        double v = 0.0;
                        for (int t = 0; t < nca[a]; ++t)
                        {
                            const double ta = blk[a][(size_t)t * nsa[a] + m];
                            if (ta == 0.0) continue;
                            for (int u = 0; u < nca[b]; ++u)
                                v += ta * Mc[(size_t)(c0[a] + t) * nc + c0[b] + u] * blk[b][(size_t)u * nsa[b] + k];
                        }
                        Ms[(size_t)(s0[a] + m) * ns + s0[b] + k] = v;
                    }
    }
};

// ------------------------------------------------------------------------------------------------
// Host state of one closed-shell SCF (SCFIterator.C:283-362, SCFAcceleratorDIIS.C:35-238): canonical
// orthogonaliser X = U s^{-1/2}, density, Fock matrix in the orthonormal basis and the DIIS subspace.
// ------------------------------------------------------------------------------------------------
// Near-null overlap modes to drop, by the rule of the reference's default orthogonaliser (LASolverAuto with
// the gap-detection tolerance, LASolver/Internal/Imp/LASolverLapack.C:32-62, 385-402), on ascending overlap
// eigenvalues w: the leading non-positive ones always; then, among the eigenvalues below 1e-3 of the largest,
// the largest ratio between neighbours -- above 30 it is a clean gap and everything below it goes; without a
// clean gap, every eigenvalue below the absolute floor 1e-8 goes.  0: the overlap is kept whole.
int overlap_null_modes(int n, const double* w)
{
    if (n <= 0) return 0;
    int k = 0;
    while (k < n && w[k] <= 0.0) ++k;
    int cut = k;
    double best = 1.0;
    for (int i = k; i + 1 < n && w[i] < 1e-3 * w[n - 1]; ++i)
        if (w[i + 1] / w[i] > best)
        {
            best = w[i + 1] / w[i];
            cut = i + 1;
        }
    if (best > 30.0) return cut;
    int m = k;
    while (m < n && w[m] < 1e-8) ++m;
    return m;
}

// diagonal shift of the dropped modes in X^T F X: far above every orbital energy, so never occupied
constexpr double kDroppedShift = 1e6;

struct ScfCore
{
    int n = 0, nocc = 0;
    int ndrop = 0;   // overlap modes dropped by the orthogonaliser (overlap_null_modes)
    double fdmax = 0, Enn = 0;
    std::vector<double> S, H, X, Xt, D, Dp, F, Fp, Err, tmp, Up, w, a, b, Cocc;
    std::deque<std::vector<double>> Es, Fps;
    double E = 0, Eold = 0, En = 0;
    GpuLinalg* gl = nullptr;   // set: the O(n^3) steps run on the GPU

    void xsyev(const double* A, double* wv, double* V)
    {
        if (gl) gl->syev(n, A, wv, V);
        else syev(n, A, wv, V);
    }
    void xgemm(const double* A, bool ta, const double* B, bool tb, double* C)
    {
        if (gl) gl->gemm(n, A, ta, B, tb, C);
        else gemm(n, A, ta, B, tb, C);
    }

    void init(int n_, int nocc_, std::vector<double> S_, std::vector<double> H_, double fdmax_, double Enn_,
              const double* guess)
    {
        n = n_;
        nocc = nocc_;
        fdmax = fdmax_;
        Enn = Enn_;
        const size_t nn = (size_t)n * n;
        S = std::move(S_);
        H = std::move(H_);
        X.assign(nn, 0.0);
        // orthogonaliser X with X^T S X = 1 on the kept modes, chosen as the reference's default does
        // (LASolverAuto): the overlap's eigenvalues decide whether near-null modes are dropped.  None dropped:
        // on the host X = L^{-T} from the Cholesky factor S = L L^T, which differs from the canonical
        // U s^{-1/2} by a rotation that leaves the DIIS error norms, the aufbau density and the energy
        // unchanged; on the GPU X = U s^{-1/2}.  Modes dropped: the canonical X with their columns zero, and
        // X^T F X shifted by kDroppedShift on them (ortho), so that the eigenproblem is the kept modes' one.
        {
            std::vector<double> sw(n), U(nn);
            xsyev(S.data(), sw.data(), U.data());
            ndrop = overlap_null_modes(n, sw.data());
            require(ndrop < n, "the overlap matrix has no mode to keep");
            if (gl || ndrop > 0 || !cholesky_orthogonaliser(n, S.data(), X.data()))
            {
                require(sw[ndrop] > 0, "overlap matrix is not positive definite");
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j)
                        X[(size_t)i * n + j] = j < ndrop ? 0.0 : U[(size_t)i * n + j] / std::sqrt(sw[j]);
            }
            require(n - ndrop >= nocc, "more occupied orbitals than kept basis modes");
        }
        Xt.assign(nn, 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) Xt[(size_t)j * n + i] = X[(size_t)i * n + j];
        Cocc.assign((size_t)n * std::max(nocc, 1), 0.0);
        tmp.assign(nn, 0.0);
        Fp.assign(nn, 0.0);
        Dp.assign(nn, 0.0);
        D.assign(nn, 0.0);
        Up.assign(nn, 0.0);
        w.assign(n, 0.0);
        F.assign(nn, 0.0);
        Err.assign(nn, 0.0);
        a.assign(nn, 0.0);
        b.assign(nn, 0.0);
        if (guess)
        {
            // caller's initial density (e.g. a learned guess): D as given, symmetrised; its orthonormal-basis
            // image D' = X^T S D S X (X^T S X = 1) enters the first DIIS error
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                {
                    const double x = 0.5 * (guess[(size_t)i * n + j] + guess[(size_t)j * n + i]);
                    require(std::isfinite(x), "non-finite initial density", QCG_ERR_NONFINITE);
                    D[(size_t)i * n + j] = x;
                }
            xgemm(S.data(), false, X.data(), false, tmp.data());       // S X
            xgemm(D.data(), false, tmp.data(), false, Up.data());      // D S X
            xgemm(tmp.data(), true, Up.data(), false, Dp.data());      // X^T S D S X
        }
        else
        {
            ortho(H, Fp);
            diag_fill(Fp);   // core guess (Seed.C:70-80)
        }
    }
    void ortho(const std::vector<double>& M, std::vector<double>& out)
    {
        xgemm(M.data(), false, X.data(), false, tmp.data());
        if (gl) xgemm(X.data(), true, tmp.data(), false, out.data());
        else gemm(n, Xt.data(), false, tmp.data(), false, out.data());   // X^T kept from set-up
        for (int j = 0; j < ndrop; ++j) out[(size_t)j * n + j] += kDroppedShift;
    }
    // aufbau density of an orthonormal-basis Fock matrix, back in the AO basis (exactly symmetric)
    void diag_fill(const std::vector<double>& Fo)
    {
        // only the occupied eigenvectors enter the density
        if (gl) gl->syev(n, Fo.data(), w.data(), Up.data());
        else syev_lowest(n, Fo.data(), nocc, w.data(), Up.data());
        if (gl)
        {
            gl->occ_density(n, nocc, Up.data(), Dp.data());
            xgemm(X.data(), false, Dp.data(), false, tmp.data());
            xgemm(tmp.data(), false, X.data(), true, D.data());
            for (int i = 0; i < n; ++i)
                for (int j = i + 1; j < n; ++j)
                {
                    const double v = 0.5 * (D[(size_t)i * n + j] + D[(size_t)j * n + i]);
                    D[(size_t)i * n + j] = D[(size_t)j * n + i] = v;
                }
            return;
        }
        // host: D' = 2 U_occ U_occ^T and D = X D' X^T = 2 C C^T with C = X U_occ, O(n^2 nocc) each and
        // symmetric by construction
        for (int i = 0; i < n; ++i)
            for (int j = 0; j <= i; ++j)
            {
                double s = 0;
                for (int k = 0; k < nocc; ++k) s += Up[(size_t)i * n + k] * Up[(size_t)j * n + k];
                Dp[(size_t)i * n + j] = Dp[(size_t)j * n + i] = 2 * s;
            }
        for (int i = 0; i < n; ++i)
        {
            double* ci = &Cocc[(size_t)i * nocc];
            for (int k = 0; k < nocc; ++k) ci[k] = 0.0;
            for (int j = 0; j < n; ++j)
            {
                const double xij = X[(size_t)i * n + j];
                const double* uj = &Up[(size_t)j * n];
                for (int k = 0; k < nocc; ++k) ci[k] += xij * uj[k];
            }
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j <= i; ++j)
            {
                double s = 0;
                const double* ci = &Cocc[(size_t)i * nocc];
                const double* cj = &Cocc[(size_t)j * nocc];
                for (int k = 0; k < nocc; ++k) s += ci[k] * cj[k];
                D[(size_t)i * n + j] = D[(size_t)j * n + i] = 2 * s;
            }
    }
    // F = H + J - K/2, the energy of the current density and the DIIS error ||F'D' - D'F'||
    void fock(const double* J, const double* K)
    {
        const size_t nn = (size_t)n * n;
        double e = 0;
        for (size_t k = 0; k < nn; ++k)
        {
            F[k] = H[k] + J[k] - 0.5 * K[k];
            e += D[k] * (H[k] + F[k]);
        }
        E = 0.5 * e + Enn;
        if (!std::isfinite(E)) throw Error{QCG_ERR_NONFINITE, "non-finite SCF energy"};
        ortho(F, Fp);
        xgemm(Fp.data(), false, Dp.data(), false, a.data());
        if (gl)
        {
            xgemm(Dp.data(), false, Fp.data(), false, b.data());
            for (size_t k = 0; k < nn; ++k) Err[k] = a[k] - b[k];
        }
        else
            // F' and D' are symmetric, so D'F' = (F'D')^T
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) Err[(size_t)i * n + j] = a[(size_t)i * n + j] - a[(size_t)j * n + i];
        En = 0;
        for (size_t k = 0; k < nn; ++k) En += Err[k] * Err[k];
        En = std::sqrt(En);
    }
    // Pulay extrapolation over the last nproj (Err, F') pairs -- entered only while En <= fdmax, pruned from
    // the oldest while the bordered matrix has a singular value below svtol -- then the new density
    void step(const qcg_scf_params& prm)
    {
        const size_t nn = (size_t)n * n;
        std::vector<double> Fuse = Fp;
        if (En != 0.0 && En <= fdmax)
        {
            Es.push_back(Err);
            Fps.push_back(Fp);
            if ((int)Es.size() > prm.diis_nproj)
            {
                Es.pop_front();
                Fps.pop_front();
            }
            auto bordered = [&]() {
                const int m = (int)Es.size();
                std::vector<double> B((m + 1) * (m + 1), 0.0);
                for (int i = 0; i < m; ++i)
                {
                    B[i * (m + 1) + m] = B[m * (m + 1) + i] = 1.0;
                    for (int j = i; j < m; ++j)
                    {
                        double s = 0;
                        for (size_t k = 0; k < nn; ++k) s += Es[i][k] * Es[j][k];
                        B[i * (m + 1) + j] = B[j * (m + 1) + i] = s;
                    }
                }
                return B;
            };
            auto minsv = [&](const std::vector<double>& B) {
                const int m1 = (int)std::lround(std::sqrt((double)B.size()));
                std::vector<double> ev(m1), vv(B.size());
                syev(m1, B.data(), ev.data(), vv.data());
                double mn = 1e300;
                for (double x : ev) mn = std::min(mn, std::fabs(x));
                return mn;
            };
            if (Es.size() >= 2)
            {
                auto B = bordered();
                while (Es.size() >= 2 && minsv(B) < prm.diis_svtol)
                {
                    Es.pop_front();
                    Fps.pop_front();
                    B = bordered();
                }
                const int m = (int)Es.size();
                if (m >= 2)
                {
                    std::vector<double> rhs(m + 1, 0.0);
                    rhs[m] = 1.0;
                    auto c = solve_dense(m + 1, B, rhs);
                    std::fill(Fuse.begin(), Fuse.end(), 0.0);
                    for (int i = 0; i < m; ++i)
                        for (size_t k = 0; k < nn; ++k) Fuse[k] += c[i] * Fps[i][k];
                }
            }
        }
        diag_fill(Fuse);
    }
};

// nuclear repulsion and total nuclear charge of natom nuclei
void nuclei(int natom, const double* Z, const double* R, double& Ztot, double& Enn)
{
    Ztot = 0;
    Enn = 0;
    for (int i = 0; i < natom; ++i)
    {
        Ztot += Z[i];
        for (int j = 0; j < i; ++j)
        {
            double d2 = 0;
            for (int x = 0; x < 3; ++x) d2 += (R[3 * i + x] - R[3 * j + x]) * (R[3 * i + x] - R[3 * j + x]);
            Enn += Z[i] * Z[j] / std::sqrt(d2);
        }
    }
}

// the handle's side streams and their fork/join events (class kernels of one build run side by side)
void ensure_side_streams(qcg_handle* h)
{
    if (h->fork) return;
    h->fork = h->new_event(false);
    for (int s = 0; s < qcg_handle::kSide; ++s)
    {
        h->side[s] = h->new_stream();
        h->join[s] = h->new_event(false);
    }
}

void ensure_jk_buffers(qcg_handle* h)
{
    if (h->d_Jp) return;
    const size_t nn = (size_t)h->packed;
    h->d_D = h->alloc<double>(nn);
    // room for the deterministic mode's low words (QCG_JK_DETERMINISTIC): J' and K' are 2 nn words each
    h->d_Jp = h->alloc<double>(2 * nn);
    h->d_Kp = h->alloc<double>(2 * nn);
    h->d_J = h->alloc<double>(nn);
    h->d_K = h->alloc<double>(nn);
    h->d_flag = h->alloc<int>(1);
}

// ------------------------------------------------------------------------------------------------
// pair lists, Schwarz bounds and screened work lists
// ------------------------------------------------------------------------------------------------
void build_screening(qcg_handle* h, double thresh)
{
    // merged uploads never outlive this call: on an error the pending copy is dropped (the screening is
    // then incomplete and h->screened stays false) and later uploads are issued one by one again
    struct UploadModeReset
    {
        qcg_handle* h;
        ~UploadModeReset()
        {
            h->pend_span = 0;
            h->defer_uploads = false;
        }
    } upload_mode_reset{h};
    // shell pairs per class, (a,b) with L_a > L_b, or L_a == L_b and a >= b
    std::vector<int> sa[kNumPairClasses], sb[kNumPairClasses];
    for (int a = 0; a < h->nshell; ++a)
        for (int b = h->mol_shell0[h->shell_mol[a]]; b <= a; ++b)   // pairs within one molecule
        {
            int x = a, y = b;
            if (h->L[y] > h->L[x]) std::swap(x, y);
            const int pc = pair_class(h->L[x], h->L[y]);
            sa[pc].push_back(x);
            sb[pc].push_back(y);
        }
    // primitive pairs in class order (unsorted), then Schwarz
    struct PP
    {
        double p, Px, Py, Pz, PAx, PAy, PAz, PBx, PBy, PBz, K;
    };
    auto make_pp = [&](int a, int i, int b, int j) {
        const int pa = h->prim0[a] + i, pb = h->prim0[b] + j;
        const double al = h->alpha[pa], be = h->alpha[pb];
        const double* A = &h->cen[3 * a];
        const double* B = &h->cen[3 * b];
        PP d;
        d.p = al + be;
        const double ip = 1.0 / d.p;
        d.Px = (al * A[0] + be * B[0]) * ip;
        d.Py = (al * A[1] + be * B[1]) * ip;
        d.Pz = (al * A[2] + be * B[2]) * ip;
        d.PAx = d.Px - A[0]; d.PAy = d.Py - A[1]; d.PAz = d.Pz - A[2];
        d.PBx = d.Px - B[0]; d.PBy = d.Py - B[1]; d.PBz = d.Pz - B[2];
        const double r2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
        d.K = h->coef[pa] * h->coef[pb] * std::exp(-al * be * ip * r2);
        return d;
    };
    auto build_pp = [&](const std::vector<int>* A_, const std::vector<int>* B_, std::vector<PP>& pp,
                        std::vector<int>* ppo, std::vector<int>* npp) {
        pp.clear();
        for (int c = 0; c < kNumPairClasses; ++c)
        {
            ppo[c].resize(A_[c].size());
            npp[c].resize(A_[c].size());
            for (size_t k = 0; k < A_[c].size(); ++k)
            {
                const int a = A_[c][k], b = B_[c][k];
                ppo[c][k] = (int)pp.size();
                npp[c][k] = h->nprim[a] * h->nprim[b];
                for (int i = 0; i < h->nprim[a]; ++i)
                    for (int j = 0; j < h->nprim[b]; ++j) pp.push_back(make_pp(a, i, b, j));
            }
        }
    };
    auto upload_pp = [&](const std::vector<PP>& pp) {
        std::vector<double> f[11];
        for (auto& x : pp)
        {
            const double v[11] = {x.p, x.Px, x.Py, x.Pz, x.PAx, x.PAy, x.PAz, x.PBx, x.PBy, x.PBz, x.K};
            for (int k = 0; k < 11; ++k) f[k].push_back(v[k]);
        }
        double* d[11];
        for (int k = 0; k < 11; ++k) d[k] = h->upload(f[k]);
        PrimPairsDev P{d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9], d[10]};
        return P;
    };
    std::vector<PP> pp;
    std::vector<int> ppo[kNumPairClasses], npp[kNumPairClasses];
    build_pp(sa, sb, pp, ppo, npp);
    h->begin_uploads();   // merged until the Schwarz launches
    PrimPairsDev P0 = upload_pp(pp);
    std::vector<double> Qc[kNumPairClasses];
    std::vector<void*> tmp;
    // the six diagonal classes side by side: the uploads are on the handle's stream, the side streams
    // start after them and the handle's stream waits for all of them before copying the bounds back (a copy
    // into pageable memory returns only when it is done, so no copy is queued between the launches)
    ensure_side_streams(h);
    std::vector<std::array<int*, 4>> lists(kNumPairClasses);
    std::vector<double*> dQs(kNumPairClasses, nullptr);
    for (int c = 0; c < kNumPairClasses; ++c)
    {
        const int n = (int)sa[c].size();
        Qc[c].assign(n, 0.0);
        if (n == 0) continue;
        lists[c] = {h->upload(sa[c]), h->upload(sb[c]), h->upload(ppo[c]), h->upload(npp[c])};
        dQs[c] = h->alloc<double>(n);
    }
    // the side streams must also see the uploads just queued on the handle's stream
    h->flush_uploads();
    CK(cudaEventRecord(h->fork, h->stream));
    for (int s = 0; s < qcg_handle::kSide; ++s) CK(cudaStreamWaitEvent(h->side[s], h->fork, 0));
    for (int c = kNumPairClasses - 1; c >= 0; --c)
    {
        const int n = (int)sa[c].size();
        if (n == 0) continue;
        cudaStream_t st = h->side[c % qcg_handle::kSide];
        PairListDev pl{n, lists[c][0], lists[c][1], lists[c][2], lists[c][3], nullptr, nullptr};
        kSchwarzLaunchers[c](pl, P0, dQs[c], h->d_boys, st, h->nsm);
        CK(cudaGetLastError());
        tmp.insert(tmp.end(), {lists[c][0], lists[c][1], lists[c][2], lists[c][3], dQs[c]});
    }
    for (int s = 0; s < qcg_handle::kSide; ++s)
    {
        CK(cudaEventRecord(h->join[s], h->side[s]));
        CK(cudaStreamWaitEvent(h->stream, h->join[s], 0));
    }
    for (int c = 0; c < kNumPairClasses; ++c)
        if (!sa[c].empty())
            CK(cudaMemcpyAsync(Qc[c].data(), dQs[c], sa[c].size() * sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (void* p : tmp) h->release(p);
    for (const double* p : {P0.p, P0.Px, P0.Py, P0.Pz, P0.PAx, P0.PAy, P0.PAz, P0.PBx, P0.PBy, P0.PBz, P0.K})
        h->release((void*)p);
    for (int c = 0; c < kNumPairClasses; ++c)
        for (size_t k = 0; k < sa[c].size(); ++k)
            if (!std::isfinite(Qc[c][k])) throw Error{QCG_ERR_NONFINITE, "non-finite Schwarz bound"};
    // full Q matrix for callers (single molecule)
    h->Qfull.clear();
    if (h->nmol == 1)
    {
        h->Qfull.assign((size_t)h->nshell * h->nshell, 0.0);
        for (int c = 0; c < kNumPairClasses; ++c)
            for (size_t k = 0; k < sa[c].size(); ++k)
            {
                h->Qfull[(size_t)sa[c][k] * h->nshell + sb[c][k]] = Qc[c][k];
                h->Qfull[(size_t)sb[c][k] * h->nshell + sa[c][k]] = Qc[c][k];
            }
    }
    // sort each class by molecule, then Q descending; rebuild primitive pairs in that order
    for (int c = 0; c < kNumPairClasses; ++c)
    {
        const size_t n = sa[c].size();
        std::vector<size_t> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
            const int mx = h->shell_mol[sa[c][x]], my = h->shell_mol[sa[c][y]];
            return mx != my ? mx < my : Qc[c][x] > Qc[c][y];
        });
        h->pl_sa[c].resize(n);
        h->pl_sb[c].resize(n);
        h->pl_Q[c].resize(n);
        h->pl_mol[c].resize(n);
        for (size_t k = 0; k < n; ++k)
        {
            h->pl_sa[c][k] = sa[c][ord[k]];
            h->pl_sb[c][k] = sb[c][ord[k]];
            h->pl_Q[c][k] = Qc[c][ord[k]];
            h->pl_mol[c][k] = h->shell_mol[sa[c][ord[k]]];
        }
    }
    build_pp(h->pl_sa, h->pl_sb, pp, h->pl_ppo, h->pl_npp);
    h->begin_uploads();   // merged until the end of the screening
    h->pp_dev = upload_pp(pp);
    for (int c = 0; c < kNumPairClasses; ++c)
    {
        const int n = (int)h->pl_sa[c].size();
        h->pl_dev[c] = PairListDev{n, h->upload(h->pl_sa[c]), h->upload(h->pl_sb[c]), h->upload(h->pl_ppo[c]),
                                   h->upload(h->pl_npp[c]), h->upload(h->pl_Q[c]),
                                   h->nmol > 1 ? h->upload(h->pl_mol[c]) : nullptr};
    }
    // each molecule's range [seg[c][m], seg[c][m+1]) in the sorted pair list of class c
    std::vector<std::vector<int>> seg(kNumPairClasses, std::vector<int>(h->nmol + 1, 0));
    for (int c = 0; c < kNumPairClasses; ++c)
    {
        std::vector<int> cnt(h->nmol, 0);
        for (int m : h->pl_mol[c]) ++cnt[m];
        for (int m = 0; m < h->nmol; ++m) seg[c][m + 1] = seg[c][m] + cnt[m];
    }
    // work lists: bra pair i of class X against the prefix of class Y with Q_i Q_j >= thresh
    h->work_quartets = 0;
    h->work_prim_quartets = 0;
    h->work_flops = 0;
    for (int X = 0; X < kNumPairClasses; ++X)
        for (int Y = 0; Y <= X; ++Y)
        {
            const int k = X * (X + 1) / 2 + Y;
            const auto& qx = h->pl_Q[X];
            const auto& qy = h->pl_Q[Y];
            std::vector<long long> offs(qx.size() + 1, 0);
            std::vector<int> kbase(qx.size(), 0);
            // prefix sums of ket primitive-pair counts for the primitive-quartet tally
            std::vector<long long>& nppy = h->pl_nppsum[Y];
            nppy.assign(qy.size() + 1, 0);
            for (size_t j = 0; j < qy.size(); ++j) nppy[j + 1] = nppy[j] + h->pl_npp[Y][j];
            std::vector<long long> cum(qx.size() + 1, 0);
            long long pq = 0;
            for (size_t i = 0; i < qx.size(); ++i)
            {
                // kets: the bra's molecule's part of class Y, Q descending
                const int m = h->pl_mol[X][i];
                const int jb = seg[Y][m], je = seg[Y][m + 1];
                long long cnt = 0;
                if (qx[i] > 0)
                {
                    const double need = thresh / qx[i];
                    // count of entries >= need (upper_bound with > keeps ties in front)
                    cnt = std::upper_bound(qy.begin() + jb, qy.begin() + je, need,
                                           [](double v, double e) { return v > e; }) -
                          (qy.begin() + jb);
                }
                if (X == Y) cnt = std::min<long long>(cnt, (long long)i - jb + 1);
                kbase[i] = jb;
                offs[i + 1] = offs[i] + cnt;
                pq += (long long)h->pl_npp[X][i] * (nppy[jb + cnt] - nppy[jb]);
                cum[i + 1] = pq;
            }
            h->work[k].total = offs.back();
            h->work[k].gbeg = 0;
            h->work[k].gend = offs.back();
            h->work[k].run = 0;
            h->work[k].cap = 0;
            h->work[k].offs = h->upload(offs);
            h->work[k].kbase = h->nmol > 1 ? h->upload(kbase) : nullptr;

            h->work[k].mols = h->mols();
            h->work[k].same_class = (X == Y);
            h->work[k].lo = 0.0;
            h->work[k].hi = HUGE_VAL;
            h->work_quartets += offs.back();
            h->work_prim_quartets += pq;
            h->work_flops += (double)pq * class_flops(kPairLA[X], kPairLB[X], kPairLA[Y], kPairLB[Y]);
            h->wh_offs[k] = std::move(offs);   // offs, kbase and cum are not used after this
            h->wh_kbase[k] = std::move(kbase);
            h->wh_cum[k] = std::move(cum);
        }
    h->flush_uploads();
    CK(cudaStreamSynchronize(h->stream));
    h->thresh = thresh;
    h->screened = true;
}

// The first quartet of share r (of w) of class k's work list: the cut lies where the primitive quartets
// before it (the ERI work: a contracted quartet costs its primitive-quartet count) reach r/w of the class's
// total, so that ranks get equal work rather than equal quartet counts.  Within the bra pair that holds the
// cut, the kets' primitive-pair prefix sums place it to the quartet.
long long shard_cut(const qcg_handle* h, int k, long long r, long long w)
{
    const std::vector<long long>& offs = h->wh_offs[k];
    const std::vector<long long>& cum = h->wh_cum[k];
    const long long total = offs.empty() ? 0 : offs.back();
    if (r <= 0) return 0;
    if (r >= w || cum.empty() || cum.back() <= 0) return r >= w ? total : total * r / w;
    const long long target = (long long)((long double)cum.back() * r / w);
    // bra pair i with cum[i] <= target < cum[i + 1]
    const size_t i = (size_t)(std::upper_bound(cum.begin(), cum.end(), target) - cum.begin()) - 1;
    if (i + 1 >= cum.size()) return total;
    int X = 0;
    while ((X + 1) * (X + 2) / 2 <= k) ++X;
    const int Y = k - X * (X + 1) / 2;
    const long long np = h->pl_npp[X][i];
    const std::vector<long long>& nppy = h->pl_nppsum[Y];
    const long long jb = h->wh_kbase[k][i], len = offs[i + 1] - offs[i];
    // smallest c in [0, len] with np * (nppy[jb + c] - nppy[jb]) >= target - cum[i]
    long long lo = 0, hi = len;
    while (lo < hi)
    {
        const long long mid = (lo + hi) / 2;
        if (np * (nppy[jb + mid] - nppy[jb]) >= target - cum[i]) hi = mid;
        else lo = mid + 1;
    }
    return offs[i] + lo;
}

// this handle's slice [gbeg, gend) of class k under qcg_set_shard
void shard_range(const qcg_handle* h, int k, long long& gbeg, long long& gend)
{
    gbeg = shard_cut(h, k, h->shard_rank, h->shard_world);
    gend = shard_cut(h, k, h->shard_rank + 1, h->shard_world);
}

// kets per work item of the warp-shared form: J'(a b) leaves the registers once per item
constexpr int kWarpItemKets = 256;

// The warp-shared form's work of class k: the class's bra pairs that have quartets, grouped by first shell
// (one shell belongs to one molecule; within a group the pair list's order, Q descending, so that a set's
// lanes have similar screened ket prefixes), cut into half-warp sets of up to 16 pairs.  The sets, ordered by
// their longest prefix, are paired two to a warp; each pair's kets [0, its longer prefix) are cut into items
// of kWarpItemKets, one int4 per half (a half past its own prefix gets an empty entry).  Built once per
// screening, before any capture.
void warp_items(qcg_handle* h, int k)
{
    if (h->witems_ready[k]) return;
    int X = 0;
    while ((X + 1) * (X + 2) / 2 <= k) ++X;
    const std::vector<long long>& offs = h->wh_offs[k];
    const std::vector<int>& sa = h->pl_sa[X];
    std::vector<int> ord;
    for (int i = 0; i + 1 < (int)offs.size(); ++i)
        if (offs[i + 1] > offs[i]) ord.push_back(i);
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return sa[x] < sa[y]; });
    struct Set
    {
        long long maxp;
        int start, cnt;
    };
    std::vector<Set> sets;
    for (size_t g0 = 0; g0 < ord.size();)
    {
        size_t g1 = g0;
        while (g1 < ord.size() && sa[ord[g1]] == sa[ord[g0]]) ++g1;
        for (size_t s0 = g0; s0 < g1; s0 += 16)
        {
            const int cnt = (int)std::min<size_t>(16, g1 - s0);
            long long maxp = 0;
            for (int l = 0; l < cnt; ++l) maxp = std::max(maxp, offs[ord[s0 + l] + 1] - offs[ord[s0 + l]]);
            sets.push_back({maxp, (int)s0, cnt});
        }
        g0 = g1;
    }
    std::stable_sort(sets.begin(), sets.end(), [](const Set& x, const Set& y) { return x.maxp > y.maxp; });
    std::vector<int4> items;
    for (size_t q = 0; q < sets.size(); q += 2)
    {
        const Set A = sets[q];
        const Set B = q + 1 < sets.size() ? sets[q + 1] : Set{0, A.start, 0};
        const long long m = std::max(A.maxp, B.maxp);
        for (long long j0 = 0; j0 < m; j0 += kWarpItemKets)
            for (const Set& S : {A, B})
            {
                if (j0 < S.maxp)
                    items.push_back(
                        make_int4(S.start, S.cnt, (int)j0, (int)std::min<long long>(S.maxp, j0 + kWarpItemKets)));
                else
                    items.push_back(make_int4(S.start, 0, (int)j0, (int)j0));
            }
    }
    h->d_wgbra[k] = ord.empty() ? nullptr : h->upload(ord);
    h->d_witems[k] = items.empty() ? nullptr : h->upload(items);
    h->nwitems[k] = (long long)items.size() / 2;   // warp items: two half-warp entries each
    h->witems_ready[k] = true;
}

#ifndef QCG_JK_WARP_DEFAULT_MASK
#define QCG_JK_WARP_DEFAULT_MASK 0u
#endif
// The classes whose direct J/K build runs in the warp-shared form: the build's choice
// (QCG_JK_WARP_DEFAULT_MASK), unless QCG_JK_WARP_MASK in the environment names others (read once; *forced
// then true).
unsigned jk_warp_mask_default(bool* forced)
{
    static const char* const env = std::getenv("QCG_JK_WARP_MASK");
    static const bool from_env = env && *env;
    static const unsigned mask = from_env ? (unsigned)std::strtoul(env, nullptr, 0) : (unsigned)(QCG_JK_WARP_DEFAULT_MASK);
    if (forced) *forced = from_env;
    return mask;
}

bool team_scratch(qcg_handle* h, int k, TeamScratchDev& scr, TeamShape& sh);
unsigned jk_team_mask_default(bool* forced);
// smallest per-rank quartet count of a class for the build's default team form (2^20: ~220 groups of 32
// quartets per CTA on 148 SMs)
constexpr long long kJKTeamMinQuartets = 1LL << 20;

// fp32_below: quartets whose density-weighted bound Q_ab Q_cd max|D| (max over the six D blocks the
// quartet digests) is below it are evaluated in FP32 (FP64 accumulation); 0 = all FP64, HUGE_VAL = all
// FP32.  The weighting is what makes FP32 safe: the FP32 error of a quartet's contribution to J and K is
// about 3e-7 of its bound.  dmax (the density maxima of dD) is computed here when the caller has none.
void jk_device(qcg_handle* h, const double* dD, double* dJ, double* dK, int flags, qcg_stats* stats,
               const double* dmax = nullptr, double dthr = 0.0, double fp32_below = 0.0)
{
    require(h->screened, "qcg_schwarz must be called before qcg_fock_jk", QCG_ERR_STATE);
    ensure_jk_buffers(h);
    const int n = h->nbf;
    const size_t nn = (size_t)h->packed;
    // density screening and the density-weighted FP32 band index a shell x shell table: single molecule
    require(h->nmol == 1 || (!dmax && (fp32_below <= 0 || fp32_below >= HUGE_VAL)),
            "density-weighted screening and mixed precision need a single-molecule handle");
    if (fp32_below > 0 && fp32_below < HUGE_VAL && !dmax)
    {
        if (!h->d_dmaxD) h->d_dmaxD = h->alloc<double>((size_t)h->nshell * h->nshell);
        launch_block_max(dD, h->d_f0, h->bs.L, h->nshell, n, h->d_dmaxD, h->stream, h->nsm);
        dmax = h->d_dmaxD;
    }
    if (!h->ev0)
    {
        h->ev0 = h->new_event(true);
        h->ev1 = h->new_event(true);
        h->ev2 = h->new_event(true);
    }
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    if (!(flags & QCG_JK_SKIP_VALIDATION))
    {
        launch_validate(dD, (long long)nn, n, h->mols(), 1e-10, h->d_flag, h->stream, h->nsm);
        int flag = 0;
        CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (flag & 1) throw Error{QCG_ERR_NONFINITE, "density matrix has NaN/Inf entries"};
        if (flag & 2) throw Error{QCG_ERR_ASYMMETRIC, "density matrix is not symmetric"};
    }
    ensure_side_streams(h);
    // the build: zero J'/K', class kernels over the side streams, symmetrisation (timing events only
    // when the build is not a graph)
    // classes built in the team form (FP64 band only); their scratch is sized here, before any capture, and
    // their launches share it, so they run one after another on the first side stream
    // The build's default applies to a class only when its slice has at least kJKTeamMinQuartets quartets:
    // the team form is a throughput design (a CTA per SM streaming groups of 32 quartets), and on a small
    // build (a 57-function water) its classes took 3x the thread-per-quartet kernels' time.  A mask set by
    // qcg_set_jk_team_classes or QCG_JK_TEAM_MASK applies whatever the size.
    bool jk_forced = h->jk_team_mask >= 0;
    unsigned jk_mask = jk_forced ? (unsigned)h->jk_team_mask : jk_team_mask_default(&jk_forced);
    bool team_k[kNumQuartetClasses] = {};
    TeamScratchDev team_scr[kNumQuartetClasses]{};
    TeamShape team_sh[kNumQuartetClasses]{};
    for (int k = 0; k < kNumQuartetClasses; ++k)
    {
        long long gb = 0, ge = 0;
        shard_range(h, k, gb, ge);
        const long long span = ge - gb;
        if (((jk_mask >> k) & 1u) && h->work[k].total > 0 && (jk_forced || span >= kJKTeamMinQuartets))
            team_k[k] = team_scratch(h, k, team_scr[k], team_sh[k]);
    }
    for (int k = 0; k < kNumQuartetClasses; ++k)   // the buffer may have grown after an earlier class's lookup
        if (team_k[k]) team_scratch(h, k, team_scr[k], team_sh[k]);
    // classes in the warp-shared form (FP64 band, one rank, not deterministic; the team form comes first);
    // their work items are built here, before any capture.  The build's default applies to full builds of
    // classes with at least kJKTeamMinQuartets quartets: under density screening a warp evaluates every
    // quartet that one of its lanes needs, where the thread-per-quartet form skips each one alone.  A mask
    // set by qcg_set_jk_warp_classes or QCG_JK_WARP_MASK applies to every build.
    bool warp_forced = h->jk_warp_mask >= 0;
    const unsigned warp_mask =
        warp_forced ? (unsigned)h->jk_warp_mask : jk_warp_mask_default(&warp_forced);
    bool warp_k[kNumQuartetClasses] = {};
    for (int k = 0; k < kNumQuartetClasses; ++k)
        if (((warp_mask >> k) & 1u) && !team_k[k] && h->work[k].total > 0 && h->shard_world == 1 &&
            !(flags & QCG_JK_DETERMINISTIC) &&
            (warp_forced || (dmax == nullptr && dthr <= 0.0 && h->work[k].total >= kJKTeamMinQuartets)))
        {
            warp_items(h, k);
            warp_k[k] = h->nwitems[k] > 0;
        }
    // QCG_JK_DETERMINISTIC: J' and K' as integer accumulator pairs (the low words after the nn high ones),
    // every quartet in FP64
    const bool det = (flags & QCG_JK_DETERMINISTIC) != 0;
    require(!det || fp32_below <= 0, "the deterministic J/K build evaluates every quartet in FP64 (no FP32 band)");
    const size_t nacc = det ? 2 * nn : nn;
    auto enqueue = [&](bool timed) {
        CK(cudaMemsetAsync(h->d_Jp, 0, nacc * sizeof(double), h->stream));
        CK(cudaMemsetAsync(h->d_Kp, 0, nacc * sizeof(double), h->stream));
        if (timed) CK(cudaEventRecord(h->ev1, h->stream));
        CK(cudaEventRecord(h->fork, h->stream));
        for (int s = 0; s < qcg_handle::kSide; ++s) CK(cudaStreamWaitEvent(h->side[s], h->fork, 0));
        // heaviest classes first so that the short ones fill the tail; classes spread over the side streams
        int slot = 0;
        for (int k = kNumQuartetClasses - 1; k >= 0; --k)
        {
            if (h->work[k].total <= 0) continue;
            int X = 0;
            while ((X + 1) * (X + 2) / 2 <= k) ++X;
            const int Y = k - X * (X + 1) / 2;
            JKWorkDev wk = h->work[k];
            wk.run = h->tuned_run[k];
            wk.cap = h->tuned_cap[k];
            wk.mol_active = h->d_mol_active;
            // this rank's contiguous slice of the class's quartets (equal shares of its primitive quartets)
            shard_range(h, k, wk.gbeg, wk.gend);
            if (wk.gend <= wk.gbeg) continue;
            wk.dmax = dmax;
            wk.nshell = h->nshell;
            wk.dthr = dthr;
            wk.pmask = h->d_pmask;
            wk.det_lo = det ? (long long)nn : 0;
            if (fp32_below < HUGE_VAL)
            {
                wk.lo = fp32_below;
                wk.hi = HUGE_VAL;
                if (team_k[k])
                    kJKTeamLaunchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, dD, h->d_Jp, h->d_Kp, n,
                                        h->d_boys, team_scr[k], team_sh[k], h->side[0]);
                else if (warp_k[k])
                {
                    kJKWarpLaunchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, dD, h->d_Jp, h->d_Kp, n,
                                        h->d_boys, h->d_wgbra[k], h->d_witems[k], h->nwitems[k], h->side[slot],
                                        h->nsm);
                    slot = (slot + 1) % qcg_handle::kSide;
                }
                else
                {
                    kJKLaunchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, dD, h->d_Jp, h->d_Kp, n,
                                    h->d_boys, h->side[slot], h->nsm);
                    slot = (slot + 1) % qcg_handle::kSide;
                }
            }
            if (fp32_below > 0)
            {
                wk.lo = 0.0;
                wk.hi = fp32_below;
                kJK32Launchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, dD, h->d_Jp, h->d_Kp, n,
                                  h->d_boys, h->side[slot], h->nsm);
                slot = (slot + 1) % qcg_handle::kSide;
            }
        }
        CK(cudaGetLastError());
        for (int s = 0; s < qcg_handle::kSide; ++s)
        {
            CK(cudaEventRecord(h->join[s], h->side[s]));
            CK(cudaStreamWaitEvent(h->stream, h->join[s], 0));
        }
        if (timed) CK(cudaEventRecord(h->ev2, h->stream));
        if (det)
            launch_symmetrize_fixed(h->d_Jp, h->d_Kp, dJ, dK, (long long)nn, n, h->mols(), h->d_flag, h->stream,
                                    h->nsm);
        else
            launch_symmetrize(h->d_Jp, h->d_Kp, dJ, dK, (long long)nn, n, h->mols(), h->d_flag, h->stream, h->nsm);
        CK(cudaGetLastError());
    };
    // With graphs enabled (qcg_set_graphs), a build whose arguments repeat (the SCF's builds into the
    // handle's own buffers) is captured as a CUDA graph the second time it is seen and replayed from then on:
    // one launch instead of ~25.  Off by default: the class kernels of even a 57-function build run ~0.5 ms,
    // so replay saves little, and capture plus instantiation costs more than a 10-25 iteration SCF recovers.
    const QcgGraphKey key{dD, dJ, dK, dmax, dthr, fp32_below, h->screen_gen};
    cudaGraphExec_t exec = nullptr;
    if ((flags & QCG_JK_SKIP_VALIDATION) && !(flags & QCG_JK_DETERMINISTIC) && h->use_graphs &&
        h->stream != nullptr)   // no capture on the legacy stream; deterministic builds are never recorded
    {
        for (auto& g : h->graphs)
            if (g.first == key) exec = g.second;
        if (!exec && h->last_key == key)
        {
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            try
            {
                enqueue(false);
            }
            catch (...)
            {
                cudaStreamEndCapture(h->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            CK(cudaStreamEndCapture(h->stream, &graph));
            cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) throw Error{QCG_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
            if (h->graphs.size() >= 4)
            {
                cudaGraphExecDestroy(h->graphs.front().second);
                h->graphs.erase(h->graphs.begin());
            }
            h->graphs.push_back({key, exec});
        }
        h->last_key = key;
    }
    CK(cudaEventRecord(h->ev0, h->stream));
    if (exec)
    {
        CK(cudaGraphLaunch(exec, h->stream));
        CK(cudaEventRecord(h->ev1, h->stream));   // no separate ERI interval inside a graph
        CK(cudaEventRecord(h->ev2, h->stream));
    }
    else
        enqueue(true);
    if (stats)
    {
        CK(cudaEventSynchronize(h->ev2));
        float a = 0, b = 0;
        CK(cudaEventElapsedTime(&a, h->ev0, h->ev2));
        CK(cudaEventElapsedTime(&b, h->ev1, h->ev2));
        stats->ms_total = a;
        stats->ms_eri = b;
        stats->quartets = h->work_quartets;
        stats->prim_quartets = h->work_prim_quartets;
        stats->flops = h->work_flops;
    }
}

// grouped visiting order of a batch (returns the device permutation)
const int* batch_order(qcg_handle* h, const int* d_quartets, long long nq)
{
    require(nq <= 0x7fffffffLL, "at most 2^31-1 quartets per batch");
    if (nq > h->sort_cap)
    {
        if (h->d_key) { h->release(h->d_key); h->release(h->d_order); }
        if (!h->d_hist) { h->d_hist = h->alloc<int>(256); h->d_cursor = h->alloc<int>(256); }
        h->d_key = h->alloc<unsigned char>(nq);
        h->d_order = h->alloc<int>(nq);
        h->sort_cap = nq;
    }
    launch_pattern_sort(h->bs, (const int4*)d_quartets, nq, h->d_key, h->d_hist, h->d_cursor, h->d_order, h->stream,
                        h->nsm);
    CK(cudaGetLastError());
    return h->d_order;
}

int class_index(int la, int lb, int lc, int ld)
{
    if (la < lb || lc < ld || la > kMaxL || lc > kMaxL || lb < 0 || ld < 0) return -1;
    const int X = pair_class(la, lb), Y = pair_class(lc, ld);
    if (X < Y) return -1;
    return X * (X + 1) / 2 + Y;
}

}   // namespace

// =================================================================================================
// C ABI
// =================================================================================================
extern "C" {

int qcg_basis_create(const int* shell_L, const int* shell_nprim, const double* exps, const double* coefs,
                     const double* centres, int nshell, qcg_handle** out)
{
    return qcg_basis_create_batch(shell_L, shell_nprim, exps, coefs, centres, nshell, nullptr, 1, out);
}

int qcg_basis_create_batch(const int* shell_L, const int* shell_nprim, const double* exps, const double* coefs,
                           const double* centres, int nshell, const int* shell_mol, int nmol, qcg_handle** out)
{
    if (!out) return QCG_ERR_ARG;
    *out = nullptr;
    qcg_handle* h = new qcg_handle;
    int rc = guarded(h, [&] {
        require(shell_L && shell_nprim && exps && coefs && centres, "null argument");
        require(nshell > 0, "nshell must be positive");
        require(nmol >= 1 && (nmol == 1 || shell_mol), "nmol must be positive (shell_mol is needed for several)");
        h->nshell = nshell;
        h->nmol = nmol;
        h->shell_mol.assign(nshell, 0);
        if (shell_mol)
            for (int s = 0; s < nshell; ++s)
            {
                require(shell_mol[s] >= 0 && shell_mol[s] < nmol, "shell molecule index out of range");
                require(s == 0 || shell_mol[s] == shell_mol[s - 1] || shell_mol[s] == shell_mol[s - 1] + 1,
                        "shells must be grouped by molecule in molecule order");
                h->shell_mol[s] = shell_mol[s];
            }
        require(h->shell_mol[0] == 0 && h->shell_mol[nshell - 1] == nmol - 1, "every molecule needs shells");
        h->mol_shell0.assign(nmol, 0);
        h->mol_nbf.assign(nmol, 0);
        for (int s = nshell - 1; s >= 0; --s) h->mol_shell0[h->shell_mol[s]] = s;
        int np = 0;
        for (int s = 0; s < nshell; ++s)
        {
            require(shell_L[s] >= 0 && shell_L[s] <= kMaxL, "shell L must be 0, 1 or 2");
            require(shell_nprim[s] >= 1, "shell_nprim must be >= 1");
            for (int x = 0; x < 3; ++x) require(std::isfinite(centres[3 * s + x]), "non-finite centre", QCG_ERR_NONFINITE);
            h->L.push_back(shell_L[s]);
            h->nprim.push_back(shell_nprim[s]);
            h->prim0.push_back(np);
            // function offset local to the shell's molecule (global for a single molecule)
            h->f0.push_back(h->mol_nbf[h->shell_mol[s]]);
            h->mol_nbf[h->shell_mol[s]] += ncart(shell_L[s]);
            h->nbf += ncart(shell_L[s]);
            for (int i = 0; i < shell_nprim[s]; ++i)
            {
                const double a = exps[np + i], c = coefs[np + i];
                require(std::isfinite(a) && a > 0, "exponents must be finite and positive");
                require(std::isfinite(c), "non-finite contraction coefficient", QCG_ERR_NONFINITE);
                h->alpha.push_back(a);
                h->coef.push_back(c * prim_norm(a, shell_L[s]));
            }
            np += shell_nprim[s];
            for (int x = 0; x < 3; ++x) h->cen.push_back(centres[3 * s + x]);
        }
        // radial normalisation: unit self-overlap of the (L,0,...) component up to the component factor
        // prod (2n_x-1)!!, which the kernels apply per component (PGData.C:17-33)
        for (int s = 0; s < nshell; ++s)
        {
            double ss = 0.0;
            const int Ls = h->L[s];
            for (int i = 0; i < h->nprim[s]; ++i)
                for (int j = 0; j < h->nprim[s]; ++j)
                {
                    const double p = h->alpha[h->prim0[s] + i] + h->alpha[h->prim0[s] + j];
                    ss += h->coef[h->prim0[s] + i] * h->coef[h->prim0[s] + j] * std::pow(kPi / p, 1.5) / std::pow(2 * p, Ls);
                }
            require(ss > 0, "shell with zero self-overlap");
            const double nrad = 1.0 / std::sqrt(ss);
            for (int i = 0; i < h->nprim[s]; ++i) h->coef[h->prim0[s] + i] *= nrad;
            for (int k = 0; k < ncart(Ls); ++k)
                h->ns.push_back(nrad * comp_norm(Ls, k));
        }
        CK(cudaGetDevice(&h->device));
        CK(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
        h->own_stream = h->new_stream();
        h->stream = h->own_stream;
        const char* ug = std::getenv("QCG_GRAPHS");   // 1: replay repeated J/K builds as CUDA graphs
        h->use_graphs = ug && ug[0] == '1';
        h->d_boys = h->alloc<double>(121 * 23);
        CK(cudaMemcpyAsync(h->d_boys, kBoysTable, sizeof(kBoysTable), cudaMemcpyHostToDevice, h->stream));
        h->bs.nshell = nshell;
        // the device arrays carry one more shell, index nshell, never part of the basis: the unnormalised
        // s function of exponent 0 and coefficient 1, so that (ab|c) = (ab|c s0) (qcg_eri3_batch)
        auto plus = [](std::vector<int> v, int x) { v.push_back(x); return v; };
        auto plusd = [](std::vector<double> v, std::initializer_list<double> x) {
            v.insert(v.end(), x);
            return v;
        };
        h->bs.L = h->upload(plus(h->L, 0));
        h->bs.nprim = h->upload(plus(h->nprim, 1));
        h->bs.prim0 = h->upload(plus(h->prim0, np));
        h->bs.cen = h->upload(plusd(h->cen, {0.0, 0.0, 0.0}));
        h->bs.alpha = h->upload(plusd(h->alpha, {0.0}));
        h->bs.coef = h->upload(plusd(h->coef, {1.0}));
        h->d_f0 = h->upload(h->f0);
        h->mol_off.assign(nmol + 1, 0);
        for (int m = 0; m < nmol; ++m) h->mol_off[m + 1] = h->mol_off[m] + (long long)h->mol_nbf[m] * h->mol_nbf[m];
        h->packed = h->mol_off[nmol];
        if (nmol > 1)
        {
            h->d_shell_mol = h->upload(h->shell_mol);
            h->d_mol_off = h->upload(h->mol_off);
            h->d_mol_n = h->upload(h->mol_nbf);
        }
        CK(cudaStreamSynchronize(h->stream));
    });
    if (rc != QCG_OK)
    {
        // keep the handle so that the caller can read the message, then it must be destroyed
        *out = h;
        return rc;
    }
    *out = h;
    return QCG_OK;
}

void qcg_destroy(qcg_handle* h) { delete h; }

namespace {
void noalloc_forget_addresses();   // defined with the allocation-free J/K build below
}

void qcg_release_cache(void)
{
    ResourceCache::get().release_all();
    noalloc_forget_addresses();
}

const char* qcg_last_error(const qcg_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

int qcg_set_stream(qcg_handle* h, void* s)
{
    if (!h) return QCG_ERR_ARG;
    // work queued on the previous stream (uploads out of the staging buffer among it) completes first
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return QCG_ERR_CUDA;
    h->stream = (cudaStream_t)s;   // NULL is the CUDA default (legacy) stream
    return QCG_OK;
}

int qcg_set_memory_limit(qcg_handle* h, long long bytes)
{
    if (!h || bytes < 0) return QCG_ERR_ARG;
    h->mem_limit = bytes;
    return QCG_OK;
}

int qcg_nmol(const qcg_handle* h, int* nmol)
{
    if (!h || !nmol) return QCG_ERR_ARG;
    *nmol = h->nmol;
    return QCG_OK;
}

int qcg_mol_nbf(const qcg_handle* h, int* nbf)
{
    if (!h || !nbf) return QCG_ERR_ARG;
    std::copy(h->mol_nbf.begin(), h->mol_nbf.end(), nbf);
    return QCG_OK;
}

int qcg_nbf(const qcg_handle* h, int* n)
{
    if (!h || !n) return QCG_ERR_ARG;
    *n = h->nbf;
    return QCG_OK;
}

int qcg_nshell(const qcg_handle* h, int* n)
{
    if (!h || !n) return QCG_ERR_ARG;
    *n = h->nshell;
    return QCG_OK;
}

int qcg_norms(const qcg_handle* h, double* ns)
{
    if (!h || !ns) return QCG_ERR_ARG;
    std::copy(h->ns.begin(), h->ns.end(), ns);
    return QCG_OK;
}

extern "C++" {
namespace {
#ifndef QCG_TEAM_DEFAULT_MASK
#define QCG_TEAM_DEFAULT_MASK 0u
#endif
// The FP64 classes whose ERI batches run in the team form (bit k: class k): the build's choice
// (QCG_TEAM_DEFAULT_MASK, the classes measured faster in that form), unless QCG_ERI_TEAM_MASK in the
// environment names other classes (hexadecimal or decimal bit mask; read once per process).
unsigned eri_team_mask()
{
    static const unsigned mask = [] {
        const char* e = std::getenv("QCG_ERI_TEAM_MASK");
        if (!e || !*e) return (unsigned)(QCG_TEAM_DEFAULT_MASK);
        return (unsigned)std::strtoul(e, nullptr, 0);
    }();
    return mask;
}

// the team form's scratch for class k: one wave of CTAs, each with stage slots for the class's longest
// primitive loop in this basis (the product of the largest contraction lengths of the four angular
// momenta) and its recurrence blocks.  False when that exceeds kTeamScratchMax bytes; the batch then runs in
// the thread-per-quartet form.
constexpr long long kTeamScratchMax = 4LL << 30;

bool team_scratch(qcg_handle* h, int k, TeamScratchDev& scr, TeamShape& sh)
{
    int X = 0;
    while ((X + 1) * (X + 2) / 2 <= k) ++X;
    const int Y = k - X * (X + 1) / 2;
    const int Ls[4] = {kPairLA[X], kPairLB[X], kPairLA[Y], kPairLB[Y]};
    if (!h->maxnp[0])
        for (int l = 0; l <= kMaxL; ++l)
        {
            int mx = 1;
            for (int i = 0; i < h->nshell; ++i)
                if (h->L[i] == l) mx = std::max(mx, h->nprim[i]);
            h->maxnp[l] = mx;
        }
    long long kmax = 1;
    for (int l : Ls) kmax *= h->maxnp[l];
    sh = kEriTeamShapes[k](h->nsm);
    const long long need = (long long)sh.grid * (kmax * sh.slot_doubles + sh.hrr_doubles);
    if (need * (long long)sizeof(double) > kTeamScratchMax) return false;
    if (need > h->team_cap)
    {
        if (h->d_team) h->release(h->d_team);
        h->d_team = nullptr;
        h->team_cap = 0;
        h->d_team = h->alloc<double>((size_t)need);
        h->team_cap = need;
    }
    if (!h->d_team_err)
    {
        h->d_team_err = h->alloc<int>(1);
        CK(cudaMemsetAsync(h->d_team_err, 0, sizeof(int), h->stream));
    }
    scr.rcache = h->d_team;
    scr.kmax = (int)kmax;
    scr.hrr = h->d_team + (long long)sh.grid * kmax * sh.slot_doubles;
    scr.err = h->d_team_err;
    h->team_pending = true;
    return true;
}

// the team kernels' error word (a bulk-copy wait that gave up, or a group longer than the stage slots):
// read after a synchronising call, then cleared
void check_team_error(qcg_handle* h)
{
    if (!h->d_team_err || !h->team_pending) return;
    h->team_pending = false;
    int e = 0;
    CK(cudaMemcpy(&e, h->d_team_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!e) return;
    CK(cudaMemset(h->d_team_err, 0, sizeof(int)));
    throw Error{QCG_ERR_CUDA, e & 1 ? "team kernel: a bulk-copy wait gave up; the results are not valid"
                                    : "team kernel: a primitive loop longer than the stage slots"};
}

#ifndef QCG_JK_TEAM_DEFAULT_MASK
#define QCG_JK_TEAM_DEFAULT_MASK 0u
#endif
// The classes whose direct J/K build runs in the team form: the build's choice (QCG_JK_TEAM_DEFAULT_MASK),
// unless QCG_JK_TEAM_MASK in the environment names others (read once per process; *forced then true).
unsigned jk_team_mask_default(bool* forced)
{
    static const char* const env = std::getenv("QCG_JK_TEAM_MASK");
    static const bool from_env = env && *env;
    static const unsigned mask = from_env ? (unsigned)std::strtoul(env, nullptr, 0) : (unsigned)(QCG_JK_TEAM_DEFAULT_MASK);
    if (forced) *forced = from_env;
    return mask;
}

// output bytes per chunk of a host-buffer ERI batch: 512 MiB, or QCG_BATCH_CHUNK_MB (read once)
long long batch_chunk_bytes()
{
    static const long long bytes = [] {
        const char* e = std::getenv("QCG_BATCH_CHUNK_MB");
        const long long mb = (e && *e) ? std::strtoll(e, nullptr, 10) : 0;
        return mb > 0 ? mb << 20 : (1LL << 29);
    }();
    return bytes;
}

template <class T>
void eri_batch_launch(qcg_handle* h, int k, const int* dq, long long m, T* dout)
{
    const int* order = batch_order(h, dq, m);
    if constexpr (std::is_same_v<T, double>)
    {
        const unsigned mask = h->team_mask >= 0 ? (unsigned)h->team_mask : eri_team_mask();
        TeamScratchDev scr{};
        TeamShape sh{};
        if (((mask >> k) & 1u) && team_scratch(h, k, scr, sh))
            kEriTeamLaunchers[k](h->bs, (const int4*)dq, order, m, dout, h->d_boys, scr, sh, h->stream);
        else
            kEriBatchLaunchers[k](h->bs, (const int4*)dq, order, m, dout, h->d_boys, h->stream, h->nsm);
    }
    else
        kEriBatch32Launchers[k](h->bs, (const int4*)dq, order, m, dout, h->d_boys, h->stream, h->nsm);
    CK(cudaGetLastError());
}

template <class T>
int eri_batch_device(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* d_quartets, T* d_out)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        const int k = class_index(la, lb, lc, ld);
        require(k >= 0, "non-canonical or unsupported angular class");
        require(nq >= 0, "negative quartet count");
        if (nq == 0) return;
        require(d_quartets && d_out, "null argument");
        eri_batch_launch(h, k, d_quartets, nq, d_out);
    });
}

template <class T>
void eri_batch_run(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, T* out);

// Checks rows of `width` shell indices (quartets or triples) against the handle: every index in range
// and of angular momentum Ls[x] in column x.  The scan runs over the host cores and builds no message
// per element; only the first bad row, if any, is examined again to raise the error.
void check_shell_rows(const qcg_handle* h, const int* idx, long long nrow, int width, const int* Ls)
{
    const int ns = h->nshell;
    const int* L = h->L.data();
    long long bad = nrow;
#pragma omp parallel for schedule(static) reduction(min : bad) if (nrow > 65536)
    for (long long r = 0; r < nrow; ++r)
    {
        bool ok = true;
        for (int x = 0; x < width; ++x)
        {
            const int s = idx[width * r + x];
            ok = ok && (unsigned)s < (unsigned)ns && L[s] == Ls[x];
        }
        if (!ok && r < bad) bad = r;
    }
    if (bad == nrow) return;
    for (int x = 0; x < width; ++x)
    {
        const int s = idx[width * bad + x];
        require(s >= 0 && s < ns, "shell index out of range");
        require(L[s] == Ls[x], "shell angular momentum does not match the class");
    }
}

template <class T>
int eri_batch_host(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, T* out)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        const int k = class_index(la, lb, lc, ld);
        require(k >= 0, "non-canonical or unsupported angular class");
        require(nq >= 0, "negative quartet count");
        if (nq == 0) return;
        require(quartets && out, "null argument");
        const int Ls[4] = {la, lb, lc, ld};
        check_shell_rows(h, quartets, nq, 4, Ls);
        eri_batch_run(h, la, lb, lc, ld, nq, quartets, out);
    });
}

// the device part of a host-buffer batch (quartets already checked; may name the unit shell nshell)
template <class T>
void eri_batch_run(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, T* out)
{
    {
        const int k = class_index(la, lb, lc, ld);
        const long long blk = (long long)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
        // two device buffers of at most batch_chunk_bytes() of output each, kept by the handle between
        // calls: the copy of one chunk back to the host overlaps the evaluation of the next.  The chunks
        // ramp up (1/8, 1/4, 1/2 of the full size, then full), so that the copy engine starts early: the
        // evaluation of the first chunk is the one part of the call that nothing overlaps.
        const long long chunk =
            std::max<long long>(1, std::min<long long>(nq, batch_chunk_bytes() / (long long)sizeof(T) / blk));
        const size_t qbytes = (size_t)4 * chunk * sizeof(int), obytes = (size_t)chunk * blk * sizeof(T);
        if (!h->copy_stream)
        {
            h->copy_stream = h->new_stream();
            for (int b = 0; b < 2; ++b)
            {
                h->hb_done[b] = h->new_event(false);
                h->hb_free[b] = h->new_event(false);
            }
        }
        for (int b = 0; b < 2; ++b)
        {
            if (h->hb_qcap[b] < qbytes)
            {
                if (h->hb_q[b]) h->release(h->hb_q[b]);
                h->hb_q[b] = h->alloc<char>(qbytes);
                h->hb_qcap[b] = qbytes;
            }
            if (h->hb_ocap[b] < obytes)
            {
                if (h->hb_out[b]) h->release(h->hb_out[b]);
                h->hb_out[b] = h->alloc<char>(obytes);
                h->hb_ocap[b] = obytes;
            }
            CK(cudaEventRecord(h->hb_free[b], h->copy_stream));   // both buffers start free
        }
        int b = 0;
        long long step = std::max<long long>(1, chunk / 8);
        for (long long q0 = 0, m = 0; q0 < nq; q0 += m, b ^= 1, step = std::min(chunk, 2 * step))
        {
            m = std::min(step, nq - q0);
            int* dq = (int*)h->hb_q[b];
            T* dout = (T*)h->hb_out[b];
            CK(cudaStreamWaitEvent(h->stream, h->hb_free[b], 0));   // the buffer's previous copy-out is done
            CK(cudaMemcpyAsync(dq, quartets + 4 * q0, 4 * m * sizeof(int), cudaMemcpyHostToDevice, h->stream));
            eri_batch_launch(h, k, dq, m, dout);
            CK(cudaEventRecord(h->hb_done[b], h->stream));
            CK(cudaStreamWaitEvent(h->copy_stream, h->hb_done[b], 0));
            CK(cudaMemcpyAsync(out + q0 * blk, dout, m * blk * sizeof(T), cudaMemcpyDeviceToHost, h->copy_stream));
            CK(cudaEventRecord(h->hb_free[b], h->copy_stream));
        }
        CK(cudaStreamSynchronize(h->copy_stream));
        CK(cudaStreamSynchronize(h->stream));
        check_team_error(h);
    }
}
}   // namespace
}   // extern "C++"

int qcg_eri_batch_device(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* d_quartets,
                         double* d_out)
{
    return eri_batch_device(h, la, lb, lc, ld, nq, d_quartets, d_out);
}

int qcg_eri_batch_device_f32(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* d_quartets,
                             float* d_out)
{
    return eri_batch_device(h, la, lb, lc, ld, nq, d_quartets, d_out);
}

int qcg_eri_batch(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, double* out)
{
    return eri_batch_host(h, la, lb, lc, ld, nq, quartets, out);
}

int qcg_eri_batch_f32(qcg_handle* h, int la, int lb, int lc, int ld, long long nq, const int* quartets, float* out)
{
    return eri_batch_host(h, la, lb, lc, ld, nq, quartets, out);
}

// (ab|c) = (ab|c s0) with the handle's unit shell s0 (exponent 0, coefficient 1, index nshell): the 4-centre
// class (la lb|lc s) when the bra pair class is not below (lc s), else (lc s|la lb) with the block transposed
int qcg_eri3_batch(qcg_handle* h, int la, int lb, int lc, long long nt, const int* triples, double* out)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(la >= 0 && la <= kMaxL && lb >= 0 && lb <= la && lc >= 0 && lc <= kMaxL,
                "need 2 >= la >= lb >= 0 and 0 <= lc <= 2");
        require(nt >= 0, "negative triple count");
        if (nt == 0) return;
        require(triples && out, "null argument");
        const int Ls[3] = {la, lb, lc};
        check_shell_rows(h, triples, nt, 3, Ls);
        const int U = h->nshell;
        const bool direct = pair_class(la, lb) >= pair_class(lc, 0);
        std::vector<int> q(4 * (size_t)nt);
        for (long long t = 0; t < nt; ++t)
        {
            const int a = triples[3 * t], b = triples[3 * t + 1], c = triples[3 * t + 2];
            const int v[4] = {direct ? a : c, direct ? b : U, direct ? c : a, direct ? U : b};
            std::copy(v, v + 4, q.begin() + 4 * t);
        }
        const int na = ncart(la), nb = ncart(lb), nc = ncart(lc);
        const long long blk = (long long)na * nb * nc;
        if (direct)
        {
            eri_batch_run(h, la, lb, lc, 0, nt, q.data(), out);
            return;
        }
        std::vector<double> tmp((size_t)nt * blk);
        eri_batch_run(h, lc, 0, la, lb, nt, q.data(), tmp.data());
        for (long long t = 0; t < nt; ++t)
            for (int c = 0; c < nc; ++c)
                for (int ab = 0; ab < na * nb; ++ab) out[t * blk + ab * nc + c] = tmp[t * blk + c * na * nb + ab];
    });
}

int qcg_schwarz(qcg_handle* h, double thresh, double* Q)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(std::isfinite(thresh) && thresh >= 0, "threshold must be finite and non-negative");
        require(!Q || h->nmol == 1, "per-pair bounds are returned for single-molecule handles only");
        if (!h->screened || h->thresh != thresh)
        {
            // drop previous screening state (device buffers of pair lists and work lists)
            if (h->screened)
            {
                for (int c = 0; c < kNumPairClasses; ++c)
                    for (const void* p : {(const void*)h->pl_dev[c].sa, (const void*)h->pl_dev[c].sb,
                                          (const void*)h->pl_dev[c].ppo, (const void*)h->pl_dev[c].npp,
                                          (const void*)h->pl_dev[c].Q, (const void*)h->pl_dev[c].mol})
                        if (p) h->release((void*)p);
                const PrimPairsDev& P = h->pp_dev;
                for (const double* p : {P.p, P.Px, P.Py, P.Pz, P.PAx, P.PAy, P.PAz, P.PBx, P.PBy, P.PBz, P.K})
                    h->release((void*)p);
                for (int k = 0; k < kNumQuartetClasses; ++k)
                {
                    h->release((void*)h->work[k].offs);
                    if (h->work[k].kbase) h->release((void*)h->work[k].kbase);
                    if (h->d_wgbra[k]) h->release(h->d_wgbra[k]);
                    if (h->d_witems[k]) h->release(h->d_witems[k]);
                    h->d_wgbra[k] = nullptr;
                    h->d_witems[k] = nullptr;
                    h->nwitems[k] = 0;
                    h->witems_ready[k] = false;
                }
                h->screened = false;
            }
            h->drop_graphs();
            ++h->screen_gen;
            build_screening(h, thresh);
            for (int k = 0; k < kNumQuartetClasses; ++k) h->tuned_run[k] = h->tuned_cap[k] = 0;   // new lists
        }
        if (Q) std::copy(h->Qfull.begin(), h->Qfull.end(), Q);
    });
}

int qcg_fock_jk_device(qcg_handle* h, const double* d_D, double* d_J, double* d_K, int flags, qcg_stats* stats)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(d_D && d_J && d_K, "null argument");
        jk_device(h, d_D, d_J, d_K, flags, stats, nullptr, 0.0, (flags & QCG_JK_FP32) ? HUGE_VAL : h->fp32_below);
    });
}

// Autotuner of the J/K launch shapes: per class, time the class kernel on (a slice of at most 2^20 of)
// its quartets with each candidate (quartets per lane x blocks-per-SM cap) and keep the fastest for later
// builds.  The timed launches accumulate into the handle's J'/K' scratch, which every build zeroes.
int qcg_autotune_jk(qcg_handle* h, const double* d_D, int reps, int* run_out, int* cap_out)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(h->screened, "qcg_schwarz must be called before qcg_autotune_jk", QCG_ERR_STATE);
        require(d_D && reps >= 1, "bad argument");
        ensure_jk_buffers(h);
        h->drop_graphs();
        cudaEvent_t a = nullptr, b = nullptr;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        const int runs[] = {1, 2, 4, 8, 16}, caps[] = {8, 16};
        try
        {
            for (int k = 0; k < kNumQuartetClasses; ++k)
            {
                h->tuned_run[k] = h->tuned_cap[k] = 0;
                if (h->work[k].total <= 0) continue;
                int X = 0;
                while ((X + 1) * (X + 2) / 2 <= k) ++X;
                const int Y = k - X * (X + 1) / 2;
                JKWorkDev wk = h->work[k];
                wk.gbeg = 0;
                wk.gend = std::min<long long>(wk.total, 1LL << 20);
                float best = 1e30f;
                for (int r : runs)
                    for (int c : caps)
                    {
                        wk.run = r;
                        wk.cap = c;
                        kJKLaunchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, d_D, h->d_Jp, h->d_Kp,
                                        h->nbf, h->d_boys, h->stream, h->nsm);   // warm-up
                        CK(cudaEventRecord(a, h->stream));
                        for (int i = 0; i < reps; ++i)
                            kJKLaunchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, d_D, h->d_Jp, h->d_Kp,
                                            h->nbf, h->d_boys, h->stream, h->nsm);
                        CK(cudaEventRecord(b, h->stream));
                        CK(cudaEventSynchronize(b));
                        CK(cudaGetLastError());
                        float ms = 0;
                        CK(cudaEventElapsedTime(&ms, a, b));
                        if (ms < best)
                        {
                            best = ms;
                            h->tuned_run[k] = r;
                            h->tuned_cap[k] = c;
                        }
                    }
            }
        }
        catch (...)
        {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            throw;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (run_out) std::copy(h->tuned_run, h->tuned_run + kNumQuartetClasses, run_out);
        if (cap_out) std::copy(h->tuned_cap, h->tuned_cap + kNumQuartetClasses, cap_out);
    });
}

int qcg_set_shard(qcg_handle* h, int rank, int world)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(world >= 1 && rank >= 0 && rank < world, "need 0 <= rank < world");
        h->shard_rank = rank;
        h->shard_world = world;
        h->drop_graphs();
    });
}

int qcg_shard_work(qcg_handle* h, int rank, int world, long long* quartets, long long* prim_quartets)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(world >= 1 && rank >= 0 && rank < world, "need 0 <= rank < world");
        require(quartets && prim_quartets, "null argument");
        require(h->screened, "qcg_schwarz must be called first", QCG_ERR_STATE);
        long long nq = 0, npq = 0;
        for (int k = 0; k < kNumQuartetClasses; ++k)
        {
            const long long gb = shard_cut(h, k, rank, world), ge = shard_cut(h, k, rank + 1, world);
            nq += ge - gb;
            // primitive quartets of [gb, ge): the bra pairs' prefix sums, with partial bra pairs at both ends
            auto prim_before = [&](long long g) {
                const std::vector<long long>& offs = h->wh_offs[k];
                if (offs.empty() || g <= 0) return 0LL;
                const size_t i = (size_t)(std::upper_bound(offs.begin(), offs.end(), g) - offs.begin()) - 1;
                if (i + 1 >= offs.size()) return h->wh_cum[k].back();
                int X = 0;
                while ((X + 1) * (X + 2) / 2 <= k) ++X;
                const int Y = k - X * (X + 1) / 2;
                const std::vector<long long>& nppy = h->pl_nppsum[Y];
                const long long jb = h->wh_kbase[k][i];
                return h->wh_cum[k][i] + (long long)h->pl_npp[X][i] * (nppy[jb + (g - offs[i])] - nppy[jb]);
            };
            npq += prim_before(ge) - prim_before(gb);
        }
        *quartets = nq;
        *prim_quartets = npq;
    });
}

int qcg_set_jk_warp_classes(qcg_handle* h, long long mask)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(mask >= -1 && mask < (1LL << kNumQuartetClasses), "mask: -1 or bits of the 21 classes");
        h->jk_warp_mask = mask;
        h->drop_graphs();
    });
}

int qcg_set_graphs(qcg_handle* h, int enable)
{
    if (!h) return QCG_ERR_ARG;
    h->use_graphs = enable != 0;
    if (!h->use_graphs) h->drop_graphs();
    return QCG_OK;
}

int qcg_set_pair_subset(qcg_handle* h, const unsigned char* mask)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(h->nmol == 1, "a pair subset takes a single-molecule handle");
        const int ns = h->nshell;
        if (!mask)
        {
            if (h->d_pmask) h->release(h->d_pmask);
            h->d_pmask = nullptr;
        }
        else
        {
            std::vector<unsigned char> m((size_t)ns * ns);
            for (int a = 0; a < ns; ++a)
                for (int b = 0; b < ns; ++b)
                    m[(size_t)a * ns + b] = (mask[(size_t)a * ns + b] || mask[(size_t)b * ns + a]) ? 1 : 0;
            if (!h->d_pmask) h->d_pmask = h->alloc<unsigned char>(m.size());
            CK(cudaMemcpyAsync(h->d_pmask, m.data(), m.size(), cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        ++h->screen_gen;   // recorded builds (CUDA graphs) no longer apply
    });
}

int qcg_set_jk_team_classes(qcg_handle* h, long long mask)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(mask >= -1 && mask < (1LL << kNumQuartetClasses), "mask must be -1 or a 21-bit class mask");
        h->jk_team_mask = mask;
        ++h->screen_gen;   // recorded builds (CUDA graphs) no longer apply
    });
}

int qcg_set_eri_team_classes(qcg_handle* h, long long mask)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(mask >= -1 && mask < (1LL << kNumQuartetClasses), "mask must be -1 or a 21-bit class mask");
        h->team_mask = mask;
    });
}

int qcg_set_fp32_bound(qcg_handle* h, double bound)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(bound >= 0 && !std::isnan(bound), "bound must be non-negative");
        h->fp32_below = bound;
    });
}

int qcg_fock_jk(qcg_handle* h, const double* D, double* J, double* K, int flags, qcg_stats* stats)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(D && J && K, "null argument");
        const size_t nn = (size_t)h->packed;
        if (!(flags & QCG_JK_SKIP_VALIDATION))
        {
            for (size_t k = 0; k < nn; ++k)
                if (!std::isfinite(D[k])) throw Error{QCG_ERR_NONFINITE, "density matrix has NaN/Inf entries"};
            for (int m = 0; m < h->nmol; ++m)
            {
                const double* Dm = D + h->mol_off[m];
                const int n = h->mol_nbf[m];
                for (int i = 0; i < n; ++i)
                    for (int j = i + 1; j < n; ++j)
                    {
                        const double a = Dm[(size_t)i * n + j], b = Dm[(size_t)j * n + i];
                        if (std::fabs(a - b) > 1e-10 * (1.0 + std::fabs(a)))
                            throw Error{QCG_ERR_ASYMMETRIC, "density matrix is not symmetric"};
                    }
            }
        }
        require(h->screened, "qcg_schwarz must be called before qcg_fock_jk", QCG_ERR_STATE);
        ensure_jk_buffers(h);
        CK(cudaMemcpyAsync(h->d_D, D, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        jk_device(h, h->d_D, h->d_J, h->d_K, flags | QCG_JK_SKIP_VALIDATION, stats, nullptr, 0.0,
                  (flags & QCG_JK_FP32) ? HUGE_VAL : h->fp32_below);
        CK(cudaMemcpyAsync(J, h->d_J, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(K, h->d_K, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        int flag = 0;
        CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        check_team_error(h);
        if (flag & 1) throw Error{QCG_ERR_NONFINITE, "non-finite J/K result"};
    });
}

int qcg_one_electron(qcg_handle* h, int natom, const double* Z, const double* R, double* S, double* T, double* V)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(natom >= 0 && (natom == 0 || (Z && R)) && S && T && V, "bad argument");
        require(h->nmol == 1, "qcg_one_electron takes a single-molecule handle (qcg_one_electron_batch)");
        const int n = h->nbf;
        const size_t nn = (size_t)n * n;
        std::vector<double> z(Z, Z + natom), r(R, R + 3 * natom);
        for (double x : r) require(std::isfinite(x), "non-finite nuclear position", QCG_ERR_NONFINITE);
        double* dZ = h->upload(z);
        double* dR = h->upload(r);
        double* dS = h->alloc<double>(nn);
        double* dT = h->alloc<double>(nn);
        double* dV = h->alloc<double>(nn);
        launch_one_electron(h->bs, h->d_f0, n, natom, dZ, dR, dS, dT, dV, h->d_boys, h->stream, h->nsm);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(S, dS, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(T, dT, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(V, dV, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        for (void* p : {(void*)dZ, (void*)dR, (void*)dS, (void*)dT, (void*)dV}) h->release(p);
        if (e != cudaSuccess) throw Error{QCG_ERR_CUDA, std::string("one-electron integrals: ") + cudaGetErrorString(e)};
    });
}

int qcg_nbf_spherical(const qcg_handle* h, int* n)
{
    if (!h || !n) return QCG_ERR_ARG;
    int s = 0;
    for (int L : h->L) s += 2 * L + 1;
    *n = s;
    return QCG_OK;
}

namespace {
extern "C++" {
// the handle's spherical map (needs the Cartesian overlap, from the one-electron kernel without nuclei)
const SphericalMap& spherical_map(qcg_handle* h)
{
    if (!h->sph)
    {
        require(h->nmol == 1, "spherical functions need a single-molecule handle");
        const size_t nn = (size_t)h->nbf * h->nbf;
        std::vector<double> S(nn), T(nn), V(nn);
        const int e = qcg_one_electron(h, 0, nullptr, nullptr, S.data(), T.data(), V.data());
        if (e != QCG_OK) throw Error{e, h->last_error};
        auto m = std::make_shared<SphericalMap>();
        m->build(h, S);
        h->sph = m;
    }
    return *std::static_pointer_cast<SphericalMap>(h->sph);
}
}
}   // namespace

extern "C++" {
namespace {
// Device products of the symmetry-adapted (SALC) faces: one cuBLAS handle per qcg handle, on its stream,
// and grow-only device buffers for O, the square operand, the intermediate and the result.
struct SalcWork
{
    cublasHandle_t blas = nullptr;
    double* buf[4] = {};
    size_t cap[4] = {};
    ~SalcWork()
    {
        for (double* p : buf) cudaFree(p);
        if (blas) cublasDestroy(blas);
    }
    double* get(int i, size_t n)
    {
        if (n > cap[i])
        {
            cudaFree(buf[i]);
            buf[i] = nullptr;
            cap[i] = 0;
            CK(cudaMalloc(&buf[i], n * sizeof(double)));
            cap[i] = n;
        }
        return buf[i];
    }
};

SalcWork& salc_work(qcg_handle* h)
{
    if (!h->salc)
    {
        auto w = std::make_shared<SalcWork>();
        if (cublasCreate(&w->blas) != CUBLAS_STATUS_SUCCESS) throw Error{QCG_ERR_CUDA, "cublasCreate failed"};
        h->salc = w;
    }
    SalcWork& w = *static_cast<SalcWork*>(h->salc.get());
    cublasSetStream(w.blas, h->stream);
    return w;
}

// fold (Dao += sym(O X O^T), X m x m) or slice (Out += sym(O^T X O), X n x n); O is n x m row-major, which
// cuBLAS (column-major) sees as Oc = O^T, m x n
void salc_product(qcg_handle* h, bool fold, int m, const double* O, const double* X, double* Out)
{
    const int n = h->nbf;
    require(h->nmol == 1, "the symmetry-adapted faces take a single-molecule handle");
    require(m >= 1 && m <= n, "need 1 <= m <= nbf columns");
    require(O && X && Out, "null argument");
    SalcWork& w = salc_work(h);
    const size_t nm = (size_t)n * m, nx = fold ? (size_t)m * m : (size_t)n * n, no = fold ? (size_t)n * n : (size_t)m * m;
    double* dO = w.get(0, nm);
    double* dX = w.get(1, nx);
    double* dT = w.get(2, nm);
    double* dR = w.get(3, no);
    CK(cudaMemcpyAsync(dO, O, nm * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(dX, X, nx * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const double one = 1.0, zero = 0.0;
    cublasStatus_t a, b;
    if (fold)
    {
        // T = X Oc (m x n) = X O^T;  R = Oc^T T (n x n) = O X O^T
        a = cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, m, n, m, &one, dX, m, dO, m, &zero, dT, m);
        b = cublasDgemm(w.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, m, &one, dO, m, dT, m, &zero, dR, n);
    }
    else
    {
        // T = X Oc^T (n x m) = X O;  R = Oc T (m x m) = O^T X O
        a = cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_T, n, m, n, &one, dX, n, dO, m, &zero, dT, n);
        b = cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, m, m, n, &one, dO, m, dT, n, &zero, dR, m);
    }
    if (a != CUBLAS_STATUS_SUCCESS || b != CUBLAS_STATUS_SUCCESS) throw Error{QCG_ERR_CUDA, "cublasDgemm failed"};
    std::vector<double> R(no);
    CK(cudaMemcpyAsync(R.data(), dR, no * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int k = fold ? n : m;
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) Out[(size_t)i * k + j] += 0.5 * (R[(size_t)i * k + j] + R[(size_t)j * k + i]);
}
}   // namespace
}   // extern "C++"

int qcg_salc_fold(qcg_handle* h, int m, const double* O, const double* D, double* Dao)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] { salc_product(h, true, m, O, D, Dao); });
}

int qcg_salc_slice(qcg_handle* h, int m, const double* O, const double* Fao, double* Fab)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] { salc_product(h, false, m, O, Fao, Fab); });
}

int qcg_spherical_transform(qcg_handle* h, double* T)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(T != nullptr, "null argument");
        const SphericalMap& m = spherical_map(h);
        std::fill(T, T + (size_t)m.nc * m.ns, 0.0);
        for (size_t a = 0; a < m.c0.size(); ++a)
            for (int t = 0; t < m.nca[a]; ++t)
                for (int k = 0; k < m.nsa[a]; ++k)
                    T[(size_t)(m.c0[a] + t) * m.ns + m.s0[a] + k] = m.blk[a][(size_t)t * m.nsa[a] + k];
    });
}

int qcg_fock_jk_spherical(qcg_handle* h, const double* D, double* J, double* K, int flags, qcg_stats* stats)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(D && J && K, "null argument");
        const SphericalMap& m = spherical_map(h);
        const size_t nc = (size_t)m.nc * m.nc;
        std::vector<double> Dc(nc), Jc(nc), Kc(nc);
        m.to_cart(D, Dc.data());
        const int e = qcg_fock_jk(h, Dc.data(), Jc.data(), Kc.data(), flags, stats);
        if (e != QCG_OK) throw Error{e, h->last_error};
        m.to_sph(Jc.data(), J);
        m.to_sph(Kc.data(), K);
    });
}

int qcg_one_electron_batch(qcg_handle* h, const int* mol_natom, const double* Z, const double* R, double* S,
                           double* T, double* V)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(mol_natom && Z && R && S && T && V, "null argument");
        std::vector<int> atom0(h->nmol), nat(mol_natom, mol_natom + h->nmol);
        int total = 0;
        for (int m = 0; m < h->nmol; ++m)
        {
            require(nat[m] > 0, "every molecule needs at least one nucleus");
            atom0[m] = total;
            total += nat[m];
        }
        std::vector<double> z(Z, Z + total), r(R, R + 3 * total);
        for (double x : r) require(std::isfinite(x), "non-finite nuclear position", QCG_ERR_NONFINITE);
        // shell pairs (a >= b) within each molecule
        std::vector<int2> pairs;
        for (int a = 0; a < h->nshell; ++a)
            for (int b = h->mol_shell0[h->shell_mol[a]]; b <= a; ++b) pairs.push_back(int2{a, b});
        const size_t nn = (size_t)h->packed;
        double* dZ = h->upload(z);
        double* dR = h->upload(r);
        int* dA0 = h->upload(atom0);
        int* dNA = h->upload(nat);
        int2* dP = h->upload(pairs);
        int* dSM = h->nmol > 1 ? h->d_shell_mol : h->upload(std::vector<int>(h->nshell, 0));
        std::vector<long long> off1 = {0, (long long)nn};
        std::vector<int> n1 = {h->nbf};
        long long* dOff = h->nmol > 1 ? h->d_mol_off : h->upload(off1);
        int* dN = h->nmol > 1 ? h->d_mol_n : h->upload(n1);
        double* dS = h->alloc<double>(nn);
        double* dT = h->alloc<double>(nn);
        double* dV = h->alloc<double>(nn);
        launch_one_electron(h->bs, h->d_f0, h->nbf, total, dZ, dR, dS, dT, dV, h->d_boys, h->stream, h->nsm, dP,
                            (long long)pairs.size(), dSM, MolLayoutDev{std::max(h->nmol, 2), dOff, dN}, dA0, dNA);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(S, dS, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(T, dT, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(V, dV, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        for (void* p : {(void*)dZ, (void*)dR, (void*)dA0, (void*)dNA, (void*)dP, (void*)dS, (void*)dT, (void*)dV})
            h->release(p);
        if (h->nmol == 1)
            for (void* p : {(void*)dSM, (void*)dOff, (void*)dN}) h->release(p);
        if (e != cudaSuccess) throw Error{QCG_ERR_CUDA, std::string("one-electron integrals: ") + cudaGetErrorString(e)};
    });
}

void qcg_scf_default_params(qcg_scf_params* p)
{
    if (!p) return;
    p->max_iter = 100;
    p->de_tol = 1e-10;
    p->fd_tol = 1e-5;
    p->schwarz_thresh = 1e-10;
    p->diis_nproj = 4;
    p->diis_fdmax = 0.0;
    p->diis_svtol = 5e-9;
    p->incremental = 0;
    p->inc_thresh = 1e-11;
    p->rebuild_every = 8;
    p->fp32_early = 0;
    p->fp32_switch = 1e-5;
    p->fp32_scale = 0.0;
    p->fp32_below = 0.0;
    p->D_guess = nullptr;
    p->autotune = 0;
    p->spherical = 0;
    p->deterministic = 0;
}

// Closed-shell SCF (SCFIterator.C:283-362 loop; DIIS gating/pruning per SCFAcceleratorDIIS.C:35-238)
int qcg_rhf(qcg_handle* h, int natom, const double* Z, const double* R, int nelec, const qcg_scf_params* params,
            qcg_scf_result* result, double* D_out)
{
    if (!h) return QCG_ERR_ARG;
    bool converged = false;
    int rc = guarded(h, [&] {
        auto t0 = std::chrono::steady_clock::now();
        qcg_scf_params prm;
        qcg_scf_default_params(&prm);
        if (params) prm = *params;
        require(result != nullptr, "null result");
        require(h->nmol == 1, "qcg_rhf takes a single-molecule handle (qcg_rhf_batch for several)");
        require(!prm.deterministic || (!prm.fp32_early && prm.fp32_below <= 0),
                "the deterministic SCF builds every quartet in FP64 (no fp32_early, no fp32_below)");
        const int jk_flags = QCG_JK_SKIP_VALIDATION | (prm.deterministic ? QCG_JK_DETERMINISTIC : 0);
        require(natom > 0 && Z && R, "bad nuclei");
        require(nelec > 0 && nelec % 2 == 0, "closed-shell RHF needs a positive even electron count");
        const int n = h->nbf, nocc = nelec / 2;
        require(nocc <= n, "more occupied orbitals than basis functions");
        const size_t nn = (size_t)n * n;
        double Ztot = 0, Enn = 0;
        nuclei(natom, Z, R, Ztot, Enn);
        const double fdmax = prm.diis_fdmax > 0 ? prm.diis_fdmax : Ztot * Ztot * 0.1 / 32;
        std::vector<double> S(nn), T(nn), V(nn), H(nn);
        const auto s0 = std::chrono::steady_clock::now();
        {
            int e = qcg_one_electron(h, natom, Z, R, S.data(), T.data(), V.data());
            if (e != QCG_OK) throw Error{e, h->last_error};
        }
        for (size_t k = 0; k < nn; ++k) H[k] = T[k] + V[k];
        const auto s1 = std::chrono::steady_clock::now();
        {
            int e = qcg_schwarz(h, prm.schwarz_thresh, nullptr);
            if (e != QCG_OK) throw Error{e, h->last_error};
        }
        const auto s2 = std::chrono::steady_clock::now();
        ensure_jk_buffers(h);
        // spherical basis: the SCF runs on T^T S T, T^T H T; every build takes D_cart = T D T^T and returns
        // T^T J T, T^T K T (the reference's PG_Spherical path: same Cartesian kernels, transformed)
        std::unique_ptr<SphericalMap> sph;
        int nw = n;
        if (prm.spherical)
        {
            require(prm.incremental == 0, "the spherical SCF uses full builds (incremental = 0)");
            sph = std::make_unique<SphericalMap>();
            sph->build(h, S);
            nw = sph->ns;
            require(nocc <= nw, "more occupied orbitals than spherical basis functions");
            std::vector<double> Ss((size_t)nw * nw), Hs((size_t)nw * nw);
            sph->to_sph(S.data(), Ss.data());
            sph->to_sph(H.data(), Hs.data());
            S = std::move(Ss);
            H = std::move(Hs);
        }
        ScfCore sc;
        std::unique_ptr<GpuLinalg> gl;
        if (nw >= gpu_linalg_min())
        {
            gl = std::make_unique<GpuLinalg>(h->stream);
            sc.gl = gl.get();
        }
        sc.init(nw, nocc, std::move(S), std::move(H), fdmax, Enn, prm.D_guess);
        const auto s3 = std::chrono::steady_clock::now();
        std::vector<double>& D = sc.D;
        std::vector<double> J(nn), K(nn);
        // the density goes up and J, K come back every iteration: through pinned (cached) host arrays
        PinnedArray Dpin(nn), Jpin(nn), Kpin(nn);
        std::vector<double> Dc(sph ? nn : 0), Js(sph ? (size_t)nw * nw : 0), Ks(sph ? (size_t)nw * nw : 0);
        std::vector<double> Dprev, Jprev, Kprev;
        double fock_ms = 0;
        const bool inc = prm.incremental != 0;
        int since_full = 0, nfull = 0, ninc = 0, n32 = 0;
        bool force_full = true;
        // the final phase of an incremental SCF: full builds once |dE| is within 1000x the tolerance.  Each
        // density-screened build adds its own small error (skipped quartets below inc_thresh), about 1e-8 Eh
        // at 456 functions of this even-tempered basis, which would keep |dE| above de_tol for good.
        bool inc_final = false;
        // precision schedule: until the DIIS error first falls below fp32_switch, quartets whose density-
        // weighted bound is below fp32_scale * (previous DIIS error) are FP32; then FP64 (quartets below
        // fp32_below still FP32).  The build that confirms convergence is always all-FP64.  A quartet's FP32
        // error is about 3e-7 of its bound and up to ~nbf^2 quartets add into one Fock element, with the
        // same sign in the worst case (early densities of diffuse bases have entries of 1e4 and more that
        // cancel in the sums), so the default scale keeps nbf^2 * 3e-7 * bound at 1e-4 of the DIIS error.
        // (At 1e-2 the early, oscillating iterations of the even-tempered water dimer were perturbed into a
        // two-cycle that never converged; at 1e-3 and below every tested SCF kept its FP64 trajectory.)
        bool fp32_phase = prm.fp32_early != 0, exact_next = false;
        const double fp32_scale = prm.fp32_scale > 0 ? prm.fp32_scale : 1e-4 / (3e-7 * (double)n * n);
        double En_prev = 1.0;
        // QCG_SCF_TRACE=1: one line per iteration on stderr (energy, change, DIIS error, build kind);
        // QCG_SCF_TRACE=2 adds the host wall time of the iteration's phases (enqueue of the upload and the
        // build, wait for the build and the download, Fock/energy/DIIS error, DIIS step and diagonalisation)
        const char* tr = std::getenv("QCG_SCF_TRACE");
        const bool trace = tr && (tr[0] == '1' || tr[0] == '2');
        const bool trace_times = tr && tr[0] == '2';
        using clk = std::chrono::steady_clock;
        auto us = [](clk::time_point a, clk::time_point b) {
            return std::chrono::duration<double, std::micro>(b - a).count();
        };
        double t_enq = 0, t_wait = 0, t_fock = 0, t_step = 0;
        double* d_dmax = nullptr;
        if (inc) d_dmax = h->alloc<double>((size_t)h->nshell * h->nshell);
        int it;
        for (it = 1; it <= prm.max_iter; ++it)
        {
            const auto c0 = clk::now();
            qcg_stats st{};
            const bool full = !inc || inc_final || force_full || since_full >= prm.rebuild_every || exact_next;
            const double band = exact_next ? 0.0 : (fp32_phase ? fp32_scale * En_prev : prm.fp32_below);
            exact_next = false;
            if (band > 0) ++n32;
            if (full)
            {
                const double* Dup = D.data();
                if (sph)
                {
                    sph->to_cart(D.data(), Dc.data());
                    Dup = Dc.data();
                }
                std::copy(Dup, Dup + nn, Dpin.p);
                CK(cudaMemcpyAsync(h->d_D, Dpin.p, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
                if (it == 1 && prm.autotune)
                {
                    const int e = qcg_autotune_jk(h, h->d_D, 1, nullptr, nullptr);
                    if (e != QCG_OK) throw Error{e, h->last_error};
                }
                jk_device(h, h->d_D, h->d_J, h->d_K, jk_flags, &st, nullptr, 0.0, band);
            }
            else
            {
                for (size_t k = 0; k < nn; ++k) Dpin.p[k] = D[k] - Dprev[k];
                CK(cudaMemcpyAsync(h->d_D, Dpin.p, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
                launch_block_max(h->d_D, h->d_f0, h->bs.L, h->nshell, n, d_dmax, h->stream, h->nsm);
                jk_device(h, h->d_D, h->d_J, h->d_K, jk_flags, &st, d_dmax, prm.inc_thresh, band);
            }
            const auto c1 = clk::now();
            CK(cudaMemcpyAsync(Jpin.p, h->d_J, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(Kpin.p, h->d_K, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            check_team_error(h);
            std::copy(Jpin.p, Jpin.p + nn, J.begin());
            std::copy(Kpin.p, Kpin.p + nn, K.begin());
            const auto c2 = clk::now();
            fock_ms += st.ms_total;
            if (full)
            {
                since_full = 0;
                force_full = false;
                ++nfull;
            }
            else
            {
                for (size_t k = 0; k < nn; ++k) { J[k] += Jprev[k]; K[k] += Kprev[k]; }
                ++since_full;
                ++ninc;
            }
            if (inc) { Dprev = D; Jprev = J; Kprev = K; }
            if (sph)
            {
                sph->to_sph(J.data(), Js.data());
                sph->to_sph(K.data(), Ks.data());
                sc.fock(Js.data(), Ks.data());
            }
            else
                sc.fock(J.data(), K.data());
            const auto c3 = clk::now();
            t_enq += us(c0, c1);
            t_wait += us(c1, c2);
            t_fock += us(c2, c3);
            if (it > 1 && std::fabs(sc.E - sc.Eold) < prm.de_tol && sc.En < prm.fd_tol)
            {
                if (!full || band != 0.0)
                {
                    // confirm on a full all-FP64 build before stopping
                    force_full = true;
                    exact_next = true;
                    fp32_phase = false;
                }
                else
                {
                    converged = true;
                    break;
                }
            }
            if (trace)
                std::fprintf(stderr, "qcg_rhf it %3d  E %.12f  dE %+.3e  [F,D] %.3e  %s  fp32 below %.2e\n", it, sc.E,
                             sc.E - sc.Eold, sc.En, full ? "full" : "incr", band);
            En_prev = sc.En;
            if (inc && !inc_final && it > 1 && std::fabs(sc.E - sc.Eold) < 1e3 * prm.de_tol)
            {
                inc_final = true;
                force_full = true;
            }
            if (fp32_phase && it > 1 && sc.En < prm.fp32_switch)
            {
                fp32_phase = false;   // FP64 from here on, starting from a full rebuild
                force_full = true;
            }
            sc.Eold = sc.E;
            const auto c4 = clk::now();
            sc.step(prm);
            t_step += us(c4, clk::now());
        }
        if (trace_times)
            std::fprintf(stderr, "qcg_rhf host times over %d iterations (us): enqueue %.0f, wait %.0f, fock %.0f, "
                         "step %.0f; device J/K %.0f; set-up and rest %.0f\n", std::min(it, prm.max_iter), t_enq,
                         t_wait, t_fock, t_step, 1e3 * fock_ms,
                         std::chrono::duration<double, std::micro>(clk::now() - t0).count() - t_enq - t_wait -
                             t_fock - t_step);
        if (trace_times)
            std::fprintf(stderr, "qcg_rhf set-up (us): one-electron %.0f, screening %.0f, orthogonaliser and guess %.0f\n",
                         us(s0, s1), us(s1, s2), us(s2, s3));
        result->energy = sc.E;
        result->e_nuc = Enn;
        result->iterations = std::min(it, prm.max_iter);
        result->converged = converged ? 1 : 0;
        result->fd_error = sc.En;
        result->fock_ms = fock_ms;
        result->full_builds = nfull;
        result->incremental_builds = ninc;
        result->fp32_builds = n32;
        if (d_dmax) h->release(d_dmax);
        result->wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (D_out) std::copy(D.begin(), D.end(), D_out);
    });
    if (rc == QCG_OK && !converged) return QCG_ERR_NOCONV;
    return rc;
}

// ------------------------------------------------------------------------------------------------
// J/K build that allocates nothing.  Its J'/K' accumulators and result flag live in this file-scope
// device array (every GPU that loads the library holds it until the process exits).  Host code must not
// hand the array's name to a kernel: on the host it is only a stand-in, so the device address is looked
// up once per device with cudaGetSymbolAddress and cached.
// ------------------------------------------------------------------------------------------------
constexpr int kNoAllocMaxNbf = 512;
constexpr size_t kNoAllocScratchDoubles = 2 * (size_t)kNoAllocMaxNbf * kNoAllocMaxNbf + 32;
static __device__ __align__(256) double qcg_noalloc_scratch[kNoAllocScratchDoubles];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_scratch[kNoAllocMaxDevices] = {};

double* noalloc_scratch_for(int device)
{
    require(device >= 0 && device < kNoAllocMaxDevices, "device index out of range");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_scratch[device])
    {
        int cur = -1;
        CK(cudaGetDevice(&cur));
        require(cur == device, "the handle's device must be the current device", QCG_ERR_STATE);
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, qcg_noalloc_scratch));
        g_noalloc_scratch[device] = (double*)p;
    }
    return g_noalloc_scratch[device];
}

// qcg_release_cache runs before a cudaDeviceReset: the array's address may change when the module is loaded
// again, so the next allocation-free call looks it up anew
void noalloc_forget_addresses()
{
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    for (double*& p : g_noalloc_scratch) p = nullptr;
}
}   // namespace

extern "C" int qcg_fock_jk_device_noalloc(qcg_handle* h, const double* d_D, double* d_J, double* d_K)
{
    if (!h) return QCG_ERR_ARG;
    return guarded(h, [&] {
        require(d_D && d_J && d_K, "null argument");
        require(h->nbf <= kNoAllocMaxNbf,
                "qcg_fock_jk_device_noalloc supports at most " + std::to_string(kNoAllocMaxNbf) +
                    " basis functions (this basis has " + std::to_string(h->nbf) + ")");
        require(h->screened, "qcg_schwarz must be called before qcg_fock_jk_device_noalloc", QCG_ERR_STATE);
        require(h->nmol == 1, "qcg_fock_jk_device_noalloc takes a single-molecule handle");
        double* scratch = noalloc_scratch_for(h->device);
        const int n = h->nbf;
        const size_t nn = (size_t)n * n;
        double* Jp = scratch;
        double* Kp = scratch + nn;
        int* flag = (int*)(scratch + 2 * nn);
        // the array keeps the previous call's contents: the accumulators must start from zero
        CK(cudaMemsetAsync(scratch, 0, (2 * nn + 1) * sizeof(double), h->stream));
        for (int k = kNumQuartetClasses - 1; k >= 0; --k)
        {
            if (h->work[k].total <= 0) continue;
            int X = 0;
            while ((X + 1) * (X + 2) / 2 <= k) ++X;
            const int Y = k - X * (X + 1) / 2;
            // the same slice and launch shape as qcg_fock_jk_device: this rank's shard (qcg_set_shard) and the
            // autotuned run and grid cap; the build is always FP64 (qcg_set_fp32_bound does not apply)
            JKWorkDev wk = h->work[k];
            wk.run = h->tuned_run[k];
            wk.cap = h->tuned_cap[k];
            wk.mol_active = h->d_mol_active;
            shard_range(h, k, wk.gbeg, wk.gend);
            if (wk.gend <= wk.gbeg) continue;
            wk.nshell = h->nshell;
            wk.pmask = h->d_pmask;
            kJKLaunchers[k](wk, h->pl_dev[X], h->pl_dev[Y], h->pp_dev, h->d_f0, d_D, Jp, Kp, n, h->d_boys, h->stream,
                            h->nsm);
        }
        CK(cudaGetLastError());
        launch_symmetrize(Jp, Kp, d_J, d_K, (long long)nn, n, MolLayoutDev{1, nullptr, nullptr}, flag, h->stream,
                          h->nsm);
        CK(cudaGetLastError());
    });
}

extern "C++" {
namespace {
// FMA peak of the current device: TFLOP/s of a pure-FMA kernel over `reps` timed launches
template <class T, class Launch>
int measure_fma_peak(int reps, double* tflops, double* ms_per_launch, Launch launch)
{
    if (!tflops || reps <= 0) return QCG_ERR_ARG;
    T* out = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int rc = QCG_OK;
    try
    {
        int dev = 0, nsm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaMalloc(&out, sizeof(T)));
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        const int blocks = nsm * 8, threads = 256, iters = 2048;
        launch(out, blocks, threads, iters, nullptr);   // warm-up
        CK(cudaEventRecord(a, nullptr));
        for (int r = 0; r < reps; ++r) launch(out, blocks, threads, iters, nullptr);
        CK(cudaEventRecord(b, nullptr));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks * reps;
        *tflops = flops / (ms * 1e-3) / 1e12;
        if (ms_per_launch) *ms_per_launch = ms / reps;
    }
    catch (const Error& e)
    {
        rc = e.code;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (out) cudaFree(out);
    return rc;
}
}   // namespace
}   // extern "C++"

int qcg_measure_fp64_peak(int reps, double* tflops, double* ms_per_launch)
{
    return measure_fma_peak<double>(reps, tflops, ms_per_launch, launch_dfma_peak);
}

int qcg_measure_fp32_peak(int reps, double* tflops, double* ms_per_launch)
{
    return measure_fma_peak<float>(reps, tflops, ms_per_launch, launch_ffma_peak);
}

int qcg_selftest_bounded_wait(long long polls, int arrive, int* gave_up, double* ms)
{
    if (!gave_up || polls <= 0) return QCG_ERR_ARG;
    int* err = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int rc = QCG_OK;
    try
    {
        CK(cudaMalloc(&err, sizeof(int)));
        CK(cudaMemset(err, 0, sizeof(int)));
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        CK(cudaEventRecord(a, nullptr));
        launch_bounded_wait_selftest(polls, arrive ? 1 : 0, err, nullptr);
        CK(cudaGetLastError());
        CK(cudaEventRecord(b, nullptr));
        CK(cudaEventSynchronize(b));
        float t = 0;
        CK(cudaEventElapsedTime(&t, a, b));
        int e = 0;
        CK(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
        *gave_up = e & 1;
        if (ms) *ms = t;
    }
    catch (const Error& e)
    {
        rc = e.code;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (err) cudaFree(err);
    return rc;
}

// Several closed-shell SCFs advanced together (one handle from qcg_basis_create_batch): every iteration is
// ONE J/K build over all molecules (the class kernels take every molecule's quartets), then each molecule's
// host step (Fock matrix, energy, DIIS, diagonalisation) runs in parallel over the molecules.  A molecule
// stops updating once it meets the convergence test; the loop ends when all have.
int qcg_rhf_batch(qcg_handle* h, const int* mol_natom, const double* Z, const double* R, const int* nelec,
                  const qcg_scf_params* params, qcg_scf_result* results, double* D_out)
{
    if (!h) return QCG_ERR_ARG;
    bool all_converged = false;
    int rc = guarded(h, [&] {
        auto t0 = std::chrono::steady_clock::now();
        qcg_scf_params prm;
        qcg_scf_default_params(&prm);
        if (params) prm = *params;
        require(mol_natom && Z && R && nelec && results, "null argument");
        const int nmol = h->nmol;
        std::vector<int> atom0(nmol + 1, 0);
        for (int m = 0; m < nmol; ++m)
        {
            require(mol_natom[m] > 0, "every molecule needs at least one nucleus");
            require(nelec[m] > 0 && nelec[m] % 2 == 0, "closed-shell RHF needs a positive even electron count");
            require(nelec[m] / 2 <= h->mol_nbf[m], "more occupied orbitals than basis functions");
            atom0[m + 1] = atom0[m] + mol_natom[m];
        }
        const size_t nn = (size_t)h->packed;
        std::vector<double> S(nn), T(nn), V(nn);
        {
            int e = qcg_one_electron_batch(h, mol_natom, Z, R, S.data(), T.data(), V.data());
            if (e != QCG_OK) throw Error{e, h->last_error};
            e = qcg_schwarz(h, prm.schwarz_thresh, nullptr);
            if (e != QCG_OK) throw Error{e, h->last_error};
        }
        ensure_jk_buffers(h);
        std::vector<ScfCore> sc(nmol);
        std::vector<std::string> err(nmol);
        std::vector<double> Enn(nmol);
        std::vector<int> done(nmol, 0), iters(nmol, 0);
#pragma omp parallel for schedule(dynamic)
        for (int m = 0; m < nmol; ++m)
        {
            try
            {
                const int n = h->mol_nbf[m];
                const size_t o = h->mol_off[m], mm = (size_t)n * n;
                double Ztot = 0;
                nuclei(mol_natom[m], Z + atom0[m], R + 3 * atom0[m], Ztot, Enn[m]);
                std::vector<double> Sm(S.begin() + o, S.begin() + o + mm), Hm(mm);
                for (size_t k = 0; k < mm; ++k) Hm[k] = T[o + k] + V[o + k];
                const double fdmax = prm.diis_fdmax > 0 ? prm.diis_fdmax : Ztot * Ztot * 0.1 / 32;
                // D_guess, when given, is packed like every batch matrix: molecule m's block at mol_off[m]
                sc[m].init(n, nelec[m] / 2, std::move(Sm), std::move(Hm), fdmax, Enn[m],
                           prm.D_guess ? prm.D_guess + o : nullptr);
            }
            catch (const Error& e)
            {
                err[m] = e.msg;
            }
        }
        for (int m = 0; m < nmol; ++m)
            if (!err[m].empty()) throw Error{QCG_ERR_ARG, "molecule " + std::to_string(m) + ": " + err[m]};
        // the packed D, J and K cross PCIe every iteration: pinned (cached) host arrays; each molecule writes
        // its next density into Dh in the parallel step
        PinnedArray Dh(nn), Jp(nn), Kp(nn);
        double* J = Jp.p;
        double* K = Kp.p;
        // converged molecules leave the J/K builds: a device flag per molecule, cleared as each converges
        struct ActiveReset
        {
            qcg_handle* h;
            int* d = nullptr;
            ~ActiveReset()
            {
                h->d_mol_active = nullptr;
                if (d) h->release(d);
            }
        } active{h};
        std::vector<int> act(nmol, 1);
        if (nmol > 1)
        {
            active.d = h->alloc<int>(nmol);
            CK(cudaMemcpyAsync(active.d, act.data(), nmol * sizeof(int), cudaMemcpyHostToDevice, h->stream));
            h->d_mol_active = active.d;
        }
#pragma omp parallel for schedule(static)
        for (int m = 0; m < nmol; ++m) std::copy(sc[m].D.begin(), sc[m].D.end(), Dh.p + h->mol_off[m]);
        double fock_ms = 0;
        int it, nconv = 0, nbuild = 0;
        for (it = 1; it <= prm.max_iter && nconv < nmol; ++it)
        {
            ++nbuild;
            qcg_stats st{};
            CK(cudaMemcpyAsync(h->d_D, Dh.p, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            if (it == 1 && prm.autotune)
            {
                const int e = qcg_autotune_jk(h, h->d_D, 1, nullptr, nullptr);
                if (e != QCG_OK) throw Error{e, h->last_error};
            }
            jk_device(h, h->d_D, h->d_J, h->d_K,
                      QCG_JK_SKIP_VALIDATION | (prm.deterministic ? QCG_JK_DETERMINISTIC : 0), &st);
            CK(cudaMemcpyAsync(J, h->d_J, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(K, h->d_K, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            check_team_error(h);
            fock_ms += st.ms_total;
#pragma omp parallel for schedule(dynamic)
            for (int m = 0; m < nmol; ++m)
            {
                if (done[m]) continue;
                try
                {
                    ScfCore& c = sc[m];
                    c.fock(J + h->mol_off[m], K + h->mol_off[m]);
                    iters[m] = it;
                    if (it > 1 && std::fabs(c.E - c.Eold) < prm.de_tol && c.En < prm.fd_tol)
                    {
                        done[m] = 1;
                        continue;
                    }
                    c.Eold = c.E;
                    c.step(prm);
                    std::copy(c.D.begin(), c.D.end(), Dh.p + h->mol_off[m]);
                }
                catch (const Error& e)
                {
                    err[m] = e.msg;
                    done[m] = 1;
                }
            }
            nconv = 0;
            bool changed = false;
            for (int m = 0; m < nmol; ++m)
            {
                if (!err[m].empty()) throw Error{QCG_ERR_NONFINITE, "molecule " + std::to_string(m) + ": " + err[m]};
                nconv += done[m];
                if (done[m] && act[m])
                {
                    act[m] = 0;
                    changed = true;
                }
            }
            // the copy is ordered before the next build on the same stream; act is not touched again until
            // the stream is synchronised after that build
            if (changed && active.d)
                CK(cudaMemcpyAsync(active.d, act.data(), nmol * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (int m = 0; m < nmol; ++m)
        {
            qcg_scf_result& r = results[m];
            r = qcg_scf_result{};
            r.energy = sc[m].E;
            r.e_nuc = Enn[m];
            r.iterations = iters[m];
            r.converged = done[m];
            r.fd_error = sc[m].En;
            r.wall_s = wall;
            r.fock_ms = fock_ms;
            r.full_builds = nbuild;
            if (D_out) std::copy(sc[m].D.begin(), sc[m].D.end(), D_out + h->mol_off[m]);
        }
        all_converged = nconv == nmol;
    });
    if (rc == QCG_OK && !all_converged) return QCG_ERR_NOCONV;
    return rc;
}

// test hook: the host eigensolver used by the SCF (not part of the public header)
int qcg_internal_syev(int n, const double* A, double* w, double* V)
{
    try
    {
        syev(n, A, w, V);
        return QCG_OK;
    }
    catch (const Error& e)
    {
        return e.code;
    }
}

// test hook: the overlap modes the SCF's orthogonaliser drops, for ascending eigenvalues w
int qcg_internal_null_modes(int n, const double* w)
{
    return overlap_null_modes(n, w);
}

// test hook: the host SCF's Cholesky orthogonaliser (1: X written; 0: S is not positive definite)
int qcg_internal_orthogonaliser(int n, const double* S, double* X)
{
    return cholesky_orthogonaliser(n, S, X) ? 1 : 0;
}

// test hook: the SCF step's partial eigensolver (the k lowest eigenpairs)
int qcg_internal_syev_lowest(int n, const double* A, int k, double* w, double* V)
{
    try
    {
        syev_lowest(n, A, k, w, V);
        return QCG_OK;
    }
    catch (const Error& e)
    {
        return e.code;
    }
}

}   // extern "C"
