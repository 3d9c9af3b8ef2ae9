// mlp.cu -- the learned initial guess: a small multilayer perceptron (SiLU hidden layers, linear output)
// trained and evaluated by the kernels below.  Operands of every matrix product are rounded to BF16 and
// the products are accumulated in FP32 (FP32 master weights, Adam in FP32).  The network maps per-atom-
// pair geometry features to density-matrix blocks; it has no counterpart in the reference, whose SCF
// always starts from the core Hamiltonian (src/SCFIterator/Imp/Seed.C:70-80).
//
// Matrix products run on the tensor cores (tcgen05.mma, accumulators in tensor memory; see tc::gemm_kernel).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qchem_b200.h"
#include "smem_attr.h"
#include "team_sync.cuh"

namespace {

struct MlpError
{
    int code;
    std::string msg;
};

#define MCK(x)                                                                                                \
    do                                                                                                        \
    {                                                                                                         \
        cudaError_t e_ = (x);                                                                                 \
        if (e_ != cudaSuccess) throw MlpError{QCG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

// ------------------------------------------------------------------------------------------------
// Matrix products on the 5th-generation tensor cores (tcgen05), one 128 x 128 output tile per CTA:
//   C[m][n] (+)= sum_k A(m,k) B(k,n) (+ bias[n]);  A(m,k) = TA ? A[k*lda+m] : A[m*lda+k],
//   B(k,n) = TB ? B[n*ldb+k] : B[k*ldb+n].
// The 128 threads stage a 128 x 64 slice of A and of B^T into shared memory per step, rounded to BF16, in
// the K-major canonical layout without swizzle (8-row x 16-byte core matrices; rows 16 B apart, 8-row
// groups 128 B apart, the 8-element K halves of one MMA R*16 B apart for an R-row tile); one thread issues
// four tcgen05.mma (kind::f16, M = 128, N = 128, K = 16) per step with the FP32 accumulator in tensor
// memory (128 columns), and commits them to the step's mbarrier, which frees that stage two steps later.
// The epilogue reads the accumulator back with tcgen05.ld (warp w: lanes, i.e. rows, 32w..32w+31).  Long
// K (the weight gradients, K = rows) is split over CTAs, whose partial tiles are added with FP32 atomics.
// Every wait is bounded: a wait that gives up sets the error word, waits (bounded) for the MMAs in flight
// and frees the tensor memory before the CTA returns.
namespace tc {
constexpr int BM = 128, BN = 128, BK = 64, THREADS = 128, NSTAGE = 2;
constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
// two stages need 64 KB; the allocation is 96 KB so that every address a descriptor of these tiles can
// form, read either way round (LBO and SBO), stays inside it
constexpr size_t SMEM = 96 * 1024;
// instruction descriptor: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both
// K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

// shared-memory matrix descriptor: start address, leading-dimension byte offset (between the K core
// matrices), stride byte offset (between 8-row groups), all in 16-byte units; version 1 (bits 46-47);
// base offset, LBO mode and layout type (no swizzle) zero
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     qcg::team::smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Rows [r0, r0 + R) x k [k0, k0 + BK) of an operand whose element (r, k) is X[r*ld + k] (KMAJ) or
// X[k*ld + r], zero outside [0, nrows) x [0, K), rounded to BF16 into the canonical layout at dst: the
// 16-byte chunk (r, c) (k = 8c..8c+7) at byte c*R*16 + r*16.  Consecutive threads take consecutive rows, so
// that the shared-memory stores do not conflict and the loads of a non-K-major operand coalesce.
template <bool KMAJ, int R>
__device__ __forceinline__ void stage(const float* __restrict__ X, int ld, int nrows, int K, int r0, int k0,
                                      uint8_t* dst)
{
    for (int e = threadIdx.x; e < R * (BK / 8); e += THREADS)
    {
        const int r = e % R, c = e / R;
        const int gr = r0 + r, gk = k0 + 8 * c;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            v[j] = 0.f;
            if (gr < nrows && gk + j < K)
                v[j] = KMAJ ? __ldg(X + (size_t)gr * ld + gk + j) : __ldg(X + (size_t)(gk + j) * ld + gr);
        }
        uint4 u;
        __nv_bfloat162 h;
        h = __floats2bfloat162_rn(v[0], v[1]);
        u.x = *reinterpret_cast<uint32_t*>(&h);
        h = __floats2bfloat162_rn(v[2], v[3]);
        u.y = *reinterpret_cast<uint32_t*>(&h);
        h = __floats2bfloat162_rn(v[4], v[5]);
        u.z = *reinterpret_cast<uint32_t*>(&h);
        h = __floats2bfloat162_rn(v[6], v[7]);
        u.w = *reinterpret_cast<uint32_t*>(&h);
        *reinterpret_cast<uint4*>(dst + (size_t)c * R * 16 + (size_t)r * 16) = u;
    }
}

// mode 0: C = AB + bias; 1: C += AB + bias; 2: atomicAdd (split K; bias from the first split)
template <bool TA, bool TB>
__global__ void __launch_bounds__(THREADS) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                       const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                       int ldc, const float* __restrict__ bias, int mode,
                                                       int chunks_per_split, int* __restrict__ err)
{
    extern __shared__ __align__(128) uint8_t tc_smem[];
    __shared__ uint64_t bar[NSTAGE];
    __shared__ uint32_t tmem_base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nchunks = (K + BK - 1) / BK > 0 ? (K + BK - 1) / BK : 1;
    const int kc0 = blockIdx.z * chunks_per_split;
    const int nk = min(kc0 + chunks_per_split, nchunks) - kc0;   // >= 1: the host launches no empty split
    if (threadIdx.x == 0)
    {
        for (int s = 0; s < NSTAGE; ++s) qcg::team::mbar_init(&bar[s]);
        qcg::team::mbar_init_fence();
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         qcg::team::smem_addr(&tmem_base)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    bool ok = true;
    int issued = 0;   // steps whose MMAs were committed
    for (int i = 0; i < nk; ++i)
    {
        const int s = i % NSTAGE;
        uint8_t* sa = tc_smem + s * STAGE_BYTES;
        uint8_t* sb = sa + A_BYTES;
        if (i >= NSTAGE)
        {
            // the MMAs of step i - NSTAGE read this stage
            bool late = false;
            if (threadIdx.x == 0) late = !qcg::team::mbar_wait(&bar[s], (uint32_t)(((i - NSTAGE) / NSTAGE) & 1));
            if (__syncthreads_or(late))
            {
                ok = false;
                break;
            }
        }
        const int k0 = (kc0 + i) * BK;
        stage<!TA, BM>(A, lda, M, K, m0, k0, sa);
        stage<TB, BN>(B, ldb, N, K, n0, k0, sb);
        // the generic-proxy stores become visible to the tensor cores (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0)
        {
            fence_after();
            const uint32_t a0 = qcg::team::smem_addr(sa), b0 = qcg::team::smem_addr(sb);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
                mma(tmem, smem_desc(a0 + kk * 2 * BM * 16, BM * 16, 128), smem_desc(b0 + kk * 2 * BN * 16, BN * 16, 128),
                    kIdesc, (i > 0 || kk > 0) ? 1u : 0u);
            commit(&bar[s]);
        }
        issued = i + 1;
    }
    if (ok)
    {
        // the last commit covers every MMA this thread issued
        bool late = false;
        if (threadIdx.x == 0)
            late = !qcg::team::mbar_wait(&bar[(nk - 1) % NSTAGE], (uint32_t)(((nk - 1) / NSTAGE) & 1));
        ok = !__syncthreads_or(late);
    }
    else if (threadIdx.x == 0 && issued > 0)
        qcg::team::mbar_wait(&bar[(issued - 1) % NSTAGE], (uint32_t)(((issued - 1) / NSTAGE) & 1));
    fence_after();
    if (ok)
    {
        const int row = m0 + 32 * warp + lane;
        const bool add_bias = bias && blockIdx.z == 0;
        for (int c = 0; c < BN; c += 16)
        {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, r);
            if (row < M)
            {
                float* crow = C + (size_t)row * ldc;
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    const int n = n0 + c + j;
                    if (n >= N) continue;
                    const float v = __uint_as_float(r[j]) + (add_bias ? bias[n] : 0.f);
                    if (mode == 2) atomicAdd(crow + n, v);
                    else if (mode == 1) crow[n] += v;
                    else crow[n] = v;
                }
            }
        }
    }
    else if (threadIdx.x == 0)
        atomicOr(err, 1);
    fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

__global__ void zero_2d_kernel(float* __restrict__ C, int M, int N, int ldc)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < (long long)M * N) C[(e / N) * ldc + e % N] = 0.f;
}
}   // namespace tc

// the error word of the tensor-core products (bit 0: a wait for an MMA gave up); read and cleared by the
// calls that synchronise
__device__ int g_mlp_err;

template <bool TA, bool TB>
void gemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, const float* bias,
          bool accumulate, cudaStream_t st)
{
    if (M <= 0 || N <= 0) return;
    static std::atomic<unsigned long long> ready{0};
    qcg::ensure_smem(tc::gemm_kernel<TA, TB>, tc::SMEM, ready);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int tm = (M + tc::BM - 1) / tc::BM, tn = (N + tc::BN - 1) / tc::BN;
    const int nchunks = std::max(1, (K + tc::BK - 1) / tc::BK);
    // split K until about two CTAs per SM are busy, keeping at least 4 steps per split
    int splits = std::min(std::max(1, nchunks / 4), std::max(1, 2 * nsm / (tm * tn)));
    const int per = (nchunks + splits - 1) / splits;
    splits = (nchunks + per - 1) / per;   // no empty split
    int mode = accumulate ? 1 : 0;
    if (splits > 1)
    {
        mode = 2;
        if (!accumulate)
            tc::zero_2d_kernel<<<(unsigned)(((long long)M * N + 255) / 256), 256, 0, st>>>(C, M, N, ldc);
    }
    int* err = nullptr;
    MCK(cudaGetSymbolAddress((void**)&err, g_mlp_err));
    dim3 grid(tn, tm, splits);
    tc::gemm_kernel<TA, TB><<<grid, tc::THREADS, tc::SMEM, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, mode, per, err);
}

// reads (after the caller synchronised the stream) and clears the tensor-core error word
void check_mlp_err()
{
    int e = 0;
    MCK(cudaMemcpyFromSymbol(&e, g_mlp_err, sizeof(int)));
    if (!e) return;
    const int zero = 0;
    MCK(cudaMemcpyToSymbol(g_mlp_err, &zero, sizeof(int)));
    throw MlpError{QCG_ERR_CUDA, "MLP matrix product: a wait for the tensor cores gave up; the results are not valid"};
}

__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + __expf(-z)); }

__global__ void silu_kernel(const float* __restrict__ z, float* __restrict__ y, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = z[i] * sigmoid(z[i]);
}

// dz = dy * silu'(z), silu'(z) = s (1 + z (1 - s)), s = sigmoid(z)
__global__ void silu_back_kernel(const float* __restrict__ z, float* __restrict__ d, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const float s = sigmoid(z[i]);
        d[i] *= s * (1.f + z[i] * (1.f - s));
    }
}

// masked mean-squared error: dy = 2 mask (y - t) / sum(mask); loss partial sums into acc[0], mask sum in acc[1]
__global__ void mask_sum_kernel(const float* __restrict__ mask, long long n, float* acc)
{
    float s = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += mask[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc + 1, s);
}

__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ mask,
                                long long n, float* __restrict__ dy, float* acc)
{
    const float inv = acc[1] > 0.f ? 1.f / acc[1] : 0.f;
    float s = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const float r = mask[i] * (y[i] - t[i]);
        s += r * r;
        dy[i] = 2.f * r * inv;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s * inv);
}

// db[o] = sum_rows d[row][o]
__global__ void colsum_kernel(const float* __restrict__ d, int rows, int cols, float* __restrict__ db)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += d[(size_t)r * cols + o];
    db[o] = s;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            long long n, float lr, float b1, float b2, float eps, float wd, float c1, float c2)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const float gi = g[i];
        m[i] = b1 * m[i] + (1.f - b1) * gi;
        v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
        const float mh = m[i] / c1, vh = v[i] / c2;
        p[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
    }
}

int grid_1d(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 8); }

}   // namespace

struct qcg_mlp
{
    std::vector<int> w;          // widths: w[0] inputs ... w[L] outputs
    std::vector<size_t> woff, boff;
    long long nparam = 0;
    float *d_p = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr, *d_acc = nullptr;
    // activations for training: X[l] input of layer l (rows x w[l]), Z[l] pre-activation (rows x w[l+1])
    int cap_rows = 0;
    std::vector<float*> X, Z;
    float *d_dA = nullptr, *d_dB = nullptr;
    int adam_t = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;

    int L() const { return (int)w.size() - 1; }
    int maxw() const
    {
        int m = 0;
        for (int x : w) m = std::max(m, x);
        return m;
    }
    void free_acts()
    {
        for (float* p : X) cudaFree(p);
        for (float* p : Z) cudaFree(p);
        X.clear();
        Z.clear();
        cudaFree(d_dA);
        cudaFree(d_dB);
        d_dA = d_dB = nullptr;
        cap_rows = 0;
    }
    void ensure_rows(int rows)
    {
        if (rows <= cap_rows) return;
        free_acts();
        X.resize(L() + 1, nullptr);
        Z.resize(L(), nullptr);
        for (int l = 0; l <= L(); ++l) MCK(cudaMalloc(&X[l], (size_t)rows * w[l] * sizeof(float)));
        for (int l = 0; l < L(); ++l) MCK(cudaMalloc(&Z[l], (size_t)rows * w[l + 1] * sizeof(float)));
        MCK(cudaMalloc(&d_dA, (size_t)rows * maxw() * sizeof(float)));
        MCK(cudaMalloc(&d_dB, (size_t)rows * maxw() * sizeof(float)));
        cap_rows = rows;
    }
    ~qcg_mlp()
    {
        free_acts();
        cudaFree(d_p);
        cudaFree(d_g);
        cudaFree(d_m);
        cudaFree(d_v);
        cudaFree(d_acc);
    }
    // forward over `rows`; keeps X/Z for a backward pass; output in X[L]
    void forward(int rows, const float* d_x)
    {
        ensure_rows(rows);
        MCK(cudaMemcpyAsync(X[0], d_x, (size_t)rows * w[0] * sizeof(float), cudaMemcpyDeviceToDevice, stream));
        for (int l = 0; l < L(); ++l)
        {
            const int in = w[l], out = w[l + 1];
            float* zt = (l + 1 < L()) ? Z[l] : X[L()];
            gemm<false, true>(rows, out, in, X[l], in, d_p + woff[l], in, zt, out, d_p + boff[l], false, stream);
            if (l + 1 < L())
                silu_kernel<<<grid_1d((long long)rows * out), 256, 0, stream>>>(Z[l], X[l + 1], (long long)rows * out);
        }
        MCK(cudaGetLastError());
    }
};

namespace {
template <class F>
int mguard(qcg_mlp* m, F&& f)
{
    try
    {
        f();
        return QCG_OK;
    }
    catch (const MlpError& e)
    {
        if (m) m->last_error = e.msg;
        return e.code;
    }
    catch (const std::bad_alloc&)
    {
        if (m) m->last_error = "host allocation failed";
        return QCG_ERR_ALLOC;
    }
}
void mrequire(bool c, const char* msg)
{
    if (!c) throw MlpError{QCG_ERR_ARG, msg};
}
}   // namespace

extern "C" {

int qcg_mlp_create(int nlayers, const int* widths, unsigned long long seed, qcg_mlp** out)
{
    if (!out) return QCG_ERR_ARG;
    *out = nullptr;
    if (nlayers < 1 || nlayers > 16 || !widths) return QCG_ERR_ARG;
    for (int l = 0; l <= nlayers; ++l)
        if (widths[l] < 1 || widths[l] > 65536) return QCG_ERR_ARG;
    auto* m = new qcg_mlp();
    int rc = mguard(m, [&] {
        int dev = 0;
        MCK(cudaGetDevice(&dev));
        MCK(cudaFree(nullptr));
        m->w.assign(widths, widths + nlayers + 1);
        size_t off = 0;
        for (int l = 0; l < nlayers; ++l)
        {
            m->woff.push_back(off);
            off += (size_t)m->w[l + 1] * m->w[l];
            m->boff.push_back(off);
            off += (size_t)m->w[l + 1];
        }
        m->nparam = (long long)off;
        // Kaiming-uniform weights for SiLU layers, zero biases; deterministic in `seed`
        std::vector<float> h(off, 0.f);
        std::mt19937_64 rng(seed);
        for (int l = 0; l < nlayers; ++l)
        {
            const float bound = std::sqrt(6.f / (float)m->w[l]) * (l + 1 < nlayers ? 1.f : 0.5f);
            std::uniform_real_distribution<float> U(-bound, bound);
            for (size_t k = 0; k < (size_t)m->w[l + 1] * m->w[l]; ++k) h[m->woff[l] + k] = U(rng);
        }
        MCK(cudaMalloc(&m->d_p, off * sizeof(float)));
        MCK(cudaMalloc(&m->d_g, off * sizeof(float)));
        MCK(cudaMalloc(&m->d_m, off * sizeof(float)));
        MCK(cudaMalloc(&m->d_v, off * sizeof(float)));
        MCK(cudaMalloc(&m->d_acc, 2 * sizeof(float)));
        MCK(cudaMemcpy(m->d_p, h.data(), off * sizeof(float), cudaMemcpyHostToDevice));
        MCK(cudaMemset(m->d_g, 0, off * sizeof(float)));
        MCK(cudaMemset(m->d_m, 0, off * sizeof(float)));
        MCK(cudaMemset(m->d_v, 0, off * sizeof(float)));
    });
    if (rc != QCG_OK)
    {
        delete m;
        return rc;
    }
    *out = m;
    return QCG_OK;
}

void qcg_mlp_destroy(qcg_mlp* m) { delete m; }

const char* qcg_mlp_last_error(const qcg_mlp* m) { return m ? m->last_error.c_str() : "null mlp"; }

int qcg_mlp_set_stream(qcg_mlp* m, void* stream)
{
    if (!m) return QCG_ERR_ARG;
    m->stream = (cudaStream_t)stream;
    return QCG_OK;
}

int qcg_mlp_nparams(const qcg_mlp* m, long long* n)
{
    if (!m || !n) return QCG_ERR_ARG;
    *n = m->nparam;
    return QCG_OK;
}

int qcg_mlp_params(qcg_mlp* m, float* host)
{
    if (!m || !host) return QCG_ERR_ARG;
    return mguard(m, [&] {
        MCK(cudaMemcpyAsync(host, m->d_p, m->nparam * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        MCK(cudaStreamSynchronize(m->stream));
    });
}

int qcg_mlp_set_params(qcg_mlp* m, const float* host)
{
    if (!m || !host) return QCG_ERR_ARG;
    return mguard(m, [&] {
        for (long long k = 0; k < m->nparam; ++k) mrequire(std::isfinite(host[k]), "non-finite parameter");
        MCK(cudaMemcpyAsync(m->d_p, host, m->nparam * sizeof(float), cudaMemcpyHostToDevice, m->stream));
        MCK(cudaStreamSynchronize(m->stream));
        m->adam_t = 0;
        MCK(cudaMemsetAsync(m->d_m, 0, m->nparam * sizeof(float), m->stream));
        MCK(cudaMemsetAsync(m->d_v, 0, m->nparam * sizeof(float), m->stream));
    });
}

int qcg_mlp_forward(qcg_mlp* m, int rows, const float* d_x, float* d_y)
{
    if (!m) return QCG_ERR_ARG;
    return mguard(m, [&] {
        mrequire(rows >= 0, "negative row count");
        if (rows == 0) return;
        mrequire(d_x && d_y, "null argument");
        m->forward(rows, d_x);
        MCK(cudaMemcpyAsync(d_y, m->X[m->L()], (size_t)rows * m->w.back() * sizeof(float), cudaMemcpyDeviceToDevice,
                            m->stream));
    });
}

int qcg_mlp_loss_grad(qcg_mlp* m, int rows, const float* d_x, const float* d_t, const float* d_mask, float* loss,
                      float* grad_host)
{
    if (!m) return QCG_ERR_ARG;
    return mguard(m, [&] {
        mrequire(rows > 0 && d_x && d_t && d_mask, "bad argument");
        m->forward(rows, d_x);
        const int L = m->L(), nout = m->w[L];
        const long long ny = (long long)rows * nout;
        MCK(cudaMemsetAsync(m->d_acc, 0, 2 * sizeof(float), m->stream));
        mask_sum_kernel<<<grid_1d(ny), 256, 0, m->stream>>>(d_mask, ny, m->d_acc);
        float* dcur = m->d_dA;   // gradient w.r.t. the current layer's output (pre-activation)
        float* dnext = m->d_dB;
        mse_grad_kernel<<<grid_1d(ny), 256, 0, m->stream>>>(m->X[L], d_t, d_mask, ny, dcur, m->d_acc);
        for (int l = L - 1; l >= 0; --l)
        {
            const int in = m->w[l], out = m->w[l + 1];
            if (l + 1 < L)
                silu_back_kernel<<<grid_1d((long long)rows * out), 256, 0, m->stream>>>(m->Z[l], dcur,
                                                                                        (long long)rows * out);
            // dW = dZ^T X  ([out x rows] [rows x in]),  db = column sums of dZ,  dX = dZ W
            gemm<true, false>(out, in, rows, dcur, out, m->X[l], in, m->d_g + m->woff[l], in, nullptr, false,
                              m->stream);
            colsum_kernel<<<(out + 255) / 256, 256, 0, m->stream>>>(dcur, rows, out, m->d_g + m->boff[l]);
            if (l > 0)
            {
                gemm<false, false>(rows, in, out, dcur, out, m->d_p + m->woff[l], in, dnext, in, nullptr, false,
                                   m->stream);
                std::swap(dcur, dnext);
            }
        }
        MCK(cudaGetLastError());
        float acc[2] = {0, 0};
        MCK(cudaMemcpyAsync(acc, m->d_acc, 2 * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        if (grad_host)
            MCK(cudaMemcpyAsync(grad_host, m->d_g, m->nparam * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        MCK(cudaStreamSynchronize(m->stream));
        check_mlp_err();
        if (loss) *loss = acc[0];
    });
}

int qcg_mlp_adam(qcg_mlp* m, float lr, float beta1, float beta2, float eps, float weight_decay)
{
    if (!m) return QCG_ERR_ARG;
    return mguard(m, [&] {
        mrequire(lr >= 0 && beta1 >= 0 && beta1 < 1 && beta2 >= 0 && beta2 < 1 && eps > 0, "bad Adam parameters");
        ++m->adam_t;
        const float c1 = 1.f - std::pow(beta1, (float)m->adam_t), c2 = 1.f - std::pow(beta2, (float)m->adam_t);
        adam_kernel<<<grid_1d(m->nparam), 256, 0, m->stream>>>(m->d_p, m->d_g, m->d_m, m->d_v, m->nparam, lr, beta1,
                                                                beta2, eps, weight_decay, c1, c2);
        MCK(cudaGetLastError());
    });
}

// test hook (not part of the public header): C (+)= op(A) op(B) (+ bias) on device pointers through the
// tensor-core product above, synchronous; ta/tb select the transposed operand forms
int qcg_internal_gemm_bf16(int ta, int tb, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                           float* C, int ldc, const float* bias, int accumulate)
{
    try
    {
        if (M < 0 || N < 0 || K < 0 || (K > 0 && (!A || !B)) || (M > 0 && N > 0 && !C)) return QCG_ERR_ARG;
        const bool acc = accumulate != 0;
        if (ta && tb) gemm<true, true>(M, N, K, A, lda, B, ldb, C, ldc, bias, acc, nullptr);
        else if (ta) gemm<true, false>(M, N, K, A, lda, B, ldb, C, ldc, bias, acc, nullptr);
        else if (tb) gemm<false, true>(M, N, K, A, lda, B, ldb, C, ldc, bias, acc, nullptr);
        else gemm<false, false>(M, N, K, A, lda, B, ldb, C, ldc, bias, acc, nullptr);
        MCK(cudaGetLastError());
        MCK(cudaDeviceSynchronize());
        check_mlp_err();
        return QCG_OK;
    }
    catch (const MlpError& e)
    {
        return e.code;
    }
}

}   // extern "C"
