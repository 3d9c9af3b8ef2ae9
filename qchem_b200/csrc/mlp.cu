// mlp.cu -- the learned initial guess: a small multilayer perceptron (SiLU hidden layers, linear output)
// trained and evaluated by the kernels below.  Operands of every matrix product are rounded to BF16 and
// the products are accumulated in FP32 (FP32 master weights, Adam in FP32).  The network maps per-atom-
// pair geometry features to density-matrix blocks; it has no counterpart in the reference, whose SCF
// always starts from the core Hamiltonian (src/SCFIterator/Imp/Seed.C:70-80).
//
// Matrix products are SIMT tiles (64 x 64 outputs per 256-thread block, 4 x 4 per thread, k-slices of 16
// staged in shared memory): the whole network is ~0.4 M parameters and a training step over 10^4 rows
// is a few GFLOP, far below anything the SCF spends, so tensor-core tiles would not change a measurable
// time here.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qchem_b200.h"

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

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// C[m][n] (+)= sum_k A(m,k) B(k,n) (+ bias[n]); A(m,k) = TA ? A[k*lda+m] : A[m*lda+k],
// B(k,n) = TB ? B[n*ldb+k] : B[k*ldb+n].  Operands rounded to BF16, FP32 accumulation.
constexpr int TM = 64, TN = 64, TK = 16;
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_bf16_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                        const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                        int ldc, const float* __restrict__ bias, int accumulate)
{
    __shared__ float As[TK][TM + 4];
    __shared__ float Bs[TK][TN + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += TK)
    {
        for (int e = threadIdx.x; e < TK * TM; e += 256)
        {
            const int kk = e / TM, mm = e % TM;
            const int m = m0 + mm, k = k0 + kk;
            float v = 0.f;
            if (m < M && k < K) v = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[kk][mm] = bf16r(v);
        }
        for (int e = threadIdx.x; e < TK * TN; e += 256)
        {
            const int kk = e / TN, nn = e % TN;
            const int n = n0 + nn, k = k0 + kk;
            float v = 0.f;
            if (n < N && k < K) v = TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
            Bs[kk][nn] = bf16r(v);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk)
        {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j] + (bias ? bias[n] : 0.f);
            float* c = C + (size_t)m * ldc + n;
            *c = accumulate ? *c + v : v;
        }
    }
}

template <bool TA, bool TB>
void gemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, const float* bias,
          bool accumulate, cudaStream_t st)
{
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    gemm_bf16_kernel<TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, accumulate ? 1 : 0);
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

}   // extern "C"
