// fock_kernels.cu -- the small kernels around the J/K build: density validation, J'/K' symmetrisation,
// and the one-electron integrals (overlap, kinetic, nuclear attraction) of the RHF Hamiltonian.
#include <algorithm>

#include "md_core.cuh"
#include "qcg_internal.h"
#include "team_sync.cuh"

namespace qcg {

// element k of a (packed) matrix: its row i, column j and the index of its transpose partner
struct ElemIdx
{
    int i, j;
    long long t;
};
__device__ __forceinline__ ElemIdx elem_index(long long k, int n, const MolLayoutDev& ml)
{
    long long base = 0;
    int nm = n;
    if (ml.nmol > 1)
    {
        int lo = 0, hi = ml.nmol;   // off[lo] <= k < off[hi]
        while (hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if (ml.off[mid] <= k) lo = mid;
            else hi = mid;
        }
        base = ml.off[lo];
        nm = ml.n[lo];
    }
    const long long r = k - base;
    ElemIdx e;
    e.i = (int)(r / nm);
    e.j = (int)(r % nm);
    e.t = base + (long long)e.j * nm + e.i;
    return e;
}

// any non-finite entry -> flag bit 1; |D_ij - D_ji| > tol*(1+|D_ij|) -> flag bit 2 (per molecule block)
__global__ void validate_density_kernel(const double* __restrict__ D, long long total, int n, MolLayoutDev ml,
                                        double tol, int* flag)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
    {
        const ElemIdx e = elem_index(k, n, ml);
        const double a = D[k];
        if (!isfinite(a)) atomicOr(flag, 1);
        else if (e.j > e.i)
        {
            const double b = D[e.t];
            if (fabs(a - b) > tol * (1.0 + fabs(a))) atomicOr(flag, 2);
        }
    }
}

// J = J' + J'^T, K = K' + K'^T (per molecule block); flags non-finite results
__global__ void symmetrize_kernel(const double* __restrict__ Jp, const double* __restrict__ Kp, double* __restrict__ J,
                                  double* __restrict__ K, long long total, int n, MolLayoutDev ml, int* flag)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
    {
        const long long t = elem_index(k, n, ml).t;
        const double jv = Jp[k] + Jp[t], kv = Kp[k] + Kp[t];
        J[k] = jv;
        K[k] = kv;
        if (!isfinite(jv) || !isfinite(kv)) atomicOr(flag, 1);
    }
}

// ------------------------------------------------------------------------------------------------
// Grouping of an ERI batch by contraction pattern (counting sort over 256 buckets): the batch kernels
// then visit quartets with equal primitive-loop shapes in the same warp.
// ------------------------------------------------------------------------------------------------
// contraction-pattern key of every quartet (primitive counts up to 4 per shell; larger ones share a bucket)
__global__ void pattern_key_kernel(BasisDev bs, const int4* __restrict__ quartets, long long nq,
                                   unsigned char* __restrict__ key, int* __restrict__ hist)
{
    __shared__ int h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x)
    {
        const int4 s = quartets[q];
        const int a = min(bs.nprim[s.x], 4) - 1, b = min(bs.nprim[s.y], 4) - 1, c = min(bs.nprim[s.z], 4) - 1,
                  d = min(bs.nprim[s.w], 4) - 1;
        const int k = ((a * 4 + b) * 4 + c) * 4 + d;
        key[q] = (unsigned char)k;
        atomicAdd(&h[k], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// exclusive scan of the 256 bucket counts (one block of 256 threads)
__global__ void pattern_scan_kernel(const int* __restrict__ hist, int* __restrict__ cursor)
{
    __shared__ int v[256];
    const int t = threadIdx.x;
    v[t] = hist[t];
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1)
    {
        const int x = t >= off ? v[t - off] : 0;
        __syncthreads();
        v[t] += x;
        __syncthreads();
    }
    cursor[t] = v[t] - hist[t];
}

__global__ void pattern_scatter_kernel(const unsigned char* __restrict__ key, long long nq, int* __restrict__ cursor,
                                       int* __restrict__ order)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x)
        order[atomicAdd(&cursor[key[q]], 1)] = (int)q;
}

void launch_pattern_sort(const BasisDev& bs, const int4* quartets, long long nq, unsigned char* key, int* hist,
                         int* cursor, int* order, cudaStream_t st, int nsm)
{
    cudaMemsetAsync(hist, 0, 256 * sizeof(int), st);
    const long long blocks = std::min<long long>((nq + 255) / 256, (long long)nsm * 8);
    pattern_key_kernel<<<(unsigned)blocks, 256, 0, st>>>(bs, quartets, nq, key, hist);
    pattern_scan_kernel<<<1, 256, 0, st>>>(hist, cursor);
    pattern_scatter_kernel<<<(unsigned)blocks, 256, 0, st>>>(key, nq, cursor, order);
}

// dmax[a*nshell+b] = max |D_mu nu| over mu in shell a, nu in shell b
__global__ void block_max_kernel(const double* __restrict__ D, const int* __restrict__ f0, const int* __restrict__ L,
                                 int nshell, int n, double* __restrict__ dmax)
{
    const long long total = (long long)nshell * nshell;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
    {
        const int a = (int)(k / nshell), b = (int)(k % nshell);
        const int na = (L[a] + 1) * (L[a] + 2) / 2, nb = (L[b] + 1) * (L[b] + 2) / 2;
        double m = 0.0;
        for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j) m = fmax(m, fabs(D[(long long)(f0[a] + i) * n + f0[b] + j]));
        dmax[k] = m;
    }
}

void launch_block_max(const double* D, const int* shell_f0, const int* shell_L, int nshell, int n, double* dmax,
                      cudaStream_t st, int nsm)
{
    block_max_kernel<<<nsm * 4, 256, 0, st>>>(D, shell_f0, shell_L, nshell, n, dmax);
}

void launch_validate(const double* D, long long total, int n, const MolLayoutDev& ml, double tol, int* flag,
                     cudaStream_t st, int nsm)
{
    validate_density_kernel<<<nsm * 4, 256, 0, st>>>(D, total, n, ml, tol, flag);
}
void launch_symmetrize(const double* Jp, const double* Kp, double* J, double* K, long long total, int n,
                       const MolLayoutDev& ml, int* flag, cudaStream_t st, int nsm)
{
    symmetrize_kernel<<<nsm * 4, 256, 0, st>>>(Jp, Kp, J, K, total, n, ml, flag);
}

// The same from deterministic accumulator pairs (JKWorkDev::det_lo): the element's and its transpose's
// words are added as integers (exactly), then scaled back, so the result is the same for every order of
// the atomic updates
__global__ void symmetrize_fixed_kernel(const unsigned long long* __restrict__ Jp,
                                        const unsigned long long* __restrict__ Kp, double* __restrict__ J,
                                        double* __restrict__ K, long long total, int n, MolLayoutDev ml, int* flag)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
    {
        const long long t = elem_index(k, n, ml).t;
        const long long jh = (long long)(Jp[k] + Jp[t]), jl = (long long)(Jp[k + total] + Jp[t + total]);
        const long long kh = (long long)(Kp[k] + Kp[t]), kl = (long long)(Kp[k + total] + Kp[t + total]);
        const double jv = (double)jh * 0x1p-30 + (double)jl * 0x1p-70;
        const double kv = (double)kh * 0x1p-30 + (double)kl * 0x1p-70;
        J[k] = jv;
        K[k] = kv;
        if (!isfinite(jv) || !isfinite(kv)) atomicOr(flag, 1);
    }
}

void launch_symmetrize_fixed(const double* Jp, const double* Kp, double* J, double* K, long long total, int n,
                             const MolLayoutDev& ml, int* flag, cudaStream_t st, int nsm)
{
    symmetrize_fixed_kernel<<<nsm * 4, 256, 0, st>>>(reinterpret_cast<const unsigned long long*>(Jp),
                                                    reinterpret_cast<const unsigned long long*>(Kp), J, K, total,
                                                    n, ml, flag);
}

// ------------------------------------------------------------------------------------------------
// One-electron integrals per shell pair (a,b), all Cartesian components, contracted and normalised.
// Follows qchem's PrimGaussian::Overlap2C / Grad2 / Nuclear (PG_Cart_MnD/Imp/GaussianRF.C:311-405):
//   S = (pi/p)^{3/2} E_ab E^{ab}_000, Grad2 per direction from E^{a+-1,b+-1}_0, T = Grad2/2,
//   V = -sum_C Z_C 2 pi/p E_ab sum_tuv E^{ab}_tuv R_tuv(p, P-C).
// Runtime loops (L <= 2): this is O(N^2 N_atoms) work, far off the hot path.
// ------------------------------------------------------------------------------------------------
namespace {
constexpr int kEM = 6;   // E tables up to i,j <= 3 (L+1 for the kinetic shifts), t <= 6

__device__ void herm1d(double a12, double PA, double PB, int la, int lb, double (&E)[4][4][kEM + 1])
{
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int t = 0; t <= kEM; ++t) E[i][j][t] = 0.0;
    E[0][0][0] = 1.0;
    for (int i = 1; i <= la; ++i)
        for (int t = 0; t <= i; ++t)
        {
            double v = 0.0;
            if (t >= 1) v = E[i - 1][0][t - 1] * a12;
            if (t <= i - 1) v += E[i - 1][0][t] * PA;
            if (t + 1 <= i - 1) v += E[i - 1][0][t + 1] * (t + 1);
            E[i][0][t] = v;
        }
    for (int i = 0; i <= la; ++i)
        for (int j = 1; j <= lb; ++j)
            for (int t = 0; t <= i + j; ++t)
            {
                double v = 0.0;
                if (t >= 1) v = E[i][j - 1][t - 1] * a12;
                if (t <= i + j - 1) v += E[i][j - 1][t] * PB;
                if (t + 1 <= i + j - 1) v += E[i][j - 1][t + 1] * (t + 1);
                E[i][j][t] = v;
            }
}

__device__ inline void comp_of(int L, int k, int& x, int& y, int& z)
{
    int idx = 0;
    for (int m = 0; m <= L; ++m)
        for (int l = 0; l <= L - m; ++l, ++idx)
            if (idx == k) { x = L - m - l; y = l; z = m; return; }
}

__device__ inline double e0(const double (&E)[4][4][kEM + 1], int i, int j)
{
    return (i < 0 || j < 0) ? 0.0 : E[i][j][0];
}
}   // namespace

// Several molecules (pairs != null): the listed shell pairs (a >= b, same molecule) only, each molecule's
// nuclei [atom0[m], atom0[m] + natoms[m]) only, results into its packed block.
__global__ void one_electron_kernel(BasisDev bs, const int* __restrict__ shell_f0, int n, int natom,
                                    const double* __restrict__ Z, const double* __restrict__ RC,
                                    double* __restrict__ S, double* __restrict__ T, double* __restrict__ V,
                                    const double* __restrict__ boys_table, const int2* __restrict__ pairs,
                                    long long npair_list, const int* __restrict__ shell_mol, MolLayoutDev ml,
                                    const int* __restrict__ atom0, const int* __restrict__ natoms)
{
    const long long npairs = pairs ? npair_list : (long long)bs.nshell * bs.nshell;
    for (long long pr = blockIdx.x * (long long)blockDim.x + threadIdx.x; pr < npairs;
         pr += (long long)gridDim.x * blockDim.x)
    {
        int sa, sb;
        if (pairs)
        {
            sa = pairs[pr].x;
            sb = pairs[pr].y;
        }
        else
        {
            sa = (int)(pr / bs.nshell);
            sb = (int)(pr % bs.nshell);
        }
        if (sb > sa) continue;
        long long base = 0;
        int ld = n, c0 = 0, c1 = natom;
        if (pairs)
        {
            const int m = shell_mol[sa];
            base = ml.off[m];
            ld = ml.n[m];
            c0 = atom0[m];
            c1 = c0 + natoms[m];
        }
        const int la = bs.L[sa], lb = bs.L[sb];
        const int na = ncart(la), nb = ncart(lb);
        double s[36], t[36], v[36];
        for (int k = 0; k < na * nb; ++k) { s[k] = 0.0; t[k] = 0.0; v[k] = 0.0; }
        const double ax = bs.cen[3 * sa], ay = bs.cen[3 * sa + 1], az = bs.cen[3 * sa + 2];
        const double bx = bs.cen[3 * sb], by = bs.cen[3 * sb + 1], bz = bs.cen[3 * sb + 2];
        for (int i = 0; i < bs.nprim[sa]; ++i)
            for (int j = 0; j < bs.nprim[sb]; ++j)
            {
                const double a = bs.alpha[bs.prim0[sa] + i], b = bs.alpha[bs.prim0[sb] + j];
                const double ca = bs.coef[bs.prim0[sa] + i], cb = bs.coef[bs.prim0[sb] + j];
                const PrimPairData d = make_prim_pair(a, ax, ay, az, 1.0, b, bx, by, bz, 1.0);   // d.K = E_ab
                const double a12 = 0.5 / d.p;
                double Ex[4][4][kEM + 1], Ey[4][4][kEM + 1], Ez[4][4][kEM + 1];
                herm1d(a12, d.PAx, d.PBx, la + 1, lb + 1, Ex);
                herm1d(a12, d.PAy, d.PBy, la + 1, lb + 1, Ey);
                herm1d(a12, d.PAz, d.PBz, la + 1, lb + 1, Ez);
                const double pi = 3.14159265358979323846;
                const double fac = pow(pi / d.p, 1.5) * d.K * ca * cb;
                // nuclear: R_tuv summed over nuclei, t+u+v <= la+lb <= 4
                const int Lt = la + lb;
                double Rs[5][5][5];
                for (int x = 0; x < 5; ++x)
                    for (int y = 0; y < 5; ++y)
                        for (int z = 0; z < 5; ++z) Rs[x][y][z] = 0.0;
                for (int c = c0; c < c1; ++c)
                {
                    const double X = d.Px - RC[3 * c], Y = d.Py - RC[3 * c + 1], Zc = d.Pz - RC[3 * c + 2];
                    double F[5];
                    boys<4>(d.p * (X * X + Y * Y + Zc * Zc), boys_table, F);
                    double Rn[5][5][5][5];   // [n][t][u][v]
                    double pw = 1.0;
                    for (int nn = 0; nn <= Lt; ++nn)
                    {
                        Rn[nn][0][0][0] = pw * F[nn];
                        pw *= -2.0 * d.p;
                    }
                    for (int nn = Lt - 1; nn >= 0; --nn)
                    {
                        const int m = Lt - nn;
                        for (int tt = 0; tt <= m; ++tt)
                            for (int uu = 0; uu <= m - tt; ++uu)
                                for (int vv = 0; vv <= m - tt - uu; ++vv)
                                {
                                    if (tt + uu + vv == 0) continue;
                                    double r;
                                    if (tt > 0)
                                        r = X * Rn[nn + 1][tt - 1][uu][vv] + (tt > 1 ? (tt - 1) * Rn[nn + 1][tt - 2][uu][vv] : 0.0);
                                    else if (uu > 0)
                                        r = Y * Rn[nn + 1][0][uu - 1][vv] + (uu > 1 ? (uu - 1) * Rn[nn + 1][0][uu - 2][vv] : 0.0);
                                    else
                                        r = Zc * Rn[nn + 1][0][0][vv - 1] + (vv > 1 ? (vv - 1) * Rn[nn + 1][0][0][vv - 2] : 0.0);
                                    Rn[nn][tt][uu][vv] = r;
                                }
                    }
                    for (int tt = 0; tt <= Lt; ++tt)
                        for (int uu = 0; uu <= Lt - tt; ++uu)
                            for (int vv = 0; vv <= Lt - tt - uu; ++vv) Rs[tt][uu][vv] += -Z[c] * Rn[0][tt][uu][vv];
                }
                const double vfac = 2.0 * pi / d.p * d.K * ca * cb;
                for (int ka = 0; ka < na; ++ka)
                    for (int kb = 0; kb < nb; ++kb)
                    {
                        int pax, pay, paz, pbx, pby, pbz;
                        comp_of(la, ka, pax, pay, paz);
                        comp_of(lb, kb, pbx, pby, pbz);
                        const double sx = e0(Ex, pax, pbx), sy = e0(Ey, pay, pby), sz = e0(Ez, paz, pbz);
                        s[ka * nb + kb] += fac * sx * sy * sz;
                        // Grad2 = txx + tyy + tzz, each from shifted overlaps (GaussianRF.C:311-343)
                        auto tdir = [&](const double (&E)[4][4][kEM + 1], int p1, int p2) {
                            return p1 * p2 * e0(E, p1 - 1, p2 - 1) - 2.0 * p1 * b * e0(E, p1 - 1, p2 + 1)
                                 - 2.0 * p2 * a * e0(E, p1 + 1, p2 - 1) + 4.0 * a * b * e0(E, p1 + 1, p2 + 1);
                        };
                        const double g2 = tdir(Ex, pax, pbx) * sy * sz + sx * tdir(Ey, pay, pby) * sz
                                        + sx * sy * tdir(Ez, paz, pbz);
                        t[ka * nb + kb] += 0.5 * fac * g2;
                        double vv = 0.0;
                        for (int tt = 0; tt <= pax + pbx; ++tt)
                            for (int uu = 0; uu <= pay + pby; ++uu)
                                for (int ww = 0; ww <= paz + pbz; ++ww)
                                    vv += Ex[pax][pbx][tt] * Ey[pay][pby][uu] * Ez[paz][pbz][ww] * Rs[tt][uu][ww];
                        v[ka * nb + kb] += vfac * vv;
                    }
            }
        const int fa = shell_f0[sa], fb = shell_f0[sb];
        for (int ka = 0; ka < na; ++ka)
            for (int kb = 0; kb < nb; ++kb)
            {
                int pax, pay, paz, pbx, pby, pbz;
                comp_of(la, ka, pax, pay, paz);
                comp_of(lb, kb, pbx, pby, pbz);
                const double nn = inv_sqrt_dfact(pax) * inv_sqrt_dfact(pay) * inv_sqrt_dfact(paz) * inv_sqrt_dfact(pbx)
                                * inv_sqrt_dfact(pby) * inv_sqrt_dfact(pbz);
                const long long i1 = base + (long long)(fa + ka) * ld + fb + kb,
                                i2 = base + (long long)(fb + kb) * ld + fa + ka;
                S[i1] = S[i2] = s[ka * nb + kb] * nn;
                T[i1] = T[i2] = t[ka * nb + kb] * nn;
                V[i1] = V[i2] = v[ka * nb + kb] * nn;
            }
    }
}

void launch_one_electron(const BasisDev& bs, const int* f0, int n, int natom, const double* Z, const double* R,
                         double* S, double* T, double* V, const double* boys, cudaStream_t st, int nsm,
                         const int2* pairs, long long npair_list, const int* shell_mol, const MolLayoutDev& ml,
                         const int* atom0, const int* natoms)
{
    one_electron_kernel<<<nsm * 2, 64, 0, st>>>(bs, f0, n, natom, Z, R, S, T, V, boys, pairs, npair_list, shell_mol,
                                                ml, atom0, natoms);
}

}   // namespace qcg

// ------------------------------------------------------------------------------------------------
// FMA throughput probe (FP64 or FP32): 8 independent dependency chains per thread, ITER fused
// multiply-adds each, full grid.  Measures the roofline denominators of the ERI kernels on the running GPU.
// ------------------------------------------------------------------------------------------------
namespace qcg {
template <class T>
__global__ void fma_peak_kernel(T* out, int iters, T a, T b)
{
    T x0 = threadIdx.x * T(1e-9), x1 = x0 + T(1e-9), x2 = x0 + T(2e-9), x3 = x0 + T(3e-9);
    T x4 = x0 + T(4e-9), x5 = x0 + T(5e-9), x6 = x0 + T(6e-9), x7 = x0 + T(7e-9);
    for (int i = 0; i < iters; ++i)
    {
#pragma unroll
        for (int k = 0; k < 16; ++k)
        {
            x0 = qfma(x0, a, b); x1 = qfma(x1, a, b); x2 = qfma(x2, a, b); x3 = qfma(x3, a, b);
            x4 = qfma(x4, a, b); x5 = qfma(x5, a, b); x6 = qfma(x6, a, b); x7 = qfma(x7, a, b);
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == T(1234.5678)) out[0] = s;   // keeps the chains alive; never true for these inputs
}

void launch_dfma_peak(double* out, int blocks, int threads, int iters, cudaStream_t st)
{
    fma_peak_kernel<double><<<blocks, threads, 0, st>>>(out, iters, 0.999999, 1e-7);
}

void launch_ffma_peak(float* out, int blocks, int threads, int iters, cudaStream_t st)
{
    fma_peak_kernel<float><<<blocks, threads, 0, st>>>(out, iters, 0.999999f, 1e-7f);
}

// The team kernels' bounded wait, run on its own: one thread initialises an mbarrier that expects one
// arrival and waits for its first phase.  With `arrive` the arrival comes first and the wait completes; without
// it nothing ever arrives, and the wait must give up after `polls` polls and say so in err (bit 0).
__global__ void bounded_wait_selftest_kernel(long long polls, int arrive, int* err)
{
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    team::mbar_init(&bar);
    team::mbar_init_fence();
    if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(team::smem_addr(&bar)) : "memory");
    if (!team::mbar_wait(&bar, 0, polls)) atomicOr(err, 1);
    team::mbar_inval(&bar);
}

void launch_bounded_wait_selftest(long long polls, int arrive, int* err, cudaStream_t st)
{
    bounded_wait_selftest_kernel<<<1, 32, 0, st>>>(polls, arrive, err);
}
}   // namespace qcg
