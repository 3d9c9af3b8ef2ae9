// md_core.cuh -- McMurchie-Davidson building blocks for sm_100a (FP64, with an FP32 form).
//
// Per primitive quartet the work is (qchem: src/BasisSet/Molecule/Evaluators/PG_Cart_MnD/Imp/GaussianRF.C:446-483)
//   1. Boys F_0..F_L(T), T = alpha |PQ|^2, alpha = pq/(p+q)   (Internal/Boys/Imp/AuxillaryFJ.C:13-48)
//   2. Hermite Coulomb integrals R^0_{tuv}, t+u+v <= L          (Internal/MnD/Imp/RNLM.C:19-68)
//   3. Hermite expansion coefficients E^{ab}_t per direction    (PG_Cart_MnD/Internal/Imp/Hermite2.C:95-139)
//   4. ket transform X^{cd}_{tuv} = sum_{t'u'v'} (-1)^{t'+u'+v'} E^{cd}_{t'u'v'} R_{t+t',u+u',v+v'}
//      bra contraction (ab|cd) = lambda sum_{tuv} E^{ab}_{tuv} X^{cd}_{tuv},
//      lambda = 2 pi^{5/2} / (p q sqrt(p+q)) * K_ab * K_cd.
// Steps 2-4 are emitted as straight-line code per angular class by gen_md.py (gen/md_class_<k>.cuh);
// this header holds what the generated code shares: the Boys function and the primitive-pair data.
#pragma once
#include <cstdint>

namespace qcg {

__host__ __device__ constexpr int ncart(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int nherm(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }   // t+u+v <= L

// Cartesian component k of a shell with angular momentum L, PG order: for m, for l: (L-m-l, l, m)
__host__ __device__ constexpr int comp_x(int L, int k)
{
    int idx = 0;
    for (int m = 0; m <= L; ++m)
        for (int l = 0; l <= L - m; ++l, ++idx)
            if (idx == k) return L - m - l;
    return 0;
}
__host__ __device__ constexpr int comp_y(int L, int k)
{
    int idx = 0;
    for (int m = 0; m <= L; ++m)
        for (int l = 0; l <= L - m; ++l, ++idx)
            if (idx == k) return l;
    return 0;
}
__host__ __device__ constexpr int comp_z(int L, int k)
{
    int idx = 0;
    for (int m = 0; m <= L; ++m)
        for (int l = 0; l <= L - m; ++l, ++idx)
            if (idx == k) return m;
    return 0;
}

// packed index of (t,u,v), t+u+v <= L: t outer, then u, then v
__host__ __device__ constexpr int hidx(int L, int t, int u, int v)
{
    int off = 0;
    for (int tt = 0; tt < t; ++tt) off += (L - tt + 1) * (L - tt + 2) / 2;
    for (int uu = 0; uu < u; ++uu) off += (L - t - uu + 1);
    return off + v;
}

// packed index of the 1-D E coefficient E^{ij}_t, i<=LA, j<=LB, t<=i+j
__host__ __device__ constexpr int eidx(int LB, int i, int j, int t)
{
    int off = 0;
    for (int ii = 0; ii < i; ++ii)
        for (int jj = 0; jj <= LB; ++jj) off += ii + jj + 1;
    for (int jj = 0; jj < j; ++jj) off += i + jj + 1;
    return off + t;
}
__host__ __device__ constexpr int esize(int LA, int LB) { return eidx(LB, LA, LB, LA + LB) + 1; }

// 1/sqrt((2k-1)!!): the component-dependent factor of the unit-self-overlap normalisation
// (PG_Cart_MnD/Imp/PGData.C:17-33 divides by sqrt(<chi|chi>), whose component dependence is
// prod_x (2 n_x - 1)!!).
__host__ __device__ constexpr double inv_sqrt_dfact(int k)
{
    return k <= 1 ? 1.0 : (k == 2 ? 0.57735026918962576451 : (k == 3 ? 0.25819888974716112568 : 0.0));
}
__host__ __device__ constexpr double comp_norm(int L, int k)
{
    return inv_sqrt_dfact(comp_x(L, k)) * inv_sqrt_dfact(comp_y(L, k)) * inv_sqrt_dfact(comp_z(L, k));
}

// ------------------------------------------------------------------------------------------------
// Boys function.  Three branches as in AuxillaryFJ.C:13-48.  The T<12 table (121 x 23, step 0.1) is
// generated from the series definition by gen_boys_table.py and read through the read-only path.
// ------------------------------------------------------------------------------------------------
template <int JMAX>
__device__ __forceinline__ void boys(double T, const double* __restrict__ table, double (&F)[JMAX + 1])
{
    const double et = exp(-T);
    if (T < 12.0)
    {
        const int it = (int)(T * 10.0 + 0.5);
        const double dt = (double)it * 0.1 - T;
        const double* FT = table + it * 23 + JMAX;
        // Taylor: F_j(T) = sum_k F_{j+k}(T*) dt^k / k!
        double f0 = __ldg(FT), f1 = __ldg(FT + 1), f2 = __ldg(FT + 2), f3 = __ldg(FT + 3), f4 = __ldg(FT + 4),
               f5 = __ldg(FT + 5), f6 = __ldg(FT + 6);
        double dt2 = dt * dt, dt3 = dt2 * dt, dt4 = dt3 * dt, dt5 = dt4 * dt, dt6 = dt5 * dt;
        double f = f0;
        f += f1 * dt / 1.0;
        f += f2 * dt2 / 2.0;
        f += f3 * dt3 / 6.0;
        f += f4 * dt4 / 24.0;
        f += f5 * dt5 / 120.0;
        f += f6 * dt6 / 720.0;
        F[JMAX] = f;
#pragma unroll
        for (int j = JMAX - 1; j >= 0; --j) F[j] = (2 * T * F[j + 1] + et) / (2 * j + 1);
    }
    else
    {
        const double pi = 3.14159265358979323846;
        double F0;
        if (T < 30.0)
        {
            double g;
            if (T < 15.0) g = 0.4999489092 - 0.2473631686 / T + 0.321180909 / (T * T) - 0.3811559346 / (T * T * T);
            else if (T < 18.0) g = 0.4998436875 - 0.24249438 / T + 0.24642845 / (T * T);
            else if (T < 24.0) g = 0.499093162 - 0.2152832 / T;
            else g = 0.49;
            F0 = 0.5 * sqrt(pi / T) - et * g / T;
        }
        else
            F0 = 0.5 * sqrt(pi / T);
        F[0] = F0;
        const double inv2T = 1.0 / (2 * T);
#pragma unroll
        for (int j = 0; j < JMAX; ++j) F[j + 1] = ((2 * j + 1) * F[j] - et) * inv2T;
    }
}

// FP32 form of the Boys function.  FP64 is kept where the table and the downward recursion live (T < 12);
// above, the asymptotic branches are evaluated in FP32.
template <int JMAX>
__device__ __forceinline__ void boys(double T, const double* __restrict__ table, float (&F)[JMAX + 1])
{
    if (T < 12.0)
    {
        double Fd[JMAX + 1];
        boys<JMAX>(T, table, Fd);
#pragma unroll
        for (int j = 0; j <= JMAX; ++j) F[j] = (float)Fd[j];
    }
    else
    {
        const float Tf = (float)T, et = expf(-Tf), iT = 1.0f / Tf;
        float F0;
        if (Tf < 30.0f)
        {
            float g;
            if (Tf < 15.0f) g = 0.4999489092f - 0.2473631686f * iT + 0.321180909f * iT * iT - 0.3811559346f * iT * iT * iT;
            else if (Tf < 18.0f) g = 0.4998436875f - 0.24249438f * iT + 0.24642845f * iT * iT;
            else if (Tf < 24.0f) g = 0.499093162f - 0.2152832f * iT;
            else g = 0.49f;
            F0 = 0.5f * sqrtf(3.14159265358979f * iT) - et * g * iT;
        }
        else
            F0 = 0.5f * sqrtf(3.14159265358979f * iT);
        F[0] = F0;
        const float inv2T = 0.5f * iT;
#pragma unroll
        for (int j = 0; j < JMAX; ++j) F[j + 1] = ((float)(2 * j + 1) * F[j] - et) * inv2T;
    }
}

// fused multiply-add in the generated code's arithmetic type
// a load served by L2 (bypassing L1): for values this thread accumulated with red.global, which L1 does
// not see
template <class T>
__device__ __forceinline__ T ld_l2(const T* p)
{
    return __ldcg(p);
}

__device__ __forceinline__ double qfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float qfma(float a, float b, float c) { return fmaf(a, b, c); }

// Primitive-pair data: exponent sum, centre, P-A, P-B, and the prefactor K (contraction coefficients,
// radial normalisations and exp(-ab/p |AB|^2) folded together).
struct PrimPairData
{
    double p, Px, Py, Pz, PAx, PAy, PAz, PBx, PBy, PBz, K;
};

__device__ __forceinline__ PrimPairData make_prim_pair(double a, double ax, double ay, double az, double ca, double b,
                                                       double bx, double by, double bz, double cb)
{
    PrimPairData d;
    d.p = a + b;
    const double ip = 1.0 / d.p;
    d.Px = (a * ax + b * bx) * ip;
    d.Py = (a * ay + b * by) * ip;
    d.Pz = (a * az + b * bz) * ip;
    d.PAx = d.Px - ax; d.PAy = d.Py - ay; d.PAz = d.Pz - az;
    d.PBx = d.Px - bx; d.PBy = d.Py - by; d.PBz = d.Pz - bz;
    const double abx = ax - bx, aby = ay - by, abz = az - bz;
    d.K = ca * cb * exp(-a * b * ip * (abx * abx + aby * aby + abz * abz));
    return d;
}

// how a sink is handed to a __noinline__ chunk function: by reference unless the sink says it is a
// stateless value (a pointer wrapper), which then travels in registers
template <class Sink, class = void>
struct SinkArg
{
    using type = Sink&;
};
template <class Sink>
struct SinkArg<Sink, decltype((void)Sink::kByValue)>
{
    using type = Sink;
};

}   // namespace qcg
