// host_md.cpp -- test harness: the generated straight-line McMurchie-Davidson code of ONE quartet class
// (qchem_b200/csrc/gen/md_class_<k>.cuh, written by gen_md.py) compiled for the host CPU, so that the
// code generator's arithmetic is checked against the oracle without a GPU.  Not part of the library: the
// CUDA qualifiers are mapped to plain C++ and __ldg to a load.  Build (see tests/test_gen_md_host.py):
//   g++ -std=c++17 -O1 -fPIC -shared -DQCG_CLASS=<k> -I qchem_b200/csrc host_md.cpp -o host_md_<k>.so
#include <cmath>
#include <cstdint>
#include <vector>

#define __host__
#define __device__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
template <class T>
static inline T __ldg(const T* p)
{
    return *p;
}
template <class T>
static inline T __ldcg(const T* p)
{
    return *p;
}
static inline void __syncthreads() {}   // the lock-step variant is not instantiated here

#include "md_core.cuh"
#include "boys_table.h"

#define HM_STR2(x) #x
#define HM_STR(x) HM_STR2(x)
#define HM_CAT2(a, b) a##b
#define HM_CAT(a, b) HM_CAT2(a, b)
#include HM_STR(gen/HM_CAT(md_class_, QCG_CLASS).cuh)

namespace {

// output accumulation into one quartet's block [a][b][c][d] (by value, like the library's store sink), in
// the arithmetic type of the evaluation
template <class RT>
struct HostSink
{
    static constexpr bool kByValue = true;
    RT* o;
    int nb, nc, nd;
    void ket_begin(int, int) {}
    void ket_end(int, int) {}
    void operator()(int ia, int ib, int ic, int id, RT v) { o[((ia * nb + ib) * nc + ic) * nd + id] += v; }
};

double dfact(int i)
{
    double r = 1;
    for (int k = i; k > 1; k -= 2) r *= k;
    return r;
}

// the library's contraction preprocessing: the (L,0,0) primitive norm folded into each coefficient, then
// the shell scaled to unit radial self-overlap (the component factors are applied by the generated code)
std::vector<double> shell_coefs(int L, int np, const double* a, const double* c)
{
    const double pi = 3.14159265358979323846;
    std::vector<double> w(np);
    for (int i = 0; i < np; ++i)
        w[i] = c[i] * std::sqrt(std::pow(4 * a[i], L) / (std::pow(pi / (2 * a[i]), 1.5) * dfact(2 * L - 1)));
    double ss = 0;
    for (int i = 0; i < np; ++i)
        for (int j = 0; j < np; ++j)
        {
            const double p = a[i] + a[j];
            ss += w[i] * w[j] * std::pow(pi / p, 1.5) / std::pow(2 * p, L);
        }
    for (double& x : w) x /= std::sqrt(ss);
    return w;
}

}   // namespace

extern "C" int host_md_class() { return QCG_CLASS; }

// nq quartets; shell s of quartet q is row 4q+s of the inputs: L, primitive count (<= 8), exponents and raw
// coefficients (8 slots each), centre (3).  out: nq blocks of ncart(la) ncart(lb) ncart(lc) ncart(ld).
template <class RT>
int host_eri(long long nq, const int* L, const int* np, const double* exps, const double* coefs, const double* cen,
             RT* out)
{
    std::vector<RT> rs(qcg::nherm(16));
    for (long long q = 0; q < nq; ++q)
    {
        int l[4], n[4];
        std::vector<double> w[4];
        for (int s = 0; s < 4; ++s)
        {
            const long long r = 4 * q + s;
            l[s] = L[r];
            n[s] = np[r];
            if (n[s] < 1 || n[s] > 8) return 1;
            w[s] = shell_coefs(l[s], n[s], exps + 8 * r, coefs + 8 * r);
        }
        const int nb = qcg::ncart(l[1]), nc = qcg::ncart(l[2]), nd = qcg::ncart(l[3]);
        RT* o = out + q * (long long)qcg::ncart(l[0]) * nb * nc * nd;
        for (int k = 0; k < qcg::ncart(l[0]) * nb * nc * nd; ++k) o[k] = RT(0);
        HostSink<RT> sink{o, nb, nc, nd};
        const double* c0 = cen + 12 * q;
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
            {
                const qcg::PrimPairData pab = qcg::make_prim_pair(
                    exps[8 * (4 * q) + i], c0[0], c0[1], c0[2], w[0][i], exps[8 * (4 * q + 1) + j], c0[3], c0[4],
                    c0[5], w[1][j]);
                for (int k = 0; k < n[2]; ++k)
                    for (int m = 0; m < n[3]; ++m)
                    {
                        const qcg::PrimPairData pcd = qcg::make_prim_pair(
                            exps[8 * (4 * q + 2) + k], c0[6], c0[7], c0[8], w[2][k], exps[8 * (4 * q + 3) + m],
                            c0[9], c0[10], c0[11], w[3][m]);
                        HM_CAT(qcg::gen::prim_quartet_, QCG_CLASS)<RT, HostSink<RT>>(pab, pcd, kBoysTable,
                                                                                    rs.data(), 1, sink);
                    }
            }
    }
    return 0;
}

extern "C" int host_md_eri(long long nq, const int* L, const int* np, const double* exps, const double* coefs,
                           const double* cen, double* out)
{
    return host_eri<double>(nq, L, np, exps, coefs, cen, out);
}

// the FP32 form: the same generated code with float arithmetic (pair data and Boys for T < 12 in FP64)
extern "C" int host_md_eri_f32(long long nq, const int* L, const int* np, const double* exps, const double* coefs,
                               const double* cen, float* out)
{
    return host_eri<float>(nq, L, np, exps, coefs, cen, out);
}

#ifdef HM_HRR
// The HRR form of the same class (gen_md.main_hrr writes gen_hrr/md_hrr_<k>.cuh): [e0|f0] accumulated over
// the primitive quartets, then the ket recurrence per e row and the bra recurrence per (c d) column.
#include HM_STR(gen_hrr/HM_CAT(md_hrr_, QCG_CLASS).cuh)

namespace {
template <class RT>
struct HrrSink
{
    RT* p;
    int nf;
    void operator()(int ie, int jf, RT v) { p[ie * nf + jf] += v; }
};
}   // namespace

template <class RT>
int host_eri_hrr(long long nq, const int* L, const int* np, const double* exps, const double* coefs,
                 const double* cen, RT* out)
{
    constexpr int NE = HM_CAT(qcg::gen::kHrrE, QCG_CLASS), NF = HM_CAT(qcg::gen::kHrrF, QCG_CLASS);
    std::vector<RT> rs(qcg::nherm(16)), P((size_t)NE * NF);
    for (long long q = 0; q < nq; ++q)
    {
        int l[4], n[4];
        std::vector<double> w[4];
        for (int s = 0; s < 4; ++s)
        {
            const long long r = 4 * q + s;
            l[s] = L[r];
            n[s] = np[r];
            if (n[s] < 1 || n[s] > 8) return 1;
            w[s] = shell_coefs(l[s], n[s], exps + 8 * r, coefs + 8 * r);
        }
        const int na = qcg::ncart(l[0]), nb = qcg::ncart(l[1]), ncd = qcg::ncart(l[2]) * qcg::ncart(l[3]);
        std::vector<RT> Y((size_t)NE * ncd);
        std::fill(P.begin(), P.end(), RT(0));
        HrrSink<RT> sink{P.data(), NF};
        const double* c0 = cen + 12 * q;
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
            {
                const qcg::PrimPairData pab = qcg::make_prim_pair(
                    exps[8 * (4 * q) + i], c0[0], c0[1], c0[2], w[0][i], exps[8 * (4 * q + 1) + j], c0[3], c0[4],
                    c0[5], w[1][j]);
                for (int k = 0; k < n[2]; ++k)
                    for (int m = 0; m < n[3]; ++m)
                    {
                        const qcg::PrimPairData pcd = qcg::make_prim_pair(
                            exps[8 * (4 * q + 2) + k], c0[6], c0[7], c0[8], w[2][k], exps[8 * (4 * q + 3) + m],
                            c0[9], c0[10], c0[11], w[3][m]);
                        HM_CAT(qcg::gen::prim_quartet_hrr_, QCG_CLASS)<RT, HrrSink<RT>>(pab, pcd, kBoysTable,
                                                                                       rs.data(), 1, sink);
                    }
            }
        const RT CDx = RT(c0[6] - c0[9]), CDy = RT(c0[7] - c0[10]), CDz = RT(c0[8] - c0[11]);
        const RT ABx = RT(c0[0] - c0[3]), ABy = RT(c0[1] - c0[4]), ABz = RT(c0[2] - c0[5]);
        for (int e = 0; e < NE; ++e)
            HM_CAT(qcg::gen::hrr_ket_, QCG_CLASS)<RT>(P.data() + (size_t)e * NF, Y.data() + (size_t)e * ncd, CDx, CDy,
                                                     CDz);
        RT* o = out + q * (long long)na * nb * ncd;
        for (int cd = 0; cd < ncd; ++cd)
            HM_CAT(qcg::gen::hrr_bra_, QCG_CLASS)<RT>(Y.data() + cd, ncd, o + cd, ncd, ABx, ABy, ABz);
    }
    return 0;
}

extern "C" int host_md_eri_hrr(long long nq, const int* L, const int* np, const double* exps, const double* coefs,
                               const double* cen, double* out)
{
    return host_eri_hrr<double>(nq, L, np, exps, coefs, cen, out);
}

// the HRR form in FP32 (primitive code and both recurrences in float)
extern "C" int host_md_eri_hrr_f32(long long nq, const int* L, const int* np, const double* exps,
                                   const double* coefs, const double* cen, float* out)
{
    return host_eri_hrr<float>(nq, L, np, exps, coefs, cen, out);
}

// The data flow planned for the GPU kernel, inside each quartet's own output block (n_a n_b rows of
// n_c n_d): [e0|f0] accumulated at o[e * ncd + f], the ket recurrence in place per e row, then the bra
// recurrence in place per (c d) column.
extern "C" int host_md_eri_hrr_inplace(long long nq, const int* L, const int* np, const double* exps,
                                       const double* coefs, const double* cen, double* out)
{
    constexpr int NE = HM_CAT(qcg::gen::kHrrE, QCG_CLASS), NF = HM_CAT(qcg::gen::kHrrF, QCG_CLASS);
    std::vector<double> rs(qcg::nherm(16));
    for (long long q = 0; q < nq; ++q)
    {
        int l[4], n[4];
        std::vector<double> w[4];
        for (int s = 0; s < 4; ++s)
        {
            const long long r = 4 * q + s;
            l[s] = L[r];
            n[s] = np[r];
            if (n[s] < 1 || n[s] > 8) return 1;
            w[s] = shell_coefs(l[s], n[s], exps + 8 * r, coefs + 8 * r);
        }
        const int na = qcg::ncart(l[0]), nb = qcg::ncart(l[1]), ncd = qcg::ncart(l[2]) * qcg::ncart(l[3]);
        if (NE > na * nb || NF > ncd) return 2;
        double* o = out + q * (long long)na * nb * ncd;
        for (int k = 0; k < na * nb * ncd; ++k) o[k] = 0.0;
        struct RowSink
        {
            double* o;
            int ncd;
            void operator()(int ie, int jf, double v) { o[ie * ncd + jf] += v; }
        } sink{o, ncd};
        const double* c0 = cen + 12 * q;
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
            {
                const qcg::PrimPairData pab = qcg::make_prim_pair(
                    exps[8 * (4 * q) + i], c0[0], c0[1], c0[2], w[0][i], exps[8 * (4 * q + 1) + j], c0[3], c0[4],
                    c0[5], w[1][j]);
                for (int k = 0; k < n[2]; ++k)
                    for (int m = 0; m < n[3]; ++m)
                    {
                        const qcg::PrimPairData pcd = qcg::make_prim_pair(
                            exps[8 * (4 * q + 2) + k], c0[6], c0[7], c0[8], w[2][k], exps[8 * (4 * q + 3) + m],
                            c0[9], c0[10], c0[11], w[3][m]);
                        HM_CAT(qcg::gen::prim_quartet_hrr_, QCG_CLASS)<double, RowSink>(pab, pcd, kBoysTable,
                                                                                       rs.data(), 1, sink);
                    }
            }
        for (int e = 0; e < NE; ++e)
            HM_CAT(qcg::gen::hrr_ket_, QCG_CLASS)<double>(o + (size_t)e * ncd, o + (size_t)e * ncd, c0[6] - c0[9],
                                                         c0[7] - c0[10], c0[8] - c0[11]);
        for (int cd = 0; cd < ncd; ++cd)
            HM_CAT(qcg::gen::hrr_bra_, QCG_CLASS)<double>(o + cd, ncd, o + cd, ncd, c0[0] - c0[3], c0[1] - c0[4],
                                                         c0[2] - c0[5]);
    }
    return 0;
}
#endif

#ifdef HM_TEAM
// The team form (gen_md.main_team writes gen_team/md_team_<k>.cuh): the arithmetic of eri_batch_team_kernel
// for one quartet on lane 0 of a stage, in the kernel's order -- per ket component f, over the primitive
// quartets (bra primitive pair outer, ket inner) the stage tables, the ket step into Y_f, and after the last
// ket primitive the bra step into acc_f; then [e0|f0] in a lane-minor scratch, the ket recurrence per e row
// into [e0|cd] there, and the bra recurrence per (c d) column into the output block, as the kernel does.
#include HM_STR(gen_team/HM_CAT(md_team_, QCG_CLASS).cuh)

extern "C" int host_md_eri_team(long long nq, const int* L, const int* np, const double* exps, const double* coefs,
                                const double* cen, double* out)
{
    constexpr int NE = HM_CAT(qcg::gen::kTeamNE, QCG_CLASS), NF = HM_CAT(qcg::gen::kTeamNF, QCG_CLASS);
    constexpr int NH = HM_CAT(qcg::gen::kTeamNH, QCG_CLASS), NS = HM_CAT(qcg::gen::kTeamStage, QCG_CLASS);
    std::vector<double> stage((size_t)NS * 32);
    for (long long q = 0; q < nq; ++q)
    {
        int l[4], n[4];
        std::vector<double> w[4];
        for (int s = 0; s < 4; ++s)
        {
            const long long r = 4 * q + s;
            l[s] = L[r];
            n[s] = np[r];
            if (n[s] < 1 || n[s] > 8) return 1;
            w[s] = shell_coefs(l[s], n[s], exps + 8 * r, coefs + 8 * r);
        }
        const int na = qcg::ncart(l[0]), nb = qcg::ncart(l[1]), ncd = qcg::ncart(l[2]) * qcg::ncart(l[3]);
        if (NE > na * nb || NF > ncd) return 2;
        double* o = out + q * (long long)na * nb * ncd;
        for (int k = 0; k < na * nb * ncd; ++k) o[k] = std::nan("");
        std::vector<double> hA((size_t)NE * NF * 32, std::nan("")), hB((size_t)NE * ncd * 32, std::nan(""));
        const double* c0 = cen + 12 * q;
        auto pair = [&](int s0, int i, int s1, int j) {
            return qcg::make_prim_pair(exps[8 * (4 * q + s0) + i], c0[3 * s0], c0[3 * s0 + 1], c0[3 * s0 + 2],
                                       w[s0][i], exps[8 * (4 * q + s1) + j], c0[3 * s1], c0[3 * s1 + 1],
                                       c0[3 * s1 + 2], w[s1][j]);
        };
        const int Kcd = n[2] * n[3];
        for (int jf = 0; jf < NF; ++jf)
        {
            double Y[NH] = {}, acc[NE] = {};
            for (int ij = 0; ij < n[0] * n[1]; ++ij)
            {
                const qcg::PrimPairData pab = pair(0, ij / n[1], 1, ij % n[1]);
                for (int kl = 0; kl < Kcd; ++kl)
                {
                    const qcg::PrimPairData pcd = pair(2, kl / n[3], 3, kl % n[3]);
                    std::fill(stage.begin(), stage.end(), std::nan(""));
                    HM_CAT(qcg::gen::team_produce_, QCG_CLASS)<double>(stage.data(), pab, pcd, kBoysTable,
                                                                      kl == Kcd - 1);
                    HM_CAT(qcg::gen::team_ket_, QCG_CLASS)<double>(jf, stage.data(), Y);
                    if (kl == Kcd - 1)
                    {
                        HM_CAT(qcg::gen::team_bra_, QCG_CLASS)<double>(stage.data(), Y, acc);
                        for (double& y : Y) y = 0.0;
                    }
                }
            }
            for (int e = 0; e < NE; ++e) hA[(size_t)(e * NF + jf) * 32] = acc[e];
        }
        for (int e = 0; e < NE; ++e)
            HM_CAT(qcg::gen::team_hrr_ket_, QCG_CLASS)<double>(hA.data() + (size_t)e * NF * 32,
                                                              hB.data() + (size_t)e * ncd * 32, c0[6] - c0[9],
                                                              c0[7] - c0[10], c0[8] - c0[11]);
        for (int cd = 0; cd < ncd; ++cd)
            HM_CAT(qcg::gen::team_hrr_bra_, QCG_CLASS)<double>(hB.data() + (size_t)cd * 32, o + cd, ncd,
                                                              c0[0] - c0[3], c0[1] - c0[4], c0[2] - c0[5]);
    }
    return 0;
}
#endif
