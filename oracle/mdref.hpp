// mdref.hpp -- CPU restatement of qchem's McMurchie-Davidson molecular Hartree-Fock path.
//
// TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA product is checked against.  Nothing in
// the product (qchem_b200/) includes, links or calls it; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py use it, through the C API in oracle_capi.cpp.
//
// Each function cites the reference file:line it restates (paths inside JanReimers/qchem):
//   Boys F_j(T)        src/BasisSet/Molecule/Evaluators/Internal/Boys/Imp/AuxillaryFJ.C:13-48
//                      (table semantics: Imp/AuxillaryData.C:8-10, 121 rows x 23 orders, T step 0.1)
//   R_NLM recursion    src/BasisSet/Molecule/Evaluators/Internal/MnD/Imp/RNLM.C:19-68
//   Hermite E coeffs   src/BasisSet/Molecule/Evaluators/PG_Cart_MnD/Internal/Imp/Hermite2.C:95-139,158-199
//   primitive pair     src/BasisSet/Molecule/Evaluators/PG_Cart_MnD/Imp/GaussianRF.C:239-252 (Omega)
//   (ab|cd) primitive  .../PG_Cart_MnD/Imp/GaussianRF.C:446-483
//   (ab|cd) contracted .../PG_Cart_MnD/Imp/GaussianRF.C:726-752
//   primitive norms    .../PG_Cart_MnD/Imp/GaussianRF.C:512-521 (GetNormalization), :566-577 (folding)
//   ns (unit self-S)   .../PG_Cart_MnD/Imp/PGData.C:17-33
//   FourC              .../PG_Cart_MnD/Evaluator.C:1912-1920
//   overlap/grad2/nuc  .../PG_Cart_MnD/Imp/GaussianRF.C:311-405
//   component order    src/BasisSet/Molecule/PG_Cart/Imp/IrrepBasisSet.C:36-54
//   J/K element loops  src/BasisSet/Molecule/IrrepBasisSet.C:138-183, contraction Internal/Imp/ERI4.C:10-17
//   RHF energy terms   src/Hamiltonian/Internal/Imp/Hamiltonians.C:36-43, HF_HT.C:48-70, Vee.C, Vxc.C
//   DIIS               src/SCFAccelerator/Internal/Imp/SCFAcceleratorDIIS.C:35-238, src/Math/DIIS.C:24-51
//
// The Boys table is NOT copied from the reference: it is computed here from the convergent series
// F_j(T) = exp(-T) sum_k (2T)^k / ((2j+1)(2j+3)...(2j+2k+1)) in long double.  The 12<=T<30 rational
// fits g(T) and the branch points are kept identical to the reference, because parity at 1e-12 needs
// the same approximation there (the fits are only good to ~1e-11 against the exact function).
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#include <algorithm>

namespace mdref {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int kBoysRows = 121, kBoysCols = 23, kJMax = 16;

// ---------------------------------------------------------------------------------------------------
// Boys function
// ---------------------------------------------------------------------------------------------------
struct BoysTable
{
    double v[kBoysRows][kBoysCols];
    BoysTable()
    {
        for (int it = 0; it < kBoysRows; ++it)
        {
            long double T = 0.1L * it;
            for (int j = 0; j < kBoysCols; ++j)
            {
                // all-positive series: no cancellation, converges for every T
                long double term = 1.0L / (2 * j + 1), sum = term;
                for (int k = 1; k < 400; ++k)
                {
                    term *= 2.0L * T / (2 * j + 2 * k + 1);
                    sum += term;
                    if (term < sum * 1e-22L) break;
                }
                v[it][j] = (double)(expl(-T) * sum);
            }
        }
    }
};
inline const BoysTable& boys_table()
{
    static const BoysTable t;
    return t;
}

// F_0..F_jmax at T.  AuxillaryFJ.C:13-48: three branches, T<12 Taylor(6) + downward recursion,
// 12<=T<30 asymptotic with the reference's g(T) fits + upward recursion, T>=30 pure asymptotic.
inline void boys(double T, int jmax, double* Fj)
{
    static const double fact[7] = {1, 1, 2, 6, 24, 120, 720};
    const double et = std::exp(-T);
    if (T < 12)
    {
        int it = (int)(T * 10.0 + 0.5);
        double Tstar = (double)it * 0.1;
        double dt = Tstar - T;
        const double* FT = &boys_table().v[it][0];
        double f = FT[jmax];
        double dtk = 1.0;
        for (int k = 1; k <= 6; ++k)
        {
            dtk *= dt;
            f += FT[k + jmax] * dtk / fact[k];
        }
        Fj[jmax] = f;
        for (int j = jmax - 1; j >= 0; --j) Fj[j] = (2 * T * Fj[j + 1] + et) / (2 * j + 1);
    }
    else
    {
        double F0;
        if (T < 30.0)
        {
            double g;
            if (T < 15) g = 0.4999489092 - 0.2473631686 / T + 0.321180909 / (T * T) - 0.3811559346 / (T * T * T);
            else if (T < 18) g = 0.4998436875 - 0.24249438 / T + 0.24642845 / (T * T);
            else if (T < 24) g = 0.499093162 - 0.2152832 / T;
            else g = 0.49;
            F0 = 0.5 * std::sqrt(kPi / T) - et * g / T;
        }
        else
            F0 = 0.5 * std::sqrt(kPi / T);
        Fj[0] = F0;
        for (int j = 0; j < jmax; ++j) Fj[j + 1] = ((2 * j + 1) * Fj[j] - et) / (2 * T);
    }
}

// ---------------------------------------------------------------------------------------------------
// Cartesian components, PG order: for m=0..L, l=0..L-m: (L-m-l, l, m)   (IrrepBasisSet.C:36-54)
// ---------------------------------------------------------------------------------------------------
inline int ncart(int L) { return (L + 1) * (L + 2) / 2; }
inline std::vector<std::array<int, 3>> components(int L)
{
    std::vector<std::array<int, 3>> c;
    for (int m = 0; m <= L; ++m)
        for (int l = 0; l <= L - m; ++l) c.push_back({L - m - l, l, m});
    return c;
}

inline double dfact(int i)   // (i)!! with (-1)!! = 1
{
    double r = 1;
    for (int k = i; k > 1; k -= 2) r *= k;
    return r;
}

// Primitive normalisation for polarisation (n,l,m): GaussianRF.C:512-521
inline double prim_norm(double alpha, int n, int l, int m)
{
    double s = std::pow(kPi / (2 * alpha), 1.5);
    double t = 1.0;
    for (int k = 0; k < n + l + m; ++k) t *= 4 * alpha;
    double f = dfact(2 * n - 1) * dfact(2 * l - 1) * dfact(2 * m - 1);
    return std::sqrt(t / (s * f));
}

// ---------------------------------------------------------------------------------------------------
// Hermite E coefficients of one primitive pair along one direction, built in the reference's layered
// order (Hermite2.C:95-139): entry (i,j) with j>=1 ends up from the b-increment of (i,j-1); j==0 from
// the a-increment of (i-1,0).  E[t][i][j], t<=i+j.
// ---------------------------------------------------------------------------------------------------
struct Herm1D
{
    int la = 0, lb = 0;
    std::vector<double> e;   // [(la+lb+1)][(la+1)][(lb+1)]
    double& at(int t, int i, int j) { return e[(t * (la + 1) + i) * (lb + 1) + j]; }
    double get(int t, int i, int j) const
    {
        if (t < 0 || t > i + j) return 0.0;
        return e[(t * (la + 1) + i) * (lb + 1) + j];
    }
    void build(double a12, double PA, double PB, int LA, int LB)
    {
        la = LA; lb = LB;
        e.assign((la + lb + 1) * (la + 1) * (lb + 1), 0.0);
        at(0, 0, 0) = 1.0;
        for (int layer = 0; layer <= la + lb - 1; ++layer)
            for (int na = 0; na <= layer; ++na)
            {
                int nb = layer - na;
                if (na > la || nb > lb) continue;
                for (int N = 0; N <= layer + 1; ++N)
                {
                    double t1 = 0, ta = 0, tb = 0, t3 = 0;
                    if (N - 1 >= 0) t1 = get(N - 1, na, nb) * a12;
                    if (N <= na + nb) { ta = get(N, na, nb) * PA; tb = get(N, na, nb) * PB; }
                    if (N + 1 <= na + nb) t3 = get(N + 1, na, nb) * (N + 1);
                    if (na + 1 <= la) at(N, na + 1, nb) = t1 + ta + t3;
                    if (nb + 1 <= lb) at(N, na, nb + 1) = t1 + tb + t3;
                }
            }
    }
};

// Primitive-pair charge distribution (GaussianRF.C:239-252)
struct PrimPair
{
    double a, b, p, ab;
    std::array<double, 3> P, A, B;
    double Eij;
    Herm1D H[3];
    void build(double alpha, const std::array<double, 3>& Ain, int La, double beta, const std::array<double, 3>& Bin,
               int Lb, int extra)
    {
        a = alpha; b = beta; p = a + b; ab = a * b; A = Ain; B = Bin;
        double r2 = 0;
        for (int x = 0; x < 3; ++x)
        {
            P[x] = (a * A[x] + b * B[x]) / p;
            double d = A[x] - B[x];
            r2 += d * d;
        }
        Eij = std::exp(-ab / p * r2);
        double a12 = 1.0 / (2 * p);
        for (int x = 0; x < 3; ++x) H[x].build(a12, P[x] - A[x], P[x] - B[x], La + extra, Lb + extra);
    }
    // H2(P,pa,pb) = d*e*f   (Hermite2.C:158-199)
    double h2(int tn, int tl, int tm, const std::array<int, 3>& pa, const std::array<int, 3>& pb) const
    {
        if (tn < 0 || tl < 0 || tm < 0) return 0.0;
        for (int x = 0; x < 3; ++x)
            if (pa[x] < 0 || pb[x] < 0) return 0.0;
        return H[0].get(tn, pa[0], pb[0]) * H[1].get(tl, pa[1], pb[1]) * H[2].get(tm, pa[2], pb[2]);
    }
};

// ---------------------------------------------------------------------------------------------------
// Hermite Coulomb integrals R^0_{NLM}(alpha, dR), N+L+M <= Lmax  (RNLM.C:19-68, Triangle3D packing)
// ---------------------------------------------------------------------------------------------------
inline int tri_size(int N) { return (N + 1) * (N + 2) * (N + 3) / 6; }
struct RTable
{
    int Lmax = 0;
    std::vector<double> v;   // indexed by (n,l,m) dense cube (Lmax+1)^3 for simplicity
    double operator()(int n, int l, int m) const { return v[(n * (Lmax + 1) + l) * (Lmax + 1) + m]; }
    void build(int Max, double alpha, const std::array<double, 3>& dR)
    {
        Lmax = Max;
        const int S = Max + 1;
        std::vector<double> cur(S * S * S, 0.0), nxt(S * S * S, 0.0);
        auto I = [S](int n, int l, int m) { return (n * S + l) * S + m; };
        double F[kJMax + 8];
        double T = alpha * (dR[0] * dR[0] + dR[1] * dR[1] + dR[2] * dR[2]);
        boys(T, Max, F);
        auto ipow = [](double x, int n) { double r = 1; for (int k = 0; k < n; ++k) r *= x; return r; };
        // level j = Max
        nxt[I(0, 0, 0)] = ipow(-2.0 * alpha, Max) * F[Max];
        for (int j = Max - 1; j >= 0; --j)
        {
            std::fill(cur.begin(), cur.end(), 0.0);
            cur[I(0, 0, 0)] = ipow(-2.0 * alpha, j) * F[j];
            int n = Max - j;
            for (int M = 0; M < n; ++M)
            {
                cur[I(0, 0, M + 1)] = M > 0 ? dR[2] * nxt[I(0, 0, M)] + M * nxt[I(0, 0, M - 1)] : dR[2] * nxt[I(0, 0, M)];
                for (int L = 0; L < n - M; ++L)
                {
                    cur[I(0, L + 1, M)] = L > 0 ? dR[1] * nxt[I(0, L, M)] + L * nxt[I(0, L - 1, M)] : dR[1] * nxt[I(0, L, M)];
                    for (int N = 0; N < n - M - L; ++N)
                        cur[I(N + 1, L, M)] = N > 0 ? dR[0] * nxt[I(N, L, M)] + N * nxt[I(N - 1, L, M)] : dR[0] * nxt[I(N, L, M)];
                }
            }
            std::swap(cur, nxt);
        }
        v = nxt;
    }
};

// (ab|cd) for one component quadruple of one primitive quartet (GaussianRF.C:446-483)
inline double prim_eri(const PrimPair& ab, const PrimPair& cd, const RTable& R, const std::array<int, 3>& pa,
                       const std::array<int, 3>& pb, const std::array<int, 3>& pc, const std::array<int, 3>& pd)
{
    const double Pi52 = kPi * kPi * std::sqrt(kPi);
    double lambda = 2 * Pi52 / (ab.p * cd.p * std::sqrt(ab.p + cd.p));
    lambda *= ab.Eij * cd.Eij;
    int Pab[3], Pcd[3];
    for (int x = 0; x < 3; ++x) { Pab[x] = pa[x] + pb[x]; Pcd[x] = pc[x] + pd[x]; }
    double s = 0.0;
    for (int an = 0; an <= Pab[0]; ++an)
        for (int al = 0; al <= Pab[1]; ++al)
            for (int am = 0; am <= Pab[2]; ++am)
            {
                const double hab = ab.h2(an, al, am, pa, pb);
                if (hab == 0.0) continue;
                for (int cn = 0; cn <= Pcd[0]; ++cn)
                    for (int cl = 0; cl <= Pcd[1]; ++cl)
                        for (int cm = 0; cm <= Pcd[2]; ++cm)
                        {
                            const double hcd = cd.h2(cn, cl, cm, pc, pd);
                            if (hcd == 0.0) continue;
                            const double r = R(an + cn, al + cl, am + cm);
                            if (r != 0.0)
                            {
                                const double sign = ((cn + cl + cm) & 1) ? -1.0 : 1.0;
                                s += hab * hcd * r * sign;
                            }
                        }
            }
    return s * lambda;
}

// ---------------------------------------------------------------------------------------------------
// Basis
// ---------------------------------------------------------------------------------------------------
struct Shell
{
    int L = 0;
    std::array<double, 3> A{0, 0, 0};
    std::vector<double> alpha, coef;   // coef already multiplied by prim_norm(alpha, L,0,0)
    int f0 = 0;                        // first basis function
};

struct Basis
{
    std::vector<Shell> shells;
    std::vector<double> ns;            // per basis function: 1/sqrt(self overlap)   (PGData.C:17-33)
    std::vector<int> fn_shell, fn_comp;
    int nbf = 0;

    // raw coefficients as in a basis file; folding of the (L,0,0) primitive norm follows GaussianRF.C:566-577
    void add_shell(int L, const std::array<double, 3>& A, const std::vector<double>& alpha, const std::vector<double>& c)
    {
        Shell s;
        s.L = L; s.A = A; s.alpha = alpha; s.coef = c;
        for (size_t i = 0; i < alpha.size(); ++i) s.coef[i] *= prim_norm(alpha[i], L, 0, 0);
        s.f0 = nbf;
        for (int k = 0; k < ncart(L); ++k) { fn_shell.push_back((int)shells.size()); fn_comp.push_back(k); }
        nbf += ncart(L);
        shells.push_back(s);
    }
    void finalize();
};

// contracted overlap between two shells' components (GaussianRF.C:328-334 per primitive)
inline double overlap_contracted(const Shell& a, int ca, const Shell& b, int cb)
{
    auto pa = components(a.L)[ca], pb = components(b.L)[cb];
    double s = 0;
    for (size_t i = 0; i < a.alpha.size(); ++i)
        for (size_t j = 0; j < b.alpha.size(); ++j)
        {
            PrimPair pp;
            pp.build(a.alpha[i], a.A, a.L, b.alpha[j], b.A, b.L, 1);
            s += a.coef[i] * b.coef[j] * std::pow(kPi / pp.p, 1.5) * pp.Eij * pp.h2(0, 0, 0, pa, pb);
        }
    return s;
}

inline void Basis::finalize()
{
    ns.resize(nbf);
    for (int f = 0; f < nbf; ++f)
    {
        const Shell& s = shells[fn_shell[f]];
        ns[f] = 1.0 / std::sqrt(overlap_contracted(s, fn_comp[f], s, fn_comp[f]));
    }
}

// One-electron integrals, contracted and normalised (Evaluator.C:71-76 with ns_i ns_j)
// Grad2 per GaussianRF.C:311-405 (GetGrad2); kinetic T = Grad2/2.  Nuclear per GaussianRF.C:383-400.
struct Atom
{
    double Z;
    std::array<double, 3> R;
};

inline void one_electron(const Basis& bs, const std::vector<Atom>& atoms, std::vector<double>& S, std::vector<double>& T,
                         std::vector<double>& V)
{
    const int n = bs.nbf;
    S.assign(n * n, 0); T.assign(n * n, 0); V.assign(n * n, 0);
    for (int f = 0; f < n; ++f)
        for (int g = 0; g <= f; ++g)
        {
            const Shell& a = bs.shells[bs.fn_shell[f]];
            const Shell& b = bs.shells[bs.fn_shell[g]];
            auto pa = components(a.L)[bs.fn_comp[f]], pb = components(b.L)[bs.fn_comp[g]];
            double s = 0, t = 0, v = 0;
            for (size_t i = 0; i < a.alpha.size(); ++i)
                for (size_t j = 0; j < b.alpha.size(); ++j)
                {
                    PrimPair pp;
                    pp.build(a.alpha[i], a.A, a.L, b.alpha[j], b.A, b.L, 1);
                    double cc = a.coef[i] * b.coef[j];
                    double fac = std::pow(kPi / pp.p, 1.5) * pp.Eij;
                    s += cc * fac * pp.h2(0, 0, 0, pa, pb);
                    // Grad2
                    double g2 = 0;
                    for (int x = 0; x < 3; ++x)
                    {
                        auto am = pa, ap = pa, bm = pb, bp = pb;
                        am[x] -= 1; ap[x] += 1; bm[x] -= 1; bp[x] += 1;
                        g2 += pa[x] * pb[x] * pp.h2(0, 0, 0, am, bm) - 2 * pa[x] * pp.b * pp.h2(0, 0, 0, am, bp)
                            - 2 * pb[x] * pp.a * pp.h2(0, 0, 0, ap, bm) + 4 * pp.ab * pp.h2(0, 0, 0, ap, bp);
                    }
                    t += cc * fac * g2;
                    // Nuclear attraction
                    int Lt = a.L + b.L;
                    std::vector<double> Rsum((Lt + 1) * (Lt + 1) * (Lt + 1), 0.0);
                    for (const Atom& at : atoms)
                    {
                        RTable R;
                        std::array<double, 3> PC{pp.P[0] - at.R[0], pp.P[1] - at.R[1], pp.P[2] - at.R[2]};
                        R.build(Lt, pp.p, PC);
                        for (size_t k = 0; k < Rsum.size(); ++k) Rsum[k] += R.v[k] * (-1.0 * at.Z);
                    }
                    double sv = 0;
                    for (int tn = 0; tn <= pa[0] + pb[0]; ++tn)
                        for (int tl = 0; tl <= pa[1] + pb[1]; ++tl)
                            for (int tm = 0; tm <= pa[2] + pb[2]; ++tm)
                            {
                                double h = pp.h2(tn, tl, tm, pa, pb);
                                if (h != 0) sv += h * Rsum[(tn * (Lt + 1) + tl) * (Lt + 1) + tm];
                            }
                    v += cc * sv * 2 * kPi / pp.p * pp.Eij;
                }
            double nn = bs.ns[f] * bs.ns[g];
            S[f * n + g] = S[g * n + f] = s * nn;
            T[f * n + g] = T[g * n + f] = 0.5 * t * nn;
            V[f * n + g] = V[g * n + f] = v * nn;
        }
}

inline double nuclear_repulsion(const std::vector<Atom>& atoms)
{
    double e = 0;
    for (size_t i = 0; i < atoms.size(); ++i)
        for (size_t j = 0; j < i; ++j)
        {
            double d2 = 0;
            for (int x = 0; x < 3; ++x) { double d = atoms[i].R[x] - atoms[j].R[x]; d2 += d * d; }
            e += atoms[i].Z * atoms[j].Z / std::sqrt(d2);
        }
    return e;
}

// ---------------------------------------------------------------------------------------------------
// FourC for single basis functions, the reference's per-component route (Evaluator.C:1912-1920,
// GaussianRF.C:726-752): contraction over primitives, per-component Hermite sums, times four ns.
// ---------------------------------------------------------------------------------------------------
inline double fourc(const Basis& bs, int fa, int fb, int fc, int fd)
{
    const Shell& A = bs.shells[bs.fn_shell[fa]];
    const Shell& B = bs.shells[bs.fn_shell[fb]];
    const Shell& C = bs.shells[bs.fn_shell[fc]];
    const Shell& D = bs.shells[bs.fn_shell[fd]];
    auto pa = components(A.L)[bs.fn_comp[fa]], pb = components(B.L)[bs.fn_comp[fb]];
    auto pc = components(C.L)[bs.fn_comp[fc]], pd = components(D.L)[bs.fn_comp[fd]];
    double s = 0;
    for (size_t i = 0; i < A.alpha.size(); ++i)
        for (size_t j = 0; j < B.alpha.size(); ++j)
        {
            PrimPair ab;
            ab.build(A.alpha[i], A.A, A.L, B.alpha[j], B.A, B.L, 1);
            for (size_t k = 0; k < C.alpha.size(); ++k)
                for (size_t l = 0; l < D.alpha.size(); ++l)
                {
                    PrimPair cd;
                    cd.build(C.alpha[k], C.A, C.L, D.alpha[l], D.A, D.L, 1);
                    RTable R;
                    std::array<double, 3> PQ{ab.P[0] - cd.P[0], ab.P[1] - cd.P[1], ab.P[2] - cd.P[2]};
                    R.build(A.L + B.L + C.L + D.L, ab.p * cd.p / (ab.p + cd.p), PQ);
                    s += A.coef[i] * B.coef[j] * C.coef[k] * D.coef[l] * prim_eri(ab, cd, R, pa, pb, pc, pd);
                }
        }
    return s * bs.ns[fa] * bs.ns[fb] * bs.ns[fc] * bs.ns[fd];
}

// Whole shell-quartet block (all components), out[(((ia*nb+ib)*nc+ic)*nd+id)], same arithmetic as
// fourc() but with one R table per primitive quartet shared by all component quadruples.
inline void shell_quartet(const Basis& bs, int sa, int sb, int sc, int sd, double* out)
{
    const Shell& A = bs.shells[sa];
    const Shell& B = bs.shells[sb];
    const Shell& C = bs.shells[sc];
    const Shell& D = bs.shells[sd];
    auto ca = components(A.L), cb = components(B.L), cc = components(C.L), cdc = components(D.L);
    const int na = ca.size(), nb = cb.size(), nc = cc.size(), nd = cdc.size();
    const int ntot = na * nb * nc * nd;
    std::fill(out, out + ntot, 0.0);
    for (size_t i = 0; i < A.alpha.size(); ++i)
        for (size_t j = 0; j < B.alpha.size(); ++j)
        {
            PrimPair ab;
            ab.build(A.alpha[i], A.A, A.L, B.alpha[j], B.A, B.L, 0);
            for (size_t k = 0; k < C.alpha.size(); ++k)
                for (size_t l = 0; l < D.alpha.size(); ++l)
                {
                    PrimPair cd;
                    cd.build(C.alpha[k], C.A, C.L, D.alpha[l], D.A, D.L, 0);
                    RTable R;
                    std::array<double, 3> PQ{ab.P[0] - cd.P[0], ab.P[1] - cd.P[1], ab.P[2] - cd.P[2]};
                    R.build(A.L + B.L + C.L + D.L, ab.p * cd.p / (ab.p + cd.p), PQ);
                    double cf = A.coef[i] * B.coef[j] * C.coef[k] * D.coef[l];
                    int o = 0;
                    for (int a = 0; a < na; ++a)
                        for (int b = 0; b < nb; ++b)
                            for (int c = 0; c < nc; ++c)
                                for (int d = 0; d < nd; ++d, ++o)
                                    out[o] += cf * prim_eri(ab, cd, R, ca[a], cb[b], cc[c], cdc[d]);
                }
        }
    int o = 0;
    for (int a = 0; a < na; ++a)
        for (int b = 0; b < nb; ++b)
            for (int c = 0; c < nc; ++c)
                for (int d = 0; d < nd; ++d, ++o)
                    out[o] *= bs.ns[A.f0 + a] * bs.ns[B.f0 + b] * bs.ns[C.f0 + c] * bs.ns[D.f0 + d];
}

// ---------------------------------------------------------------------------------------------------
// 3-centre Coulomb (ab|c): the ab charge distribution against c's single-centre Hermite expansion, with
// the overall sign (-1)^{L_c} and prefactor 2 pi^{5/2} / (p gamma sqrt(p + gamma)) E_ab
// (GaussianRF.C:415-444); contracted and normalised like NR_Evaluator::RepulsionThreeC (Evaluator.C:1905-1908)
// ---------------------------------------------------------------------------------------------------
inline double prim_eri3(const PrimPair& ab, double gam, const Herm1D (&Hc)[3], const RTable& R,
                        const std::array<int, 3>& pa, const std::array<int, 3>& pb, const std::array<int, 3>& pc)
{
    const double Pi52 = kPi * kPi * std::sqrt(kPi);
    int Pab[3];
    for (int x = 0; x < 3; ++x) Pab[x] = pa[x] + pb[x];
    double s = 0.0;
    for (int an = 0; an <= Pab[0]; ++an)
        for (int al = 0; al <= Pab[1]; ++al)
            for (int am = 0; am <= Pab[2]; ++am)
            {
                const double hab = ab.h2(an, al, am, pa, pb);
                if (hab == 0.0) continue;
                double Rs = 0.0;
                for (int n = 0; n <= pc[0]; ++n)
                    for (int l = 0; l <= pc[1]; ++l)
                        for (int m = 0; m <= pc[2]; ++m)
                        {
                            const double h = Hc[0].get(n, pc[0], 0) * Hc[1].get(l, pc[1], 0) * Hc[2].get(m, pc[2], 0);
                            if (h != 0.0) Rs += h * R(an + n, al + l, am + m);
                        }
                if (Rs != 0.0) s += hab * Rs;
            }
    double factor = 1.0 / (ab.p * gam * std::sqrt(ab.p + gam));
    if ((pc[0] + pc[1] + pc[2]) & 1) factor = -factor;
    return s * 2 * Pi52 * ab.Eij * factor;
}

// whole shell-triple block out[((ia*nb+ib)*nc+ic)]
inline void shell_triple(const Basis& bs, int sa, int sb, int sc, double* out)
{
    const Shell& A = bs.shells[sa];
    const Shell& B = bs.shells[sb];
    const Shell& C = bs.shells[sc];
    auto ca = components(A.L), cb = components(B.L), cc = components(C.L);
    const int na = ca.size(), nb = cb.size(), nc = cc.size();
    std::fill(out, out + na * nb * nc, 0.0);
    for (size_t i = 0; i < A.alpha.size(); ++i)
        for (size_t j = 0; j < B.alpha.size(); ++j)
        {
            PrimPair ab;
            ab.build(A.alpha[i], A.A, A.L, B.alpha[j], B.A, B.L, 0);
            for (size_t k = 0; k < C.alpha.size(); ++k)
            {
                const double gam = C.alpha[k];
                Herm1D Hc[3];
                for (int x = 0; x < 3; ++x) Hc[x].build(1.0 / (2 * gam), 0.0, 0.0, C.L, 0);   // one centre: P = C
                RTable R;
                std::array<double, 3> PQ{ab.P[0] - C.A[0], ab.P[1] - C.A[1], ab.P[2] - C.A[2]};
                R.build(A.L + B.L + C.L, ab.p * gam / (ab.p + gam), PQ);
                const double cf = A.coef[i] * B.coef[j] * C.coef[k];
                int o = 0;
                for (int a = 0; a < na; ++a)
                    for (int b = 0; b < nb; ++b)
                        for (int c = 0; c < nc; ++c, ++o) out[o] += cf * prim_eri3(ab, gam, Hc, R, ca[a], cb[b], cc[c]);
            }
        }
    int o = 0;
    for (int a = 0; a < na; ++a)
        for (int b = 0; b < nb; ++b)
            for (int c = 0; c < nc; ++c, ++o) out[o] *= bs.ns[A.f0 + a] * bs.ns[B.f0 + b] * bs.ns[C.f0 + c];
}

}   // namespace mdref
