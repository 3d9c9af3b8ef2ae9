// oracle_capi.cpp -- C API over the CPU restatement in mdref.hpp.
//
// TEST INFRASTRUCTURE ONLY (the checker): loaded with ctypes by tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py.  The product never links it.
//
// Besides the per-integral restatement it provides the two CPU J/K builders the CPU baseline uses:
//   orc_jk_eri4   -- the reference's own cost structure: ERI4 supermatrices filled element by element with
//                    FourC (src/BasisSet/Molecule/IrrepBasisSet.C:138-183) with the primitive-pair and R
//                    tables memoised like the reference's Cache2 (Imp/GaussianRF.C:183-199), then
//                    ERI4::MatMul (src/BasisSet/Internal/Imp/ERI4.C:10-17).  Serial, like the reference.
//   orc_jk_direct -- shell quartets with 8-fold symmetry, Schwarz screening and OpenMP threads.
// and an RHF driver (core guess, Pulay DIIS with the reference's gating and pruning rules, Jacobi
// eigensolver) following src/SCFIterator/Imp/SCFIterator.C:283-362 and
// src/SCFAccelerator/Internal/Imp/SCFAcceleratorDIIS.C:35-238.
#include "mdref.hpp"
#include <chrono>
#include <deque>
#include <memory>
#include <omp.h>

using namespace mdref;

namespace {

// --------------------------- small dense linear algebra (row-major) ---------------------------------
void jacobi_eigen(int n, const double* Ain, double* w, double* V)   // A = V diag(w) V^T, ascending
{
    std::vector<double> A(Ain, Ain + n * n);
    for (int i = 0; i < n * n; ++i) V[i] = 0;
    for (int i = 0; i < n; ++i) V[i * n + i] = 1;
    for (int sweep = 0; sweep < 100; ++sweep)
    {
        double off = 0, tot = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) { double a = A[i * n + j] * A[i * n + j]; tot += a; if (i != j) off += a; }
        if (off <= 1e-30 * tot || off == 0) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q)
            {
                double apq = A[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                double app = A[p * n + p], aqq = A[q * n + q];
                double theta = (aqq - app) / (2 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k)
                {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k)
                {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k)
                {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return A[a * n + a] < A[b * n + b]; });
    std::vector<double> Vs(n * n);
    for (int j = 0; j < n; ++j)
    {
        w[j] = A[idx[j] * n + idx[j]];
        for (int k = 0; k < n; ++k) Vs[k * n + j] = V[k * n + idx[j]];
    }
    std::copy(Vs.begin(), Vs.end(), V);
}

void matmul(int n, int m, int k, const double* A, bool ta, const double* B, bool tb, double* C)   // C[n x m] = op(A)[n x k] op(B)[k x m]
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j)
        {
            double s = 0;
            for (int l = 0; l < k; ++l)
            {
                double a = ta ? A[l * n + i] : A[i * k + l];
                double b = tb ? B[j * k + l] : B[l * m + j];
                s += a * b;
            }
            C[i * m + j] = s;
        }
}

std::vector<double> solve(int n, std::vector<double> A, std::vector<double> b)   // Gaussian elimination, partial pivoting
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
        for (int r = c + 1; r < n; ++r)
        {
            double f = A[r * n + c] / A[c * n + c];
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

// ------------------------------------ J/K builders -------------------------------------------------
std::vector<double> schwarz(const Basis& bs)
{
    const int ns = bs.shells.size();
    std::vector<double> Q(ns * ns, 0.0);
#pragma omp parallel
    {
        std::vector<double> buf(6 * 6 * 6 * 6);
#pragma omp for schedule(dynamic)
        for (int a = 0; a < ns; ++a)
            for (int b = 0; b <= a; ++b)
            {
                shell_quartet(bs, a, b, a, b, buf.data());
                int na = ncart(bs.shells[a].L), nb = ncart(bs.shells[b].L);
                double m = 0;
                for (int i = 0; i < na; ++i)
                    for (int j = 0; j < nb; ++j) m = std::max(m, std::fabs(buf[((i * nb + j) * na + i) * nb + j]));
                Q[a * ns + b] = Q[b * ns + a] = std::sqrt(m);
            }
    }
    return Q;
}

// 8-fold symmetric digestion of one canonical shell quartet into J', K' (J = J'+J'^T, K = K'+K'^T)
void digest(const Basis& bs, int sa, int sb, int sc, int sd, const double* v, double s, const double* D, double* J,
            double* K, int n)
{
    const Shell &A = bs.shells[sa], &B = bs.shells[sb], &C = bs.shells[sc], &Dd = bs.shells[sd];
    const int na = ncart(A.L), nb = ncart(B.L), nc = ncart(C.L), nd = ncart(Dd.L);
    int o = 0;
    for (int a = 0; a < na; ++a)
        for (int b = 0; b < nb; ++b)
            for (int c = 0; c < nc; ++c)
                for (int d = 0; d < nd; ++d, ++o)
                {
                    const int mu = A.f0 + a, nu = B.f0 + b, la = C.f0 + c, si = Dd.f0 + d;
                    const double w = s * v[o];
                    J[mu * n + nu] += 2 * w * D[la * n + si];
                    J[la * n + si] += 2 * w * D[mu * n + nu];
                    K[mu * n + la] += w * D[nu * n + si];
                    K[nu * n + la] += w * D[mu * n + si];
                    K[mu * n + si] += w * D[nu * n + la];
                    K[nu * n + si] += w * D[mu * n + la];
                }
}

// rank/world: this call evaluates only bra shell pairs ij with ij % world == rank (a multi-rank share);
// the sum over all ranks is the full build
long long jk_direct(const Basis& bs, const std::vector<double>& Q, const double* D, double* Jout, double* Kout,
                    double thresh, int nthreads, int rank = 0, int world = 1)
{
    const int ns = bs.shells.size(), n = bs.nbf;
    std::vector<std::pair<int, int>> pairs;
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b <= a; ++b) pairs.push_back({a, b});
    const long long np = pairs.size();
    std::vector<double> Jt(n * n, 0.0), Kt(n * n, 0.0);
    long long count = 0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(+ : count)
    {
        std::vector<double> J(n * n, 0.0), K(n * n, 0.0), buf(6 * 6 * 6 * 6);
#pragma omp for schedule(dynamic, 1)
        for (long long ij = np - 1; ij >= 0; --ij)
        {
            if (ij % world != rank) continue;
            auto [a, b] = pairs[ij];
            for (long long kl = 0; kl <= ij; ++kl)
            {
                auto [c, d] = pairs[kl];
                if (Q[a * ns + b] * Q[c * ns + d] < thresh) continue;
                shell_quartet(bs, a, b, c, d, buf.data());
                double s = (a == b ? 0.5 : 1.0) * (c == d ? 0.5 : 1.0) * (ij == kl ? 0.5 : 1.0);
                digest(bs, a, b, c, d, buf.data(), s, D, J.data(), K.data(), n);
                ++count;
            }
        }
#pragma omp critical
        for (int i = 0; i < n * n; ++i) { Jt[i] += J[i]; Kt[i] += K[i]; }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            Jout[i * n + j] = Jt[i * n + j] + Jt[j * n + i];
            Kout[i * n + j] = Kt[i * n + j] + Kt[j * n + i];
        }
    return count;
}

// The direct build restricted to a subset of shell pairs: the quartets (ab|cd) of jk_direct's canonical
// enumeration whose two pairs are both in the subset (pair (a,b), a >= b, is in it when in[a * ns + b] or
// in[b * ns + a]), visiting only the subset's pairs.  Returns the number of quartets evaluated.
long long jk_direct_subset(const Basis& bs, const std::vector<double>& Q, const double* D, double* Jout, double* Kout,
                           double thresh, int nthreads, const unsigned char* in)
{
    const int ns = bs.shells.size(), n = bs.nbf;
    std::vector<std::pair<int, int>> pairs;   // the subset's pairs in jk_direct's order (a, then b <= a)
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b <= a; ++b)
            if (in[(size_t)a * ns + b] || in[(size_t)b * ns + a]) pairs.push_back({a, b});
    const long long np = pairs.size();
    std::vector<double> Jt(n * n, 0.0), Kt(n * n, 0.0);
    long long count = 0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(+ : count)
    {
        std::vector<double> J(n * n, 0.0), K(n * n, 0.0), buf(6 * 6 * 6 * 6);
#pragma omp for schedule(dynamic, 1)
        for (long long ij = np - 1; ij >= 0; --ij)
        {
            auto [a, b] = pairs[ij];
            for (long long kl = 0; kl <= ij; ++kl)
            {
                auto [c, d] = pairs[kl];
                if (Q[a * ns + b] * Q[c * ns + d] < thresh) continue;
                shell_quartet(bs, a, b, c, d, buf.data());
                double s = (a == b ? 0.5 : 1.0) * (c == d ? 0.5 : 1.0) * (ij == kl ? 0.5 : 1.0);
                digest(bs, a, b, c, d, buf.data(), s, D, J.data(), K.data(), n);
                ++count;
            }
        }
#pragma omp critical
        for (int i = 0; i < n * n; ++i) { Jt[i] += J[i]; Kt[i] += K[i]; }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            Jout[i * n + j] = Jt[i * n + j] + Jt[j * n + i];
            Kout[i * n + j] = Kt[i * n + j] + Kt[j * n + i];
        }
    return count;
}

// Reference cost structure: memoised Omega (primitive pair) and RNLM tables keyed like the reference's
// Cache2, ERI4 element loops, then MatMul.
struct Eri4Builder
{
    const Basis& bs;
    std::vector<int> prim_of_fn0;   // first global primitive of each shell
    std::vector<std::unique_ptr<PrimPair>> omega;   // by (global prim i, global prim j)
    std::unordered_map<uint64_t, std::unique_ptr<RTable>> rcache;
    int nprim = 0;
    explicit Eri4Builder(const Basis& b) : bs(b)
    {
        for (auto& s : bs.shells) { prim_of_fn0.push_back(nprim); nprim += s.alpha.size(); }
        omega.resize((size_t)nprim * nprim);
    }
    const PrimPair& om(int sa, int i, int sb, int j)
    {
        int gi = prim_of_fn0[sa] + i, gj = prim_of_fn0[sb] + j;
        auto& p = omega[(size_t)gi * nprim + gj];
        if (!p)
        {
            p.reset(new PrimPair);
            const Shell &A = bs.shells[sa], &B = bs.shells[sb];
            p->build(A.alpha[i], A.A, A.L, B.alpha[j], B.A, B.L, 1);
        }
        return *p;
    }
    const RTable& rn(int gij, int gkl, const PrimPair& ab, const PrimPair& cd, int L)
    {
        uint64_t key = (uint64_t)gij * (uint64_t)nprim * nprim + gkl;
        auto it = rcache.find(key);
        if (it != rcache.end()) return *it->second;
        auto* R = new RTable;
        std::array<double, 3> PQ{ab.P[0] - cd.P[0], ab.P[1] - cd.P[1], ab.P[2] - cd.P[2]};
        R->build(L, ab.p * cd.p / (ab.p + cd.p), PQ);
        rcache.emplace(key, std::unique_ptr<RTable>(R));
        return *R;
    }
    double fourc(int fa, int fb, int fc, int fd)
    {
        int sa = bs.fn_shell[fa], sb = bs.fn_shell[fb], sc = bs.fn_shell[fc], sd = bs.fn_shell[fd];
        const Shell &A = bs.shells[sa], &B = bs.shells[sb], &C = bs.shells[sc], &D = bs.shells[sd];
        auto pa = components(A.L)[bs.fn_comp[fa]], pb = components(B.L)[bs.fn_comp[fb]];
        auto pc = components(C.L)[bs.fn_comp[fc]], pd = components(D.L)[bs.fn_comp[fd]];
        double s = 0;
        for (size_t i = 0; i < A.alpha.size(); ++i)
            for (size_t j = 0; j < B.alpha.size(); ++j)
            {
                const PrimPair& ab = om(sa, i, sb, j);
                int gij = (prim_of_fn0[sa] + i) * nprim + prim_of_fn0[sb] + j;
                for (size_t k = 0; k < C.alpha.size(); ++k)
                    for (size_t l = 0; l < D.alpha.size(); ++l)
                    {
                        const PrimPair& cd = om(sc, k, sd, l);
                        int gkl = (prim_of_fn0[sc] + k) * nprim + prim_of_fn0[sd] + l;
                        const RTable& R = rn(gij, gkl, ab, cd, A.L + B.L + C.L + D.L);
                        s += A.coef[i] * B.coef[j] * C.coef[k] * D.coef[l] * prim_eri(ab, cd, R, pa, pb, pc, pd);
                    }
            }
        return s * bs.ns[fa] * bs.ns[fb] * bs.ns[fc] * bs.ns[fd];
    }
};

struct Eri4Store
{
    int n = 0;
    std::vector<double> Jsm, Ksm;   // [ab packed upper][cd full n*n], symmetric inner blocks stored full
    bool built = false;
};

void jk_eri4(const Basis& bs, Eri4Store& st, const double* D, double* J, double* K)
{
    const int n = bs.nbf;
    auto pidx = [n](int a, int b) { return a * n - a * (a - 1) / 2 + (b - a); };   // a<=b
    const size_t npair = (size_t)n * (n + 1) / 2;
    if (!st.built)
    {
        st.n = n;
        st.Jsm.assign(npair * n * n, 0.0);
        st.Ksm.assign(npair * n * n, 0.0);
        Eri4Builder eb(bs);
        // MakeDirect: J(ia<=ib)(ic<=id) = FourC(a,b,c,d)   (IrrepBasisSet.C:138-157)
        for (int ia = 0; ia < n; ++ia)
            for (int ib = ia; ib < n; ++ib)
            {
                double* blk = &st.Jsm[pidx(ia, ib) * n * n];
                for (int ic = 0; ic < n; ++ic)
                    for (int id = ic; id < n; ++id)
                    {
                        double v = eb.fourc(ia, ib, ic, id);
                        blk[ic * n + id] = blk[id * n + ic] = v;
                    }
            }
        // MakeExchange: K(ia<=ic)(ib,id) symmetrised with 0.5   (IrrepBasisSet.C:159-183)
        for (int ia = 0; ia < n; ++ia)
            for (int ib = 0; ib < n; ++ib)
                for (int ic = ia; ic < n; ++ic)
                {
                    double* blk = &st.Ksm[pidx(ia, ic) * n * n];
                    for (int id = 0; id < n; ++id)
                    {
                        double v = eb.fourc(ia, ib, ic, id);
                        if (ib == id) blk[ib * n + id] = v;
                        else if (ib < id) { blk[ib * n + id] += 0.5 * v; }
                        else { blk[id * n + ib] += 0.5 * v; }
                    }
                }
        // mirror the upper triangles (symmetric storage)
        for (size_t p = 0; p < npair; ++p)
        {
            double* blk = &st.Ksm[p * n * n];
            for (int i = 0; i < n; ++i)
                for (int j = i + 1; j < n; ++j) blk[j * n + i] = blk[i * n + j];
        }
        st.built = true;
    }
    // MatMul: S(a,b) += sum_cd block(a,b) (.) D   (ERI4.C:10-17)
    for (int ia = 0; ia < n; ++ia)
        for (int ib = ia; ib < n; ++ib)
        {
            const double* bj = &st.Jsm[pidx(ia, ib) * n * n];
            const double* bk = &st.Ksm[pidx(ia, ib) * n * n];
            double sj = 0, sk = 0;
            for (int k = 0; k < n * n; ++k) { sj += bj[k] * D[k]; sk += bk[k] * D[k]; }
            J[ia * n + ib] = J[ib * n + ia] = sj;
            K[ia * n + ib] = K[ib * n + ia] = sk;
        }
}

struct OBasis
{
    Basis bs;
    std::vector<double> Q;
    Eri4Store eri4;
};

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}   // namespace

extern "C" {

void* orc_basis_new() { return new OBasis; }
void orc_basis_free(void* h) { delete (OBasis*)h; }
void orc_basis_add_shell(void* h, int L, const double* A, int nprim, const double* alpha, const double* coef)
{
    auto* o = (OBasis*)h;
    o->bs.add_shell(L, {A[0], A[1], A[2]}, std::vector<double>(alpha, alpha + nprim), std::vector<double>(coef, coef + nprim));
}
int orc_basis_finalize(void* h)
{
    auto* o = (OBasis*)h;
    o->bs.finalize();
    return o->bs.nbf;
}
void orc_basis_norms(void* h, double* ns)
{
    auto* o = (OBasis*)h;
    std::copy(o->bs.ns.begin(), o->bs.ns.end(), ns);
}
void orc_boys(double T, int jmax, double* F) { boys(T, jmax, F); }
void orc_boys_table(double* out)
{
    const auto& t = boys_table();
    std::memcpy(out, t.v, sizeof(t.v));
}
double orc_fourc(void* h, int a, int b, int c, int d) { return fourc(((OBasis*)h)->bs, a, b, c, d); }
void orc_shell_quartet(void* h, int sa, int sb, int sc, int sd, double* out)
{
    shell_quartet(((OBasis*)h)->bs, sa, sb, sc, sd, out);
}
// nq quartets (4 shell indices each) of one class; out holds nq blocks of `block` doubles
void orc_eri_batch(void* h, long long nq, const int* q, long long block, double* out, int nthreads)
{
    auto* o = (OBasis*)h;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long i = 0; i < nq; ++i) shell_quartet(o->bs, q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3], out + i * block);
}
// nt triples (3 shell indices each); out holds nt blocks of `block` doubles (3-centre Coulomb)
void orc_eri3_batch(void* h, long long nt, const int* t, long long block, double* out, int nthreads)
{
    auto* o = (OBasis*)h;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long i = 0; i < nt; ++i) shell_triple(o->bs, t[3 * i], t[3 * i + 1], t[3 * i + 2], out + i * block);
}
void orc_one_electron(void* h, int natom, const double* Z, const double* R, double* S, double* T, double* V)
{
    auto* o = (OBasis*)h;
    std::vector<Atom> atoms;
    for (int i = 0; i < natom; ++i) atoms.push_back({Z[i], {R[3 * i], R[3 * i + 1], R[3 * i + 2]}});
    std::vector<double> s, t, v;
    one_electron(o->bs, atoms, s, t, v);
    std::copy(s.begin(), s.end(), S);
    std::copy(t.begin(), t.end(), T);
    std::copy(v.begin(), v.end(), V);
}
void orc_schwarz(void* h, double* Q)
{
    auto* o = (OBasis*)h;
    if (o->Q.empty()) o->Q = schwarz(o->bs);
    std::copy(o->Q.begin(), o->Q.end(), Q);
}
long long orc_jk_direct(void* h, const double* D, double* J, double* K, double thresh, int nthreads)
{
    auto* o = (OBasis*)h;
    if (o->Q.empty()) o->Q = schwarz(o->bs);
    return jk_direct(o->bs, o->Q, D, J, K, thresh, nthreads);
}
long long orc_jk_direct_shard(void* h, const double* D, double* J, double* K, double thresh, int nthreads, int rank,
                              int world)
{
    auto* o = (OBasis*)h;
    if (o->Q.empty()) o->Q = schwarz(o->bs);
    return jk_direct(o->bs, o->Q, D, J, K, thresh, nthreads, rank, world);
}
long long orc_jk_direct_subset(void* h, const double* D, double* J, double* K, double thresh, int nthreads,
                               const unsigned char* in)
{
    auto* o = (OBasis*)h;
    if (o->Q.empty()) o->Q = schwarz(o->bs);
    return jk_direct_subset(o->bs, o->Q, D, J, K, thresh, nthreads, in);
}
void orc_jk_eri4(void* h, const double* D, double* J, double* K)
{
    auto* o = (OBasis*)h;
    jk_eri4(o->bs, o->eri4, D, J, K);
}

// RHF with core guess + DIIS.  jk_mode 0 = direct (OpenMP), 1 = ERI4 supermatrix (serial).
// stats[0]=wall seconds total, [1]=seconds in J/K builds, [2]=final ||[F',D']||, [3]=nuclear repulsion
// Near-null overlap modes to drop, by the rule of the reference's default orthogonaliser (LASolverAuto with
// the gap-detection tolerance, LASolver/Internal/Imp/LASolverLapack.C:32-62, 385-402), on ascending overlap
// eigenvalues w: the leading non-positive ones always; then, among the eigenvalues below 1e-3 of the largest,
// the largest ratio between neighbours -- above 30 it is a clean gap and everything below it goes; without a
// clean gap, every eigenvalue below the absolute floor 1e-8 goes.  0: S is kept whole (Cholesky there).
int null_modes(int n, const double* w)
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
int orc_null_modes(int n, const double* w) { return null_modes(n, w); }

int orc_rhf2(void* h, int natom, const double* Z, const double* R, int nelec, int jk_mode, double thresh,
             double dE_tol, int maxiter, int nthreads, double fdmax, double* E_out, int* iters, double* D_out,
             double* stats);

int orc_rhf(void* h, int natom, const double* Z, const double* R, int nelec, int jk_mode, double thresh,
            double dE_tol, int maxiter, int nthreads, double* E_out, int* iters, double* D_out, double* stats)
{
    double st5[5] = {};
    const int rc = orc_rhf2(h, natom, Z, R, nelec, jk_mode, thresh, dE_tol, maxiter, nthreads, 0.0, E_out, iters,
                            D_out, st5);
    if (stats) std::copy(st5, st5 + 4, stats);
    return rc;
}

// fdmax > 0 replaces the DIIS switch-on bound Z^2 * 0.1 / 32 (the GPU SCF's diis_fdmax); stats[4] = the
// number of overlap modes dropped
int orc_rhf2(void* h, int natom, const double* Z, const double* R, int nelec, int jk_mode, double thresh,
             double dE_tol, int maxiter, int nthreads, double fdmax, double* E_out, int* iters, double* D_out,
             double* stats)
{
    double t0 = now(), tjk = 0;
    auto* o = (OBasis*)h;
    const Basis& bs = o->bs;
    const int n = bs.nbf, nocc = nelec / 2;
    std::vector<Atom> atoms;
    double Ztot = 0;
    for (int i = 0; i < natom; ++i) { atoms.push_back({Z[i], {R[3 * i], R[3 * i + 1], R[3 * i + 2]}}); Ztot += Z[i]; }
    std::vector<double> S, T, V;
    one_electron(bs, atoms, S, T, V);
    std::vector<double> H(n * n);
    for (int i = 0; i < n * n; ++i) H[i] = T[i] + V[i];
    const double Enn = nuclear_repulsion(atoms);
    // canonical orthogonalisation X = U s^-1/2 (LASolverLapack.C LASolverEigen); the near-null modes of the
    // reference's automatic rule (null_modes) are dropped: their columns of X are zero and X^T F X gets a
    // large diagonal shift on them, so that the eigenproblem is that of the kept modes and a dropped mode is
    // never occupied.  Without dropped modes the reference uses Cholesky, which differs from this X by a
    // rotation that leaves densities and energies unchanged.
    std::vector<double> sw(n), U(n * n), X(n * n);
    jacobi_eigen(n, S.data(), sw.data(), U.data());
    const int ndrop = null_modes(n, sw.data());
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) X[i * n + j] = j < ndrop ? 0.0 : U[i * n + j] / std::sqrt(sw[j]);
    auto ortho = [&](const std::vector<double>& F) {   // X^T F X
        std::vector<double> t(n * n), r(n * n);
        matmul(n, n, n, F.data(), false, X.data(), false, t.data());
        matmul(n, n, n, X.data(), true, t.data(), false, r.data());
        for (int j = 0; j < ndrop; ++j) r[j * n + j] += 1e6;
        return r;
    };
    std::vector<double> Dp(n * n, 0.0), D(n * n, 0.0), w(n), Up(n * n);
    auto diag_fill = [&](const std::vector<double>& Fp) {
        jacobi_eigen(n, Fp.data(), w.data(), Up.data());
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
            {
                double s = 0;
                for (int k = 0; k < nocc; ++k) s += Up[i * n + k] * Up[j * n + k];
                Dp[i * n + j] = 2 * s;
            }
        std::vector<double> t(n * n);
        matmul(n, n, n, X.data(), false, Dp.data(), false, t.data());
        matmul(n, n, n, t.data(), false, X.data(), true, D.data());
    };
    diag_fill(ortho(H));   // core guess: static terms only (Seed.C:70-80, HamiltonianImp.C:58-63)
    if (o->Q.empty() && jk_mode == 0) o->Q = schwarz(bs);
    const int Nproj = 4;
    const double FDMax = fdmax > 0 ? fdmax : Ztot * Ztot * 0.1 / 32, SVTol = 5e-9;
    std::deque<std::vector<double>> Es, Fps;
    std::vector<double> J(n * n), K(n * n), F(n * n);
    double E = 0, Eold = 0, En = 0;
    int it;
    bool conv = false;
    for (it = 1; it <= maxiter; ++it)
    {
        double tj = now();
        if (jk_mode == 0) jk_direct(bs, o->Q, D.data(), J.data(), K.data(), thresh, nthreads);
        else jk_eri4(bs, o->eri4, D.data(), J.data(), K.data());
        tjk += now() - tj;
        for (int i = 0; i < n * n; ++i) F[i] = H[i] + J[i] - 0.5 * K[i];
        double e = 0;
        for (int i = 0; i < n * n; ++i) e += D[i] * (H[i] + F[i]);
        E = 0.5 * e + Enn;
        // DIIS on F' with error [F',D']
        std::vector<double> Fp = ortho(F), Err(n * n), a(n * n), b(n * n);
        matmul(n, n, n, Fp.data(), false, Dp.data(), false, a.data());
        matmul(n, n, n, Dp.data(), false, Fp.data(), false, b.data());
        En = 0;
        for (int i = 0; i < n * n; ++i) { Err[i] = a[i] - b[i]; En += Err[i] * Err[i]; }
        En = std::sqrt(En);
        double dE = E - Eold;
        if (it > 1 && std::fabs(dE) < dE_tol && En < 1e-5) { conv = true; break; }
        Eold = E;
        std::vector<double> Fuse = Fp;
        if (En != 0.0 && En <= FDMax)
        {
            Es.push_back(Err); Fps.push_back(Fp);
            if ((int)Es.size() > Nproj) { Es.pop_front(); Fps.pop_front(); }
            auto bordered = [&]() {
                int m = Es.size();
                std::vector<double> B((m + 1) * (m + 1), 0.0);
                for (int i = 0; i < m; ++i)
                {
                    B[i * (m + 1) + m] = B[m * (m + 1) + i] = 1.0;
                    for (int j = i; j < m; ++j)
                    {
                        double s = 0;
                        for (int k = 0; k < n * n; ++k) s += Es[i][k] * Es[j][k];
                        B[i * (m + 1) + j] = B[j * (m + 1) + i] = s;
                    }
                }
                return B;
            };
            auto minsv = [&](const std::vector<double>& B) {
                int m1 = std::sqrt((double)B.size()) + 0.5;
                std::vector<double> ev(m1), vv(m1 * m1);
                jacobi_eigen(m1, B.data(), ev.data(), vv.data());
                double mn = 1e300;
                for (double x : ev) mn = std::min(mn, std::fabs(x));
                return mn;
            };
            if (Es.size() >= 2)
            {
                auto B = bordered();
                while (minsv(B) < SVTol && Es.size() >= 2) { Es.pop_front(); Fps.pop_front(); B = bordered(); }
                int m = Es.size();
                if (m + 1 > 2)
                {
                    std::vector<double> rhs(m + 1, 0.0);
                    rhs[m] = 1.0;
                    auto c = solve(m + 1, B, rhs);
                    std::fill(Fuse.begin(), Fuse.end(), 0.0);
                    for (int i = 0; i < m; ++i)
                        for (int k = 0; k < n * n; ++k) Fuse[k] += c[i] * Fps[i][k];
                }
            }
        }
        diag_fill(Fuse);
    }
    *E_out = E;
    *iters = conv ? it : maxiter;   // iterations run (the loop exits at maxiter + 1)
    if (D_out) std::copy(D.begin(), D.end(), D_out);
    if (stats) { stats[0] = now() - t0; stats[1] = tjk; stats[2] = En; stats[3] = Enn; stats[4] = ndrop; }
    return conv ? 0 : 1;
}

}   // extern "C"
