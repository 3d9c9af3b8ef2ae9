// qchem_b200.hpp -- header-only C++ adapter over the C ABI (qchem_b200.h) for qchem's HF contraction face.
//
// qcg::FockEngine owns one qcg_handle and answers the questions qchem's Hartree-Fock code asks of a basis
// with the WholeSystemFock_IBS<double> face (src/BasisSet/Orbital_HF_IBS.C:75-87):
//   AODimension(), AddAODensity(Dao, D), MakeAOFock(Dao, exchange) -> J[Dao] or K[Dao], SliceAOFock(F, Fao)
// and the Orbital_HF_IBS<double> contraction face (src/BasisSet/Orbital_HF_IBS.C:33-54) for a basis that is
// one irrep: AccumulateDirect(S, D, bs_cd) adds J[D], AccumulateExchange(S, D, bs_cd) adds K[D], and the
// irrep-pair forms AccumulateDirectBoth / AccumulateExchangeBoth.  The engine is one irrep, so the partner
// basis bs_cd must be the engine itself (or null); any other basis is rejected with QCG_ERR_ARG.  qchem calls the
// Coulomb and the exchange face separately with the same density (Vee then Vxc, HF_HT.C:48-70); the
// engine builds J and K together in one GPU pass and keeps them for the density it last saw, so the
// second call costs nothing.  Status codes from the C ABI become qcg::Error exceptions here, the way the
// reference's own substrate throws std::runtime_error (Internal/Imp/Orbital_ERI4_IBS.C:19-32).
// qcg::SalcBlock adds the symmetry-adapted faces (src/BasisSet/Imp/SymmetryAdapted_IBS.C:45-140): one irrep
// block of SALC columns over a FockEngine, sharing its one AO build.
#pragma once
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "qchem_b200.h"

namespace qcg {

struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error("qchem_b200: " + m), code(c) {}
};

// One shell in basis order: angular momentum 0..2, centre (bohr), exponents and raw contraction coefficients.
struct ShellSpec
{
    int L;
    double centre[3];
    std::vector<double> exps, coefs;
};

class FockEngine
{
public:
    explicit FockEngine(const std::vector<ShellSpec>& shells, double schwarz_thresh = 1e-10)
    {
        std::vector<int> L, np;
        std::vector<double> ex, co, cen;
        for (const auto& s : shells)
        {
            L.push_back(s.L);
            np.push_back((int)s.exps.size());
            ex.insert(ex.end(), s.exps.begin(), s.exps.end());
            co.insert(co.end(), s.coefs.begin(), s.coefs.end());
            cen.insert(cen.end(), s.centre, s.centre + 3);
        }
        int rc = qcg_basis_create(L.data(), np.data(), ex.data(), co.data(), cen.data(), (int)shells.size(), &h_);
        if (rc != QCG_OK)
        {
            std::string msg = h_ ? qcg_last_error(h_) : "qcg_basis_create failed";
            qcg_destroy(h_);
            h_ = nullptr;
            throw Error(rc, msg);
        }
        check(qcg_nbf(h_, &n_));
        check(qcg_schwarz(h_, schwarz_thresh, nullptr));
    }
    ~FockEngine() { qcg_destroy(h_); }
    FockEngine(const FockEngine&) = delete;
    FockEngine& operator=(const FockEngine&) = delete;

    size_t AODimension() const { return (size_t)n_; }

    // J (exchange=false) or K (exchange=true) of a dense row-major n x n density into out (n x n)
    void MakeAOFock(const double* Dao, bool exchange, double* out)
    {
        build(Dao);
        const std::vector<double>& X = exchange ? K_ : J_;
        std::memcpy(out, X.data(), X.size() * sizeof(double));
    }
    // Dao += D and F += Fao: the whole system is this one block, so the fold and the slice are identities
    void AddAODensity(double* Dao, const double* D) const
    {
        for (size_t k = 0; k < (size_t)n_ * n_; ++k) Dao[k] += D[k];
    }
    void SliceAOFock(double* F, const double* Fao) const
    {
        for (size_t k = 0; k < (size_t)n_ * n_; ++k) F[k] += Fao[k];
    }
    // S += J[D] and S += K[D] (qchem's AccumulateDirect / AccumulateExchange for a single-irrep basis)
    void AccumulateDirect(double* S, const double* D, const FockEngine* bs_cd = nullptr)
    {
        partner(bs_cd);
        add(S, D, false);
    }
    void AccumulateExchange(double* S, const double* D, const FockEngine* bs_cd = nullptr)
    {
        partner(bs_cd);
        add(S, D, true);
    }
    // The irrep-pair forms, Ji += J(i,j) Dj and Jj += J(j,i) Di (and K alike), for the pair (this, cd); the
    // engine is one irrep, so both blocks are its own J (K).  A zero density adds nothing, as in the
    // reference, where either irrep of the pair may be empty.
    void AccumulateDirectBoth(double* Ji, double* Jj, const double* Di, const double* Dj, const FockEngine* cd = nullptr)
    {
        partner(cd);
        if (nonzero(Dj)) add(Ji, Dj, false);
        if (nonzero(Di)) add(Jj, Di, false);
    }
    void AccumulateExchangeBoth(double* Ki, double* Kj, const double* Di, const double* Dj, const FockEngine* cd = nullptr)
    {
        partner(cd);
        if (nonzero(Dj)) add(Ki, Dj, true);
        if (nonzero(Di)) add(Kj, Di, true);
    }

    qcg_handle* handle() const { return h_; }

private:
    void check(int rc)
    {
        if (rc != QCG_OK) throw Error(rc, qcg_last_error(h_));
    }
    void partner(const FockEngine* cd) const
    {
        if (cd && cd != this) throw Error(QCG_ERR_ARG, "the partner basis must be this engine (one irrep)");
    }
    bool nonzero(const double* D) const
    {
        for (size_t k = 0; k < (size_t)n_ * n_; ++k)
            if (D[k] != 0.0) return true;
        return false;
    }
    void build(const double* D)
    {
        const size_t nn = (size_t)n_ * n_;
        if (D_.size() == nn && std::memcmp(D_.data(), D, nn * sizeof(double)) == 0) return;   // same density
        J_.resize(nn);
        K_.resize(nn);
        check(qcg_fock_jk(h_, D, J_.data(), K_.data(), 0, nullptr));
        D_.assign(D, D + nn);
    }
    void add(double* S, const double* D, bool exchange)
    {
        build(D);
        const std::vector<double>& X = exchange ? K_ : J_;
        for (size_t k = 0; k < X.size(); ++k) S[k] += X[k];
    }

    qcg_handle* h_ = nullptr;
    int n_ = 0;
    std::vector<double> D_, J_, K_;
};

// One irrep block of a symmetry-adapted (SALC) basis over an AO FockEngine: qchem's SymmetryAdapted_IBS
// (src/BasisSet/Imp/SymmetryAdapted_IBS.C:45-140).  The block is m functions, the columns of O (AODimension()
// x m, row-major).  J and K are linear in D, so every block shares ONE AO build: the partner block folds its
// density up (AddAODensity, Dao += sym(O D O^T)), the engine builds J or K of Dao (MakeAOFock), and this
// block slices its part out (SliceAOFock, Fab += sym(O^T Fao O)).  The folds and slices run on the GPU.
class SalcBlock
{
public:
    SalcBlock(FockEngine& ao, std::vector<double> O, int m) : ao_(ao), O_(std::move(O)), m_(m)
    {
        if (m < 1 || (size_t)m > ao.AODimension() || O_.size() != ao.AODimension() * (size_t)m)
            throw Error(QCG_ERR_ARG, "O must be AODimension() x m with 1 <= m <= AODimension()");
    }
    size_t Dimension() const { return (size_t)m_; }

    // WholeSystemFock_IBS<double>
    size_t AODimension() const { return ao_.AODimension(); }
    void AddAODensity(double* Dao, const double* D) const
    {
        check(qcg_salc_fold(ao_.handle(), m_, O_.data(), D, Dao));
    }
    void MakeAOFock(const double* Dao, bool exchange, double* out) const
    {
        const size_t nn = AODimension() * AODimension();
        if (!nonzero(Dao, nn))   // the reference's pre-screen: an empty density builds nothing
        {
            std::memset(out, 0, nn * sizeof(double));
            return;
        }
        ao_.MakeAOFock(Dao, exchange, out);
    }
    void SliceAOFock(double* Fab, const double* Fao) const
    {
        check(qcg_salc_slice(ao_.handle(), m_, O_.data(), Fao, Fab));
    }
    // sym(O^T M O) of an AO matrix (overlap, kinetic, nuclear), into out (m x m)
    void Transform(const double* M, double* out) const
    {
        std::memset(out, 0, (size_t)m_ * m_ * sizeof(double));
        SliceAOFock(out, M);
    }

    // Orbital_HF_IBS<double>: the partner cd folds its block's density up, one AO build, this block slices
    void AccumulateDirect(double* Jab, const double* Dcd, const SalcBlock* cd) const { pair(Jab, Dcd, cd, false); }
    void AccumulateExchange(double* Kab, const double* Dcd, const SalcBlock* cd) const { pair(Kab, Dcd, cd, true); }
    void AccumulateDirectBoth(double* Ji, double* Jj, const double* Di, const double* Dj, const SalcBlock* cd) const
    {
        if (nonzero(Dj, cd->Dimension() * cd->Dimension())) AccumulateDirect(Ji, Dj, cd);
        if (nonzero(Di, Dimension() * Dimension())) cd->AccumulateDirect(Jj, Di, this);
    }
    void AccumulateExchangeBoth(double* Ki, double* Kj, const double* Di, const double* Dj, const SalcBlock* cd) const
    {
        if (nonzero(Dj, cd->Dimension() * cd->Dimension())) AccumulateExchange(Ki, Dj, cd);
        if (nonzero(Di, Dimension() * Dimension())) cd->AccumulateExchange(Kj, Di, this);
    }

private:
    void check(int rc) const
    {
        if (rc != QCG_OK) throw Error(rc, qcg_last_error(ao_.handle()));
    }
    static bool nonzero(const double* X, size_t n)
    {
        for (size_t k = 0; k < n; ++k)
            if (X[k] != 0.0) return true;
        return false;
    }
    void pair(double* S, const double* Dcd, const SalcBlock* cd, bool exchange) const
    {
        if (!cd) throw Error(QCG_ERR_ARG, "the partner block is needed to fold its density");
        if (&cd->ao_ != &ao_) throw Error(QCG_ERR_ARG, "the partner block belongs to another AO engine");
        const size_t nn = AODimension() * AODimension();
        std::vector<double> Dao(nn, 0.0), F(nn);
        cd->AddAODensity(Dao.data(), Dcd);
        MakeAOFock(Dao.data(), exchange, F.data());
        SliceAOFock(S, F.data());
    }

    FockEngine& ao_;
    std::vector<double> O_;
    int m_;
};

// Frees the device slabs, pinned staging, streams and events that destroyed engines left for reuse by the
// next engine on the same device (qcg_release_cache): call it before cudaDeviceReset, or when the memory is
// wanted back.
inline void release_cache() { qcg_release_cache(); }

}   // namespace qcg
