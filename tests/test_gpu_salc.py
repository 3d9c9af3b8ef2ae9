"""Symmetry-adapted (SALC) blocks over the AO engine: qchem's SymmetryAdapted_IBS with its WholeSystemFock face
(src/BasisSet/Imp/SymmetryAdapted_IBS.C:45-140).  Water has C2v symmetry; its Cartesian AO space splits into
four irrep blocks, whose columns come from the projection operators of the group's four operations.  Checked:
the GPU folds and slices against numpy; the per-pair route (every block's AccumulateDirect/Exchange against
every partner) against the whole-system route (one fold of all blocks, ONE AO build, one slice per block) and
against the oracle's J and K; and an RHF run entirely in the symmetry-adapted blocks, which must reach the AO
SCF's energy."""
import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

# water lies in the xy plane with its two-fold axis along y: the operations of C2v are diagonal sign
# matrices; C2(y) and sigma(yz) exchange the two hydrogens (atoms 1 and 2)
OPS = [((1, 1, 1), (0, 1, 2)), ((-1, 1, -1), (0, 2, 1)), ((1, 1, -1), (0, 1, 2)), ((-1, 1, 1), (0, 2, 1))]
CHARACTERS = {"A1": (1, 1, 1, 1), "A2": (1, 1, -1, -1), "B1": (1, -1, 1, -1), "B2": (1, -1, -1, 1)}


def salc_blocks(mol, shells):
    """Columns O_G (nbf x m_G) of each irrep G: an orthonormal basis of the range of the projector
    P_G = (1/4) sum_R chi_G(R) Gamma(R), where Gamma(R) maps each Cartesian function to its image (the same
    shell on the image atom, the same component) times sign prod_i s_i^l_i."""
    funcs = []   # (atom, index of the shell within its atom, component)
    per_atom = {}
    for sh in shells:
        i = per_atom.get(sh.atom, 0)
        per_atom[sh.atom] = i + 1
        for comp in B.components(sh.L):
            funcs.append((sh.atom, i, comp))
    index = {f: k for k, f in enumerate(funcs)}
    n = len(funcs)
    gammas = []
    for signs, perm in OPS:
        G = np.zeros((n, n))
        for k, (a, i, comp) in enumerate(funcs):
            s = np.prod([signs[d] ** comp[d] for d in range(3)])
            G[index[(perm[a], i, comp)], k] = s
        gammas.append(G)
    blocks = {}
    for name, chi in CHARACTERS.items():
        P = sum(c * G for c, G in zip(chi, gammas)) / 4.0
        U, s, _ = np.linalg.svd(P)
        blocks[name] = np.ascontiguousarray(U[:, s > 0.5])
    return blocks


@pytest.fixture(scope="module")
def water_salc():
    mol = W.water()
    sh = B.even_tempered(mol)
    eng = api.Engine(sh)
    ao = api.OrbitalHFIBS(eng)
    O = salc_blocks(mol, sh)
    blocks = {g: api.SymmetryAdaptedIBS(ao, O[g], g) for g in O}
    return mol, sh, eng, ao, blocks


def test_blocks_partition_the_ao_space(water_salc):
    mol, sh, eng, ao, blocks = water_salc
    full = np.hstack([b.O for b in blocks.values()])
    assert full.shape == (eng.nbf, eng.nbf)
    assert np.abs(full.T @ full - np.eye(eng.nbf)).max() < 1e-12
    assert all(b.m > 0 for b in blocks.values())


def test_fold_and_slice_match_numpy(water_salc):
    mol, sh, eng, ao, blocks = water_salc
    rng = np.random.default_rng(11)
    for b in blocks.values():
        X = rng.normal(size=(b.m, b.m))
        X = X + X.T
        Dao = np.zeros((eng.nbf, eng.nbf))
        b.AddAODensity(Dao, X)
        ref = b.O @ X @ b.O.T
        assert np.abs(Dao - ref).max() <= 1e-12 * np.abs(ref).max()
        F = rng.normal(size=(eng.nbf, eng.nbf))
        F = F + F.T
        Fab = np.zeros((b.m, b.m))
        b.SliceAOFock(Fab, F)
        ref = b.O.T @ F @ b.O
        assert np.abs(Fab - ref).max() <= 1e-12 * np.abs(ref).max()


def test_pair_route_equals_whole_system_route_and_oracle(water_salc, oracle_mod):
    mol, sh, eng, ao, blocks = water_salc
    D = eng.rhf(mol, want_density=True)["D"]   # converged: totally symmetric
    # the density has no inter-irrep blocks
    for g, b in blocks.items():
        for h, c in blocks.items():
            if g != h:
                assert np.abs(b.O.T @ D @ c.O).max() < 1e-8
    Db = {g: b.Transform(D) for g, b in blocks.items()}
    # whole-system route: fold every block, one AO build, slice
    Dao = np.zeros_like(D)
    for g, b in blocks.items():
        b.AddAODensity(Dao, Db[g])
    assert np.abs(Dao - D).max() < 1e-8
    Jao, Kao = b.MakeAOFock(Dao, False), b.MakeAOFock(Dao, True)
    Jo, Ko, _ = oracle_mod.OracleBasis(sh).jk_direct(Dao, 1e-10)
    for g, b in blocks.items():
        Jw, Kw = np.zeros((b.m, b.m)), np.zeros((b.m, b.m))
        b.SliceAOFock(Jw, Jao)
        b.SliceAOFock(Kw, Kao)
        # per-pair route: every partner's block through AccumulateDirect / AccumulateExchange
        Jp, Kp = np.zeros((b.m, b.m)), np.zeros((b.m, b.m))
        for h, c in blocks.items():
            b.AccumulateDirect(Jp, Db[h], c)
            b.AccumulateExchange(Kp, Db[h], c)
        assert np.abs(Jp - Jw).max() <= 1e-10 and np.abs(Kp - Kw).max() <= 1e-10, g
        assert np.abs(Jw - b.O.T @ Jo @ b.O).max() <= 1e-10, g
        assert np.abs(Kw - b.O.T @ Ko @ b.O).max() <= 1e-10, g
    # the irrep-pair form: Ji += J(i,j) Dj and Jj += J(j,i) Di
    bi, bj = blocks["A1"], blocks["B2"]
    Ji, Jj = np.zeros((bi.m, bi.m)), np.zeros((bj.m, bj.m))
    bi.AccumulateDirectBoth(Ji, Jj, Db["A1"], Db["B2"], bj)
    Ji_ref, Jj_ref = np.zeros_like(Ji), np.zeros_like(Jj)
    bi.AccumulateDirect(Ji_ref, Db["B2"], bj)
    bj.AccumulateDirect(Jj_ref, Db["A1"], bi)
    # (the second calls rebuild J: FP64 atomics give the same J to rounding, not bit for bit)
    assert np.abs(Ji - Ji_ref).max() <= 1e-12 and np.abs(Jj - Jj_ref).max() <= 1e-12


def test_rhf_in_symmetry_adapted_blocks_reaches_the_ao_energy(water_salc):
    """Closed-shell RHF driven entirely through the blocks, the way qchem's composite density drives a SALC
    basis: per-irrep S, H from Transform; each iteration folds every block's density up, builds J and K ONCE
    on the GPU, slices F per block; each block is diagonalised on its own and the lowest orbitals over all
    irreps are occupied; DIIS on the block-diagonal Fock matrix.  It must end at the AO SCF's energy."""
    mol, sh, eng, ao, blocks = water_salc
    ref = eng.rhf(mol)
    S, T, V = eng.one_electron(mol)
    H = T + V
    names = list(blocks)
    Sb = {g: blocks[g].Transform(S) for g in names}
    Hb = {g: blocks[g].Transform(H) for g in names}
    X = {}
    for g in names:
        w, U = np.linalg.eigh(Sb[g])
        X[g] = U / np.sqrt(w)
    nocc = mol.nelec // 2

    def densities(F):
        eps, C = [], {}
        for g in names:
            w, U = np.linalg.eigh(X[g].T @ F[g] @ X[g])
            C[g] = X[g] @ U
            eps += [(e, g, i) for i, e in enumerate(w)]
        occ = sorted(eps)[:nocc]
        D = {g: np.zeros_like(Sb[g]) for g in names}
        for _, g, i in occ:
            D[g] += 2.0 * np.outer(C[g][:, i], C[g][:, i])
        return D

    D = densities(Hb)
    hist_F, hist_e = [], []
    E_old, E = 0.0, None
    for it in range(100):
        Dao = np.zeros((eng.nbf, eng.nbf))
        for g in names:
            blocks[g].AddAODensity(Dao, D[g])
        Jao, Kao = blocks[names[0]].MakeAOFock(Dao, False), blocks[names[0]].MakeAOFock(Dao, True)
        F = {}
        for g in names:
            Fg = Hb[g].copy()
            Jg, Kg = np.zeros_like(Fg), np.zeros_like(Fg)
            blocks[g].SliceAOFock(Jg, Jao)
            blocks[g].SliceAOFock(Kg, Kao)
            F[g] = Fg + Jg - 0.5 * Kg
        E = 0.5 * sum(np.sum(D[g] * (Hb[g] + F[g])) for g in names) + mol.nuclear_repulsion()
        err = np.concatenate([(X[g].T @ (F[g] @ D[g] @ Sb[g] - Sb[g] @ D[g] @ F[g]) @ X[g]).ravel() for g in names])
        if it > 0 and abs(E - E_old) < 1e-10 and np.linalg.norm(err) < 1e-6:
            break
        E_old = E
        hist_F.append(F)
        hist_e.append(err)
        hist_F, hist_e = hist_F[-6:], hist_e[-6:]
        k = len(hist_e)
        Bm = -np.ones((k + 1, k + 1))
        Bm[k, k] = 0.0
        for a in range(k):
            for c in range(k):
                Bm[a, c] = hist_e[a] @ hist_e[c]
        rhs = np.zeros(k + 1)
        rhs[k] = -1.0
        coef = np.linalg.lstsq(Bm, rhs, rcond=None)[0][:k]
        D = densities({g: sum(cf * Fh[g] for cf, Fh in zip(coef, hist_F)) for g in names})
    assert it < 99, "the symmetry-adapted SCF did not converge"
    assert ref["converged"] and abs(E - ref["energy"]) <= 1e-8, (E, ref["energy"])
