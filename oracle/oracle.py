"""ctypes front end of the CPU oracle (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and bench.py (cpu_baseline / --impl reference) as the checker and
the CPU baseline.  The product package never imports this module.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
        P = ctypes.POINTER
        L.orc_basis_new.restype = vp
        L.orc_basis_free.argtypes = [vp]
        L.orc_basis_add_shell.argtypes = [vp, i32, P(f64), i32, P(f64), P(f64)]
        L.orc_basis_finalize.argtypes = [vp]
        L.orc_basis_finalize.restype = i32
        L.orc_basis_norms.argtypes = [vp, P(f64)]
        L.orc_boys.argtypes = [f64, i32, P(f64)]
        L.orc_boys_table.argtypes = [P(f64)]
        L.orc_fourc.argtypes = [vp, i32, i32, i32, i32]
        L.orc_fourc.restype = f64
        L.orc_shell_quartet.argtypes = [vp, i32, i32, i32, i32, P(f64)]
        L.orc_eri_batch.argtypes = [vp, i64, P(i32), i64, P(f64), i32]
        L.orc_eri3_batch.argtypes = [vp, i64, P(i32), i64, P(f64), i32]
        L.orc_one_electron.argtypes = [vp, i32, P(f64), P(f64), P(f64), P(f64), P(f64)]
        L.orc_schwarz.argtypes = [vp, P(f64)]
        L.orc_jk_direct.argtypes = [vp, P(f64), P(f64), P(f64), f64, i32]
        L.orc_jk_direct.restype = i64
        L.orc_jk_eri4.argtypes = [vp, P(f64), P(f64), P(f64)]
        L.orc_jk_direct_shard.argtypes = [vp, P(f64), P(f64), P(f64), f64, i32, i32, i32]
        L.orc_jk_direct_shard.restype = i64
        L.orc_jk_direct_subset.argtypes = [vp, P(f64), P(f64), P(f64), f64, i32, vp]
        L.orc_jk_direct_subset.restype = i64
        L.orc_rhf.argtypes = [vp, i32, P(f64), P(f64), i32, i32, f64, f64, i32, i32, P(f64), P(i32), P(f64),
                              P(f64)]
        L.orc_rhf.restype = i32
        L.orc_rhf2.argtypes = [vp, i32, P(f64), P(f64), i32, i32, f64, f64, i32, i32, f64, P(f64), P(i32), P(f64),
                               P(f64)]
        L.orc_rhf2.restype = i32
        L.orc_null_modes.argtypes = [i32, P(f64)]
        L.orc_null_modes.restype = i32
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def boys(T, jmax):
    F = np.zeros(jmax + 1)
    lib().orc_boys(float(T), int(jmax), _p(F))
    return F


def boys_table():
    t = np.zeros((121, 23))
    lib().orc_boys_table(_p(t))
    return t


class OracleBasis:
    """The oracle's copy of a shell list (qchem_b200.basis.Shell objects or equivalent)."""

    def __init__(self, shells):
        self.h = lib().orc_basis_new()
        self.shells = list(shells)
        for s in self.shells:
            c = np.ascontiguousarray(s.centre, dtype=np.float64)
            e = np.ascontiguousarray(s.exps, dtype=np.float64)
            k = np.ascontiguousarray(s.coefs, dtype=np.float64)
            lib().orc_basis_add_shell(self.h, int(s.L), _p(c), len(e), _p(e), _p(k))
        self.nbf = lib().orc_basis_finalize(self.h)
        self.offsets = np.cumsum([0] + [s.nfunc for s in self.shells])[:-1]

    def __del__(self):
        try:
            lib().orc_basis_free(self.h)
        except Exception:
            pass

    def norms(self):
        ns = np.zeros(self.nbf)
        lib().orc_basis_norms(self.h, _p(ns))
        return ns

    def fourc(self, a, b, c, d):
        return lib().orc_fourc(self.h, a, b, c, d)

    def shell_quartet(self, a, b, c, d):
        s = self.shells
        out = np.zeros((s[a].nfunc, s[b].nfunc, s[c].nfunc, s[d].nfunc))
        lib().orc_shell_quartet(self.h, a, b, c, d, _p(out))
        return out

    def eri_batch(self, quartets, nthreads=0):
        q = np.ascontiguousarray(quartets, dtype=np.int32)
        s = self.shells
        blk = s[q[0, 0]].nfunc * s[q[0, 1]].nfunc * s[q[0, 2]].nfunc * s[q[0, 3]].nfunc
        out = np.zeros((len(q), blk))
        lib().orc_eri_batch(self.h, len(q), _p(q, ctypes.c_int), blk, _p(out), int(nthreads))
        return out

    def eri3_batch(self, triples, nthreads=0):
        """3-centre Coulomb blocks (ab|c), out[t][a][b][c], normalised like the reference's RepulsionThreeC."""
        t = np.ascontiguousarray(triples, dtype=np.int32)
        s = self.shells
        blk = s[t[0, 0]].nfunc * s[t[0, 1]].nfunc * s[t[0, 2]].nfunc
        out = np.zeros((len(t), blk))
        lib().orc_eri3_batch(self.h, len(t), _p(t, ctypes.c_int), blk, _p(out), int(nthreads))
        return out

    def one_electron(self, mol):
        n = self.nbf
        Z = np.ascontiguousarray(mol.Z, dtype=np.float64)
        R = np.ascontiguousarray(mol.R, dtype=np.float64).reshape(-1)
        S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
        lib().orc_one_electron(self.h, len(Z), _p(Z), _p(R), _p(S), _p(T), _p(V))
        return S, T, V

    def schwarz(self):
        ns = len(self.shells)
        Q = np.zeros((ns, ns))
        lib().orc_schwarz(self.h, _p(Q))
        return Q

    def jk_direct(self, D, thresh=1e-10, nthreads=0):
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        J, K = np.zeros((n, n)), np.zeros((n, n))
        cnt = lib().orc_jk_direct(self.h, _p(D), _p(J), _p(K), float(thresh), int(nthreads))
        return J, K, cnt

    def jk_direct_shard(self, D, rank, world, thresh=1e-10, nthreads=0):
        """Share of one rank in a world-way split of the bra shell pairs (ij % world == rank)."""
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        J, K = np.zeros((n, n)), np.zeros((n, n))
        lib().orc_jk_direct_shard(self.h, _p(D), _p(J), _p(K), float(thresh), int(nthreads), int(rank), int(world))
        return J, K

    def jk_direct_subset(self, D, mask, thresh=1e-10, nthreads=0):
        """The direct build restricted to the quartets whose two shell pairs are both in the subset (mask:
        nshell x nshell booleans); returns J, K and the number of quartets evaluated."""
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8))
        J, K = np.zeros((n, n)), np.zeros((n, n))
        cnt = lib().orc_jk_direct_subset(self.h, _p(D), _p(J), _p(K), float(thresh), int(nthreads),
                                         m.ctypes.data_as(ctypes.c_void_p))
        return J, K, int(cnt)

    def jk_eri4(self, D):
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        J, K = np.zeros((n, n)), np.zeros((n, n))
        lib().orc_jk_eri4(self.h, _p(D), _p(J), _p(K))
        return J, K

    def rhf(self, mol, jk_mode=0, thresh=1e-10, dE_tol=1e-10, maxiter=100, nthreads=0, diis_fdmax=0.0):
        """diis_fdmax > 0 replaces the reference's DIIS switch-on bound (the GPU SCF's diis_fdmax)"""
        Z = np.ascontiguousarray(mol.Z, dtype=np.float64)
        R = np.ascontiguousarray(mol.R, dtype=np.float64).reshape(-1)
        E = np.zeros(1)
        it = np.zeros(1, dtype=np.int32)
        D = np.zeros((self.nbf, self.nbf))
        st = np.zeros(5)
        rc = lib().orc_rhf2(self.h, len(Z), _p(Z), _p(R), int(mol.nelec), int(jk_mode), float(thresh),
                            float(dE_tol), int(maxiter), int(nthreads), float(diis_fdmax), _p(E),
                            _p(it, ctypes.c_int), _p(D), _p(st))
        return {"energy": float(E[0]), "iterations": int(it[0]), "converged": rc == 0, "D": D,
                "wall_s": float(st[0]), "jk_s": float(st[1]), "fd_error": float(st[2]), "e_nn": float(st[3]),
                "dropped_modes": int(st[4])}


def null_modes(w) -> int:
    """overlap modes the reference's automatic orthogonaliser drops, for ascending eigenvalues w"""
    w = np.ascontiguousarray(w, dtype=np.float64)
    return int(lib().orc_null_modes(len(w), _p(w)))
