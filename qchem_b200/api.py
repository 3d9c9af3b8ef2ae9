"""Python front end of libqchem_b200.so (include/qchem_b200.h), loaded with ctypes.

Two layers:
  Engine         -- one handle: basis upload, Cartesian ERI batches, Schwarz screening, J/K builds,
                    one-electron integrals, RHF.
  OrbitalHFIBS   -- the face qchem's Hartree-Fock code calls, with the reference's method names:
                    Orbital_HF_IBS<double>::AccumulateDirect / AccumulateExchange (+ ...Both)
                    (src/BasisSet/Orbital_HF_IBS.C:33-54) and WholeSystemFock_IBS<double>::AODimension /
                    AddAODensity / MakeAOFock / SliceAOFock (src/BasisSet/Orbital_HF_IBS.C:75-87).
                    J and K for one density come from ONE fused GPU build, memoised by the density, so the
                    reference's separate Coulomb and exchange calls with the same D cost one build.

There is no CPU fallback: if the shared library is missing or no CUDA device is usable, constructing an
Engine raises.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
from typing import Optional, Sequence

import numpy as np

from . import basis as _basis

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libqchem_b200.so")
_lib = None

QCG_OK, QCG_ERR_ARG, QCG_ERR_CUDA, QCG_ERR_NONFINITE, QCG_ERR_ASYMMETRIC, QCG_ERR_ALLOC, QCG_ERR_STATE, \
    QCG_ERR_NOCONV = range(8)
QCG_JK_SKIP_VALIDATION = 1
QCG_JK_FP32 = 4
QCG_JK_DETERMINISTIC = 8

# every symbol include/qchem_b200.h declares
EXPORTS = ["qcg_basis_create", "qcg_destroy", "qcg_last_error", "qcg_set_stream", "qcg_set_memory_limit", "qcg_nbf",
           "qcg_nshell", "qcg_norms", "qcg_eri_batch", "qcg_eri_batch_device", "qcg_schwarz", "qcg_fock_jk",
           "qcg_fock_jk_device", "qcg_one_electron", "qcg_scf_default_params", "qcg_rhf", "qcg_measure_fp64_peak",
           "qcg_fock_jk_device_noalloc", "qcg_eri_batch_f32", "qcg_eri_batch_device_f32", "qcg_set_fp32_bound",
           "qcg_measure_fp32_peak", "qcg_mlp_create", "qcg_mlp_destroy", "qcg_mlp_last_error", "qcg_mlp_set_stream",
           "qcg_mlp_nparams", "qcg_mlp_params", "qcg_mlp_set_params", "qcg_mlp_forward", "qcg_mlp_loss_grad",
           "qcg_mlp_adam", "qcg_basis_create_batch", "qcg_nmol", "qcg_mol_nbf", "qcg_one_electron_batch",
           "qcg_rhf_batch", "qcg_set_graphs", "qcg_set_shard", "qcg_autotune_jk", "qcg_eri3_batch",
           "qcg_nbf_spherical", "qcg_spherical_transform", "qcg_fock_jk_spherical", "qcg_release_cache",
           "qcg_set_eri_team_classes", "qcg_set_pair_subset", "qcg_set_jk_team_classes", "qcg_selftest_bounded_wait", "qcg_shard_work",
           "qcg_salc_fold", "qcg_salc_slice", "qcg_set_jk_warp_classes"]


class QcgError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"qchem_b200 error {code}: {message}")
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("ms_eri", ctypes.c_double), ("quartets", ctypes.c_longlong),
                ("prim_quartets", ctypes.c_longlong), ("flops", ctypes.c_double)]


class ScfParams(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("de_tol", ctypes.c_double), ("fd_tol", ctypes.c_double),
                ("schwarz_thresh", ctypes.c_double), ("diis_nproj", ctypes.c_int), ("diis_fdmax", ctypes.c_double),
                ("diis_svtol", ctypes.c_double), ("incremental", ctypes.c_int), ("inc_thresh", ctypes.c_double),
                ("rebuild_every", ctypes.c_int), ("fp32_early", ctypes.c_int), ("fp32_switch", ctypes.c_double),
                ("fp32_scale", ctypes.c_double), ("fp32_below", ctypes.c_double),
                ("D_guess", ctypes.POINTER(ctypes.c_double)), ("autotune", ctypes.c_int), ("spherical", ctypes.c_int),
                ("deterministic", ctypes.c_int)]


class ScfResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("e_nuc", ctypes.c_double), ("iterations", ctypes.c_int),
                ("converged", ctypes.c_int), ("fd_error", ctypes.c_double), ("wall_s", ctypes.c_double),
                ("fock_ms", ctypes.c_double), ("full_builds", ctypes.c_int), ("incremental_builds", ctypes.c_int),
                ("fp32_builds", ctypes.c_int)]


def library_path() -> str:
    return _LIB_PATH


def lib():
    """Load the CUDA library; raises ImportError if it has not been built (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} not found: build it with `python -m qchem_b200.build`")
    L = ctypes.CDLL(_LIB_PATH)
    vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    P = ctypes.POINTER
    L.qcg_basis_create.argtypes = [P(i32), P(i32), P(f64), P(f64), P(f64), i32, P(vp)]
    L.qcg_basis_create_batch.argtypes = [P(i32), P(i32), P(f64), P(f64), P(f64), i32, P(i32), i32, P(vp)]
    L.qcg_nmol.argtypes = [vp, P(i32)]
    L.qcg_mol_nbf.argtypes = [vp, P(i32)]
    L.qcg_one_electron_batch.argtypes = [vp, P(i32), P(f64), P(f64), P(f64), P(f64), P(f64)]
    L.qcg_rhf_batch.argtypes = [vp, P(i32), P(f64), P(f64), P(i32), P(ScfParams), P(ScfResult), P(f64)]
    L.qcg_destroy.argtypes = [vp]
    L.qcg_destroy.restype = None
    L.qcg_release_cache.argtypes = []
    L.qcg_release_cache.restype = None
    L.qcg_last_error.argtypes = [vp]
    L.qcg_last_error.restype = ctypes.c_char_p
    L.qcg_set_stream.argtypes = [vp, vp]
    L.qcg_set_eri_team_classes.argtypes = [vp, i64]
    L.qcg_set_jk_team_classes.argtypes = [vp, i64]
    L.qcg_set_jk_warp_classes.argtypes = [vp, i64]
    L.qcg_set_pair_subset.argtypes = [vp, vp]
    L.qcg_set_memory_limit.argtypes = [vp, i64]
    L.qcg_nbf.argtypes = [vp, P(i32)]
    L.qcg_nshell.argtypes = [vp, P(i32)]
    L.qcg_norms.argtypes = [vp, P(f64)]
    L.qcg_eri_batch.argtypes = [vp, i32, i32, i32, i32, i64, P(i32), P(f64)]
    L.qcg_eri_batch_device.argtypes = [vp, i32, i32, i32, i32, i64, vp, vp]
    L.qcg_eri_batch_f32.argtypes = [vp, i32, i32, i32, i32, i64, P(i32), P(ctypes.c_float)]
    L.qcg_eri3_batch.argtypes = [vp, i32, i32, i32, i64, P(i32), P(f64)]
    L.qcg_nbf_spherical.argtypes = [vp, P(i32)]
    L.qcg_spherical_transform.argtypes = [vp, P(f64)]
    L.qcg_fock_jk_spherical.argtypes = [vp, P(f64), P(f64), P(f64), i32, P(Stats)]
    L.qcg_eri_batch_device_f32.argtypes = [vp, i32, i32, i32, i32, i64, vp, vp]
    L.qcg_set_fp32_bound.argtypes = [vp, f64]
    L.qcg_set_graphs.argtypes = [vp, i32]
    L.qcg_set_shard.argtypes = [vp, i32, i32]
    L.qcg_shard_work.argtypes = [vp, i32, i32, P(i64), P(i64)]
    L.qcg_salc_fold.argtypes = [vp, i32, P(f64), P(f64), P(f64)]
    L.qcg_salc_slice.argtypes = [vp, i32, P(f64), P(f64), P(f64)]
    L.qcg_autotune_jk.argtypes = [vp, vp, i32, P(i32), P(i32)]
    L.qcg_schwarz.argtypes = [vp, f64, P(f64)]
    L.qcg_fock_jk.argtypes = [vp, P(f64), P(f64), P(f64), i32, P(Stats)]
    L.qcg_fock_jk_device.argtypes = [vp, vp, vp, vp, i32, P(Stats)]
    L.qcg_one_electron.argtypes = [vp, i32, P(f64), P(f64), P(f64), P(f64), P(f64)]
    L.qcg_scf_default_params.argtypes = [P(ScfParams)]
    L.qcg_scf_default_params.restype = None
    L.qcg_rhf.argtypes = [vp, i32, P(f64), P(f64), i32, P(ScfParams), P(ScfResult), P(f64)]
    L.qcg_internal_syev.argtypes = [i32, P(f64), P(f64), P(f64)]
    L.qcg_internal_gemm_bf16.argtypes = [i32, i32, i32, i32, i32, vp, i32, vp, i32, vp, i32, vp, i32]
    L.qcg_internal_syev_lowest.argtypes = [i32, P(f64), i32, P(f64), P(f64)]
    L.qcg_internal_orthogonaliser.argtypes = [i32, P(f64), P(f64)]
    L.qcg_internal_null_modes.argtypes = [i32, P(f64)]
    L.qcg_measure_fp64_peak.argtypes = [i32, P(f64), P(f64)]
    L.qcg_measure_fp32_peak.argtypes = [i32, P(f64), P(f64)]
    L.qcg_selftest_bounded_wait.argtypes = [ctypes.c_longlong, i32, P(i32), P(f64)]
    f32 = ctypes.c_float
    L.qcg_mlp_create.argtypes = [i32, P(i32), ctypes.c_ulonglong, P(vp)]
    L.qcg_mlp_destroy.argtypes = [vp]
    L.qcg_mlp_destroy.restype = None
    L.qcg_mlp_last_error.argtypes = [vp]
    L.qcg_mlp_last_error.restype = ctypes.c_char_p
    L.qcg_mlp_set_stream.argtypes = [vp, vp]
    L.qcg_mlp_nparams.argtypes = [vp, P(i64)]
    L.qcg_mlp_params.argtypes = [vp, P(f32)]
    L.qcg_mlp_set_params.argtypes = [vp, P(f32)]
    L.qcg_mlp_forward.argtypes = [vp, i32, vp, vp]
    L.qcg_mlp_loss_grad.argtypes = [vp, i32, vp, vp, vp, P(f32), P(f32)]
    L.qcg_mlp_adam.argtypes = [vp, f32, f32, f32, f32, f32]
    _lib = L
    return L


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def syev(A: np.ndarray):
    """The SCF's host eigensolver (exposed for tests)."""
    A = _f64(A)
    n = A.shape[0]
    w, V = np.zeros(n), np.zeros((n, n))
    rc = lib().qcg_internal_syev(n, _p(A), _p(w), _p(V))
    if rc != QCG_OK:
        raise QcgError(rc, "eigensolver failed")
    return w, V


def syev_lowest(A: np.ndarray, k: int):
    """The SCF step's partial host eigensolver (exposed for tests): the k lowest eigenvalues (ascending) and
    their eigenvectors (columns)."""
    A = _f64(A)
    n = A.shape[0]
    w, V = np.zeros(n), np.zeros((n, n))
    rc = lib().qcg_internal_syev_lowest(n, _p(A), int(k), _p(w), _p(V))
    if rc != QCG_OK:
        raise QcgError(rc, "eigensolver failed")
    return w[:k], V[:, :k]


def orthogonaliser(S: np.ndarray):
    """The host SCF's orthogonaliser X = L^{-T} (S = L L^T), exposed for tests; None if S is not positive
    definite (the SCF then falls back to U s^{-1/2})."""
    S = _f64(S)
    n = S.shape[0]
    X = np.zeros((n, n))
    return X if lib().qcg_internal_orthogonaliser(n, _p(S), _p(X)) == 1 else None


def release_cache() -> None:
    """Free the idle device slabs, pinned staging buffers, streams and events that destroyed handles left
    for reuse (qcg_release_cache)."""
    lib().qcg_release_cache()


def null_modes(w) -> int:
    """overlap modes the SCF's orthogonaliser drops, for ascending overlap eigenvalues w (the reference's
    automatic rule: a clean spectral gap, else the eigenvalues below 1e-8)"""
    w = _f64(w)
    return int(lib().qcg_internal_null_modes(len(w), _p(w)))


def measure_fp64_peak(reps: int = 20):
    """(TFLOP/s, ms per launch) of the library's pure-DFMA probe kernel on the current device."""
    tf, ms = ctypes.c_double(), ctypes.c_double()
    rc = lib().qcg_measure_fp64_peak(int(reps), ctypes.byref(tf), ctypes.byref(ms))
    if rc != QCG_OK:
        raise QcgError(rc, "fp64 peak probe failed")
    return tf.value, ms.value


def measure_fp32_peak(reps: int = 20):
    """(TFLOP/s, ms per launch) of the library's pure-FFMA probe kernel on the current device."""
    tf, ms = ctypes.c_double(), ctypes.c_double()
    rc = lib().qcg_measure_fp32_peak(int(reps), ctypes.byref(tf), ctypes.byref(ms))
    if rc != QCG_OK:
        raise QcgError(rc, "fp32 peak probe failed")
    return tf.value, ms.value


def selftest_bounded_wait(polls: int, arrive: bool):
    """(gave_up, ms) of the team kernels' bounded mbarrier wait run on its own: with arrive the barrier's one
    expected arrival comes first and the wait completes; without it the wait gives up after `polls` polls."""
    gave, ms = ctypes.c_int(), ctypes.c_double()
    rc = lib().qcg_selftest_bounded_wait(int(polls), 1 if arrive else 0, ctypes.byref(gave), ctypes.byref(ms))
    if rc != QCG_OK:
        raise QcgError(rc, "bounded-wait self-test failed")
    return bool(gave.value), ms.value


class Engine:
    """One basis on the current CUDA device."""

    def __init__(self, shells: Sequence[_basis.Shell]):
        self.shells = list(shells)
        L, npr, cen, ex, co = _basis.flatten(self.shells)
        h = ctypes.c_void_p()
        rc = lib().qcg_basis_create(_p(L, ctypes.c_int), _p(npr, ctypes.c_int), _p(ex), _p(co), _p(cen),
                                    len(self.shells), ctypes.byref(h))
        self._h = h
        if rc != QCG_OK:
            msg = lib().qcg_last_error(h).decode() if h.value else "qcg_basis_create failed"
            self.close()
            raise QcgError(rc, msg)
        n = ctypes.c_int()
        lib().qcg_nbf(self._h, ctypes.byref(n))
        self.nbf = n.value
        self.offsets = np.cumsum([0] + [s.nfunc for s in self.shells])[:-1]
        self._screen = None

    # -- lifetime ------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().qcg_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != QCG_OK:
            raise QcgError(rc, lib().qcg_last_error(self._h).decode())

    def set_stream(self, stream_ptr: int):
        """All later work of this engine goes to CUDA stream `stream_ptr` (0 = the legacy default stream)."""
        self._check(lib().qcg_set_stream(self._h, ctypes.c_void_p(int(stream_ptr))))

    def set_memory_limit(self, nbytes: int):
        self._check(lib().qcg_set_memory_limit(self._h, int(nbytes)))

    def norms(self) -> np.ndarray:
        ns = np.zeros(self.nbf)
        self._check(lib().qcg_norms(self._h, _p(ns)))
        return ns

    # -- integrals -----------------------------------------------------------------------------
    def eri_batch(self, cls, quartets, fp32: bool = False) -> np.ndarray:
        """Cartesian ERI blocks of one class; fp32=True evaluates them in FP32 (float32 output)."""
        q = np.ascontiguousarray(quartets, dtype=np.int32)
        la, lb, lc, ld = cls
        nf = [(l + 1) * (l + 2) // 2 for l in cls]
        out = np.zeros((len(q), nf[0] * nf[1] * nf[2] * nf[3]), dtype=np.float32 if fp32 else np.float64)
        if fp32:
            self._check(lib().qcg_eri_batch_f32(self._h, la, lb, lc, ld, len(q), _p(q, ctypes.c_int),
                                                _p(out, ctypes.c_float)))
        else:
            self._check(lib().qcg_eri_batch(self._h, la, lb, lc, ld, len(q), _p(q, ctypes.c_int), _p(out)))
        return out

    # -- spherical (real solid-harmonic) functions ----------------------------------------------
    @property
    def nbf_spherical(self) -> int:
        n = ctypes.c_int()
        self._check(lib().qcg_nbf_spherical(self._h, ctypes.byref(n)))
        return n.value

    def spherical_transform(self) -> np.ndarray:
        """T (nbf x nbf_spherical): chi_s = sum_t T[t, s] phi_t, components ordered m = -l..l per shell."""
        T = np.zeros((self.nbf, self.nbf_spherical))
        self._check(lib().qcg_spherical_transform(self._h, _p(T)))
        return T

    def fock_jk_spherical(self, D, validate: bool = True):
        if self._screen is None:
            self.schwarz()
        ns = self.nbf_spherical
        D = _f64(D)
        if D.shape != (ns, ns):
            raise QcgError(QCG_ERR_ARG, f"spherical density must be {ns}x{ns}")
        J, K = np.zeros_like(D), np.zeros_like(D)
        st = Stats()
        self._check(lib().qcg_fock_jk_spherical(self._h, _p(D), _p(J), _p(K), 0 if validate else QCG_JK_SKIP_VALIDATION,
                                                ctypes.byref(st)))
        return J, K, st

    def eri3_batch(self, cls3, triples) -> np.ndarray:
        """3-centre Coulomb blocks (ab|c) of shell triples of class (la, lb, lc), la >= lb."""
        t = np.ascontiguousarray(triples, dtype=np.int32)
        la, lb, lc = cls3
        nf = [(l + 1) * (l + 2) // 2 for l in cls3]
        out = np.zeros((len(t), nf[0] * nf[1] * nf[2]))
        self._check(lib().qcg_eri3_batch(self._h, la, lb, lc, len(t), _p(t, ctypes.c_int), _p(out)))
        return out

    def eri_batch_device(self, cls, d_quartets_ptr: int, nq: int, d_out_ptr: int, fp32: bool = False):
        la, lb, lc, ld = cls
        f = lib().qcg_eri_batch_device_f32 if fp32 else lib().qcg_eri_batch_device
        self._check(f(self._h, la, lb, lc, ld, int(nq), ctypes.c_void_p(d_quartets_ptr), ctypes.c_void_p(d_out_ptr)))

    def set_shard(self, rank: int, world: int):
        """Later J/K builds evaluate this rank's slice of the quartets (1/world of every class's primitive
        quartets) and return partial J and K (summed over ranks they are the full build)."""
        self._check(lib().qcg_set_shard(self._h, int(rank), int(world)))

    def shard_work(self, rank: int, world: int):
        """(screened quartets, primitive quartets) of share `rank` of `world` under set_shard."""
        if self._screen is None:
            self.schwarz()
        nq, npq = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(lib().qcg_shard_work(self._h, int(rank), int(world), ctypes.byref(nq), ctypes.byref(npq)))
        return nq.value, npq.value

    def autotune_jk(self, d_D: int, reps: int = 1):
        """Tune the J/K launch shape of every class on the density at device pointer d_D; returns the chosen
        (quartets per lane, blocks per SM) per class (0 for classes with no quartets)."""
        if self._screen is None:
            self.schwarz()
        run, cap = np.zeros(21, dtype=np.int32), np.zeros(21, dtype=np.int32)
        self._check(lib().qcg_autotune_jk(self._h, ctypes.c_void_p(d_D), int(reps), _p(run, ctypes.c_int),
                                          _p(cap, ctypes.c_int)))
        return list(zip(run.tolist(), cap.tolist()))

    def set_graphs(self, enable: bool):
        """Replay repeated J/K builds as CUDA graphs (off by default)."""
        self._check(lib().qcg_set_graphs(self._h, int(bool(enable))))

    def set_eri_team_classes(self, mask: int):
        """FP64 ERI-batch classes (bit k: class k) evaluated by the team-form kernel; -1 restores the default."""
        self._check(lib().qcg_set_eri_team_classes(self._h, ctypes.c_longlong(mask)))

    def set_jk_team_classes(self, mask: int):
        """J/K-build classes (bit k: class k) run by the team kernel; -1 restores the default."""
        self._check(lib().qcg_set_jk_team_classes(self._h, ctypes.c_longlong(mask)))

    def set_jk_warp_classes(self, mask: int):
        """J/K-build classes (bit k: class k) run in the warp-shared form (the team form takes precedence);
        -1 restores the default."""
        self._check(lib().qcg_set_jk_warp_classes(self._h, ctypes.c_longlong(mask)))

    def set_pair_subset(self, mask):
        """Later J/K builds evaluate only quartets whose two shell pairs are both in the subset (mask: nshell x
        nshell booleans); None restores every quartet."""
        if mask is None:
            self._check(lib().qcg_set_pair_subset(self._h, None))
            return
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8))
        ns = len(self.shells)
        if m.shape != (ns, ns):
            raise ValueError(f"mask must be {ns} x {ns}")
        self._check(lib().qcg_set_pair_subset(self._h, m.ctypes.data_as(ctypes.c_void_p)))

    def set_fp32_bound(self, bound: float):
        """Later J/K builds evaluate quartets with Q_ab Q_cd < bound in FP32 (FP64 accumulation)."""
        self._check(lib().qcg_set_fp32_bound(self._h, float(bound)))

    def schwarz(self, thresh: float = 1e-10) -> np.ndarray:
        ns = len(self.shells)
        Q = np.zeros((ns, ns))
        self._check(lib().qcg_schwarz(self._h, float(thresh), _p(Q)))
        self._screen = thresh
        return Q

    def fock_jk(self, D, validate: bool = True, fp32: bool = False, deterministic: bool = False):
        """J[D], K[D] (unscaled) and the build's Stats; fp32=True evaluates every quartet in FP32;
        deterministic=True accumulates in exact integer pairs (the same bits on every build)."""
        if self._screen is None:
            self.schwarz()
        D = _f64(D)
        if D.shape != (self.nbf, self.nbf):
            raise QcgError(QCG_ERR_ARG, f"density must be {self.nbf}x{self.nbf}")
        J, K = np.zeros_like(D), np.zeros_like(D)
        st = Stats()
        flags = ((0 if validate else QCG_JK_SKIP_VALIDATION) | (QCG_JK_FP32 if fp32 else 0) |
                 (QCG_JK_DETERMINISTIC if deterministic else 0))
        self._check(lib().qcg_fock_jk(self._h, _p(D), _p(J), _p(K), flags, ctypes.byref(st)))
        return J, K, st

    def fock_jk_device(self, d_D: int, d_J: int, d_K: int, validate: bool = False, fp32: bool = False,
                       deterministic: bool = False) -> Stats:
        if self._screen is None:
            self.schwarz()
        st = Stats()
        flags = ((0 if validate else QCG_JK_SKIP_VALIDATION) | (QCG_JK_FP32 if fp32 else 0) |
                 (QCG_JK_DETERMINISTIC if deterministic else 0))
        self._check(lib().qcg_fock_jk_device(self._h, ctypes.c_void_p(d_D), ctypes.c_void_p(d_J), ctypes.c_void_p(d_K),
                                             flags, ctypes.byref(st)))
        return st

    def one_electron(self, mol: _basis.Molecule):
        n = self.nbf
        Z = _f64(mol.Z)
        R = _f64(mol.R).reshape(-1)
        S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
        self._check(lib().qcg_one_electron(self._h, len(Z), _p(Z), _p(R), _p(S), _p(T), _p(V)))
        return S, T, V

    def rhf(self, mol: _basis.Molecule, max_iter=100, de_tol=1e-10, fd_tol=1e-5, schwarz_thresh=1e-10,
            want_density=False, incremental=False, inc_thresh=1e-11, rebuild_every=8, fp32_early=False,
            fp32_switch=1e-5, fp32_scale=0.0, fp32_below=0.0, guess=None, diis_nproj=4, diis_fdmax=0.0,
            autotune=False, spherical=False, deterministic=False):
        """RHF to convergence.  incremental=True: density-difference J/K builds with density-weighted
        screening between full builds (the energy on exit is always from a full build).  fp32_early=True:
        until the DIIS error drops below fp32_switch, quartets whose density-weighted bound is below
        fp32_scale x (DIIS error) are FP32; fp32_below: quartets with a smaller bound stay FP32 afterwards
        (the build that confirms convergence is all-FP64).  guess: initial total density (nbf x nbf)
        instead of the core-Hamiltonian guess."""
        prm = ScfParams()
        lib().qcg_scf_default_params(ctypes.byref(prm))
        prm.max_iter, prm.de_tol, prm.fd_tol, prm.schwarz_thresh = max_iter, de_tol, fd_tol, schwarz_thresh
        prm.incremental, prm.inc_thresh, prm.rebuild_every = int(incremental), float(inc_thresh), int(rebuild_every)
        prm.fp32_early, prm.fp32_switch, prm.fp32_below = int(fp32_early), float(fp32_switch), float(fp32_below)
        prm.fp32_scale = float(fp32_scale)
        prm.diis_nproj, prm.diis_fdmax = int(diis_nproj), float(diis_fdmax)
        prm.autotune = int(bool(autotune))
        prm.spherical = int(bool(spherical))
        prm.deterministic = int(bool(deterministic))
        nw = self.nbf_spherical if spherical else self.nbf
        if guess is not None:
            guess = _f64(guess)
            if guess.shape != (nw, nw):
                raise QcgError(QCG_ERR_ARG, f"guess density must be {nw}x{nw}")
            prm.D_guess = _p(guess)
        res = ScfResult()
        Z = _f64(mol.Z)
        R = _f64(mol.R).reshape(-1)
        D = np.zeros((nw, nw)) if want_density else None
        rc = lib().qcg_rhf(self._h, len(Z), _p(Z), _p(R), int(mol.nelec), ctypes.byref(prm), ctypes.byref(res),
                           _p(D) if D is not None else None)
        if rc not in (QCG_OK, QCG_ERR_NOCONV):
            self._check(rc)
        self._screen = schwarz_thresh
        out = {"energy": res.energy, "e_nuc": res.e_nuc, "iterations": res.iterations,
               "converged": bool(res.converged), "fd_error": res.fd_error, "wall_s": res.wall_s,
               "fock_ms": res.fock_ms, "full_builds": res.full_builds, "incremental_builds": res.incremental_builds,
               "fp32_builds": res.fp32_builds}
        if D is not None:
            out["D"] = D
        return out


class BatchEngine(Engine):
    """Several molecules in one handle (qcg_basis_create_batch): one J/K build covers all of them, and
    rhf() advances all their SCFs together.  Matrices cross the C ABI packed (molecule blocks one after
    the other); this class packs and unpacks lists of per-molecule arrays."""

    def __init__(self, shell_lists: Sequence[Sequence[_basis.Shell]]):
        self.shell_lists = [list(x) for x in shell_lists]
        self.shells = [s for x in self.shell_lists for s in x]
        L, npr, cen, ex, co = _basis.flatten(self.shells)
        mol = np.concatenate([np.full(len(x), m, dtype=np.int32) for m, x in enumerate(self.shell_lists)])
        h = ctypes.c_void_p()
        rc = lib().qcg_basis_create_batch(_p(L, ctypes.c_int), _p(npr, ctypes.c_int), _p(ex), _p(co), _p(cen),
                                          len(self.shells), _p(mol, ctypes.c_int), len(self.shell_lists),
                                          ctypes.byref(h))
        self._h = h
        if rc != QCG_OK:
            msg = lib().qcg_last_error(h).decode() if h.value else "qcg_basis_create_batch failed"
            self.close()
            raise QcgError(rc, msg)
        self.nmol = len(self.shell_lists)
        nb = np.zeros(self.nmol, dtype=np.int32)
        self._check(lib().qcg_mol_nbf(self._h, _p(nb, ctypes.c_int)))
        self.mol_nbf = [int(x) for x in nb]
        self.nbf = int(nb.sum())
        self.packed_off = np.concatenate([[0], np.cumsum([n * n for n in self.mol_nbf])])
        self._screen = None

    def pack(self, mats):
        return np.concatenate([_f64(m).reshape(-1) for m in mats])

    def unpack(self, flat):
        return [flat[self.packed_off[m]:self.packed_off[m + 1]].reshape(n, n) for m, n in enumerate(self.mol_nbf)]

    def fock_jk(self, Ds, validate: bool = True, fp32: bool = False, deterministic: bool = False):
        if self._screen is None:
            self.schwarz()
        D = self.pack(Ds)
        J, K = np.zeros_like(D), np.zeros_like(D)
        st = Stats()
        flags = ((0 if validate else QCG_JK_SKIP_VALIDATION) | (QCG_JK_FP32 if fp32 else 0) |
                 (QCG_JK_DETERMINISTIC if deterministic else 0))
        self._check(lib().qcg_fock_jk(self._h, _p(D), _p(J), _p(K), flags, ctypes.byref(st)))
        return self.unpack(J), self.unpack(K), st

    def schwarz(self, thresh: float = 1e-10):
        self._check(lib().qcg_schwarz(self._h, float(thresh), None))
        self._screen = thresh

    def rhf(self, mols: Sequence[_basis.Molecule], max_iter=100, de_tol=1e-10, fd_tol=1e-5, schwarz_thresh=1e-10,
            want_density=False, diis_nproj=4, diis_fdmax=0.0, autotune=False, guesses=None, deterministic=False):
        """guesses: optional list of per-molecule initial densities (None entries are not allowed; omit the
        argument for the core guess everywhere)."""
        prm = ScfParams()
        lib().qcg_scf_default_params(ctypes.byref(prm))
        prm.max_iter, prm.de_tol, prm.fd_tol, prm.schwarz_thresh = max_iter, de_tol, fd_tol, schwarz_thresh
        prm.diis_nproj, prm.diis_fdmax = int(diis_nproj), float(diis_fdmax)
        prm.autotune = int(bool(autotune))
        prm.deterministic = int(bool(deterministic))
        Dg = None
        if guesses is not None:
            if len(guesses) != len(mols):
                raise QcgError(QCG_ERR_ARG, "one guess density per molecule")
            Dg = self.pack(guesses)
            prm.D_guess = _p(Dg)
        nat = np.array([len(m.Z) for m in mols], dtype=np.int32)
        Z = _f64(np.concatenate([np.asarray(m.Z, dtype=float) for m in mols]))
        R = _f64(np.concatenate([np.asarray(m.R, dtype=float).reshape(-1) for m in mols]))
        ne = np.array([m.nelec for m in mols], dtype=np.int32)
        res = (ScfResult * len(mols))()
        D = np.zeros(int(self.packed_off[-1])) if want_density else None
        rc = lib().qcg_rhf_batch(self._h, _p(nat, ctypes.c_int), _p(Z), _p(R), _p(ne, ctypes.c_int),
                                 ctypes.byref(prm), res, _p(D) if D is not None else None)
        if rc not in (QCG_OK, QCG_ERR_NOCONV):
            self._check(rc)
        self._screen = schwarz_thresh
        out = [{"energy": r.energy, "e_nuc": r.e_nuc, "iterations": r.iterations, "converged": bool(r.converged),
                "fd_error": r.fd_error, "wall_s": r.wall_s, "fock_ms": r.fock_ms, "builds": r.full_builds}
               for r in res]
        if D is not None:
            for o, d in zip(out, self.unpack(D)):
                o["D"] = d
        return out


class Mlp:
    """The learned-guess network on the current CUDA device (include/qchem_b200.h, qcg_mlp_*): BF16-operand,
    FP32-accumulated forward/backward kernels and Adam.  Activations, targets and masks are passed as device
    pointers (row-major float32)."""

    def __init__(self, widths: Sequence[int], seed: int = 0):
        self.widths = [int(w) for w in widths]
        w = np.array(self.widths, dtype=np.int32)
        h = ctypes.c_void_p()
        rc = lib().qcg_mlp_create(len(w) - 1, _p(w, ctypes.c_int), ctypes.c_ulonglong(seed), ctypes.byref(h))
        if rc != QCG_OK:
            raise QcgError(rc, "qcg_mlp_create failed")
        self._h = h
        n = ctypes.c_longlong()
        lib().qcg_mlp_nparams(self._h, ctypes.byref(n))
        self.nparams = n.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().qcg_mlp_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != QCG_OK:
            raise QcgError(rc, lib().qcg_mlp_last_error(self._h).decode())

    def set_stream(self, stream_ptr: int):
        self._check(lib().qcg_mlp_set_stream(self._h, ctypes.c_void_p(int(stream_ptr))))

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        self._check(lib().qcg_mlp_params(self._h, _p(p, ctypes.c_float)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparams:
            raise QcgError(QCG_ERR_ARG, f"expected {self.nparams} parameters")
        self._check(lib().qcg_mlp_set_params(self._h, _p(p, ctypes.c_float)))

    def forward(self, rows: int, d_x: int, d_y: int):
        self._check(lib().qcg_mlp_forward(self._h, int(rows), ctypes.c_void_p(d_x), ctypes.c_void_p(d_y)))

    def loss_grad(self, rows: int, d_x: int, d_t: int, d_mask: int, want_grad: bool = False):
        loss = ctypes.c_float()
        g = np.zeros(self.nparams, dtype=np.float32) if want_grad else None
        self._check(lib().qcg_mlp_loss_grad(self._h, int(rows), ctypes.c_void_p(d_x), ctypes.c_void_p(d_t),
                                            ctypes.c_void_p(d_mask), ctypes.byref(loss),
                                            _p(g, ctypes.c_float) if g is not None else None))
        return (loss.value, g) if want_grad else loss.value

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self._check(lib().qcg_mlp_adam(self._h, lr, beta1, beta2, eps, weight_decay))


class OrbitalHFIBS:
    """qchem's HF contraction face over the GPU engine (one irrep: the whole AO basis).

    AccumulateDirect(S, D):    S += J[D],  J_ab = sum_cd (ab|cd) D_cd   (Orbital_HF_IBS.C:36-37)
    AccumulateExchange(S, D):  S += K[D],  K_ac = sum_bd (ab|cd) D_bd   (unscaled; the caller applies -1/2)
    MakeAOFock(Dao, exchange): the whole-system J (exchange=False) or K (exchange=True) (Orbital_HF_IBS.C:84)
    """

    def __init__(self, engine: Engine, schwarz_thresh: float = 1e-10):
        self.engine = engine
        self.thresh = schwarz_thresh
        self._memo_key = None
        self._memo = None
        self.builds = 0

    def _jk(self, D):
        D = _f64(D)
        if not np.all(np.isfinite(D)):
            raise QcgError(QCG_ERR_NONFINITE, "density matrix has NaN/Inf entries")
        key = hashlib.sha1(D.tobytes()).hexdigest()
        if key != self._memo_key:
            if self.engine._screen != self.thresh:
                self.engine.schwarz(self.thresh)
            J, K, _ = self.engine.fock_jk(D)
            self._memo_key, self._memo = key, (J, K)
            self.builds += 1
        return self._memo

    # Orbital_HF_IBS<double>
    def AccumulateDirect(self, Sab, Dcd, bs_cd=None):
        Sab += self._jk(Dcd)[0]

    def AccumulateExchange(self, Sab, Dcd, bs_cd=None):
        Sab += self._jk(Dcd)[1]

    def AccumulateDirectBoth(self, Ji, Jj, Di, Dj, cd=None):
        # one irrep: the pair is the diagonal (i == j) block
        Ji += self._jk(Dj)[0]
        if Jj is not Ji:
            Jj += self._jk(Di)[0]

    def AccumulateExchangeBoth(self, Ki, Kj, Di, Dj, cd=None):
        Ki += self._jk(Dj)[1]
        if Kj is not Ki:
            Kj += self._jk(Di)[1]

    # WholeSystemFock_IBS<double>
    def AODimension(self) -> int:
        return self.engine.nbf

    def AddAODensity(self, Dao, D):
        Dao += D

    def MakeAOFock(self, Dao, exchange: bool):
        J, K = self._jk(Dao)
        return (K if exchange else J).copy()

    def SliceAOFock(self, Fab, Fao):
        Fab += Fao


class SymmetryAdaptedIBS:
    """One irrep block of a symmetry-adapted (SALC) basis over the AO engine: qchem's SymmetryAdapted_IBS
    (src/BasisSet/Imp/SymmetryAdapted_IBS.C:45-140).  The block is m functions, the columns of O
    (nbf x m, over the engine's Cartesian AO functions); `ao` is the whole-molecule HF face (OrbitalHFIBS)
    whose one AO build every block shares.

    WholeSystemFock_IBS:  AODimension(); AddAODensity(Dao, D): Dao += sym(O D O^T);
                          MakeAOFock(Dao, exchange): the AO J or K of Dao (one build, memoised on Dao);
                          SliceAOFock(Fab, Fao): Fab += sym(O^T Fao O).
    Orbital_HF_IBS:       AccumulateDirect(Jab, Dcd, bs_cd): the partner bs_cd folds its block's density up,
                          one AO build, this block slices (PairAOFock); AccumulateExchange likewise;
                          the ...Both forms serve the pair as two slices, skipping a zero density.
    Transform(M):         sym(O^T M O) of an AO matrix (overlap, kinetic, nuclear).
    The folds and slices run on the GPU (qcg_salc_fold / qcg_salc_slice).
    """

    def __init__(self, ao: "OrbitalHFIBS", O, label: str = ""):
        self.ao = ao
        self.O = np.ascontiguousarray(O, dtype=np.float64)
        n = ao.engine.nbf
        if self.O.ndim != 2 or self.O.shape[0] != n or not 1 <= self.O.shape[1] <= n:
            raise QcgError(QCG_ERR_ARG, f"O must be nbf x m with 1 <= m <= nbf (nbf = {n})")
        self.m = self.O.shape[1]
        self.label = label

    def _h(self):
        return self.ao.engine._h

    # WholeSystemFock_IBS<double>
    def AODimension(self) -> int:
        return self.ao.engine.nbf

    def AddAODensity(self, Dao, D):
        D = _f64(D)
        if Dao.dtype != np.float64 or not Dao.flags.c_contiguous:
            raise QcgError(QCG_ERR_ARG, "Dao must be a C-contiguous float64 array")
        self.ao.engine._check(lib().qcg_salc_fold(self._h(), self.m, _p(self.O), _p(D), _p(Dao)))

    def MakeAOFock(self, Dao, exchange: bool):
        if not np.any(Dao):
            return np.zeros_like(_f64(Dao))   # the reference's pre-screen: an empty density builds nothing
        return self.ao.MakeAOFock(Dao, exchange)

    def SliceAOFock(self, Fab, Fao):
        Fao = _f64(Fao)
        if Fab.dtype != np.float64 or not Fab.flags.c_contiguous:
            raise QcgError(QCG_ERR_ARG, "Fab must be a C-contiguous float64 array")
        self.ao.engine._check(lib().qcg_salc_slice(self._h(), self.m, _p(self.O), _p(Fao), _p(Fab)))

    def Transform(self, M):
        out = np.zeros((self.m, self.m))
        self.SliceAOFock(out, M)
        return out

    # Orbital_HF_IBS<double>
    def PairAOFock(self, Dcd, bs_cd: "SymmetryAdaptedIBS", exchange: bool):
        if not isinstance(bs_cd, SymmetryAdaptedIBS):
            raise QcgError(QCG_ERR_ARG, "the HF partner basis has no whole-system Fock face")
        Dao = np.zeros((self.AODimension(), self.AODimension()))
        bs_cd.AddAODensity(Dao, Dcd)   # the partner folds with its own columns
        return self.MakeAOFock(Dao, exchange)

    def AccumulateDirect(self, Jab, Dcd, bs_cd):
        self.SliceAOFock(Jab, self.PairAOFock(Dcd, bs_cd, False))

    def AccumulateExchange(self, Kab, Dcd, bs_cd):
        self.SliceAOFock(Kab, self.PairAOFock(Dcd, bs_cd, True))

    def AccumulateDirectBoth(self, Ji, Jj, Di, Dj, cd):
        if np.any(Dj):
            self.AccumulateDirect(Ji, Dj, cd)
        if np.any(Di):
            cd.AccumulateDirect(Jj, Di, self)

    def AccumulateExchangeBoth(self, Ki, Kj, Di, Dj, cd):
        if np.any(Dj):
            self.AccumulateExchange(Ki, Dj, cd)
        if np.any(Di):
            cd.AccumulateExchange(Kj, Di, self)
