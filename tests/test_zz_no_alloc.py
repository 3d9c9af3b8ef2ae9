"""qcg_fock_jk_device_noalloc: the J/K build for callers that must not allocate device memory after setup
(a host program whose device memory belongs to its own pool allocator, or one held to a fixed budget).

The entry point keeps its accumulators in a fixed device array of the library instead of allocating.  These
tests call it through the C ABI and check it against the allocating entry point qcg_fock_jk_device, twice
in a row (the array keeps the previous call's contents, so the second call also checks that it is cleared).
While it runs, the handle's device-memory cap is set below what the handle already holds, so an allocation
through the handle would fail the call, and the device's free memory is compared across the calls after the
first (which sets the array up), so an allocation outside the handle would show.  It honours the handle's shard (qcg_set_shard: the slices sum to
the whole build) and always builds in FP64 (a mixed-precision bound set on the handle does not apply).
"""
import ctypes

import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W

pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-10   # the J/K tolerance used by the other GPU tests


def _entry():
    L = api.lib()
    f = L.qcg_fock_jk_device_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _setup(seed=21, mol=None):
    import torch
    eng = api.Engine(B.even_tempered(mol or W.water()))
    eng.schwarz(1e-10)
    n = eng.nbf
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, 5)))
    D = torch.tensor(2 * Q @ Q.T, device="cuda", dtype=torch.float64)
    J_ref, K_ref = torch.empty_like(D), torch.empty_like(D)
    eng.fock_jk_device(D.data_ptr(), J_ref.data_ptr(), K_ref.data_ptr())
    torch.cuda.synchronize()
    return eng, D, J_ref, K_ref


def _noalloc(f, eng, D):
    import torch
    J, K = torch.full_like(D, np.nan), torch.full_like(D, np.nan)
    rc = f(eng._h, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()))
    torch.cuda.synchronize()
    assert rc == api.QCG_OK, api.lib().qcg_last_error(eng._h).decode()
    return J, K


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    f = _entry()
    eng, D, J_ref, K_ref = _setup()
    # result buffers first, so that the free-memory comparison sees only the entry point itself
    bufs = [(torch.full_like(D, np.nan), torch.full_like(D, np.nan)) for _ in range(3)]
    torch.cuda.synchronize()
    eng.set_memory_limit(1)   # below current use: any allocation through the handle would now fail
    try:
        free0 = None
        for i, (J, K) in enumerate(bufs):
            if i == 1:
                # the first call on the device looks up the array's address, and with lazy module loading
                # the CUDA driver materialises the library's static array then; from here on free memory must
                # not move
                free0 = torch.cuda.mem_get_info()[0]
            rc = f(eng._h, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()))
            torch.cuda.synchronize()
            assert rc == api.QCG_OK, api.lib().qcg_last_error(eng._h).decode()
            assert torch.abs(J - J_ref).max().item() <= FOCK_TOL
            assert torch.abs(K - K_ref).max().item() <= FOCK_TOL
    finally:
        eng.set_memory_limit(0)
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_shards_sum_to_the_whole_build():
    import torch
    f = _entry()
    eng, D, J_ref, K_ref = _setup(seed=22)
    Js, Ks = torch.zeros_like(D), torch.zeros_like(D)
    for r in range(2):
        eng.set_shard(r, 2)
        J, K = _noalloc(f, eng, D)
        assert torch.abs(J).max().item() > 0
        assert torch.abs(J - J_ref).max().item() > FOCK_TOL   # one slice is not the whole build
        Js += J
        Ks += K
    eng.set_shard(0, 1)
    assert torch.abs(Js - J_ref).max().item() <= FOCK_TOL
    assert torch.abs(Ks - K_ref).max().item() <= FOCK_TOL


def test_noalloc_is_fp64_under_a_mixed_precision_bound():
    import torch
    f = _entry()
    eng, D, J_ref, K_ref = _setup(seed=23)
    eng.set_fp32_bound(1e300)   # qcg_fock_jk_device would now evaluate every quartet in FP32
    try:
        J, K = _noalloc(f, eng, D)
    finally:
        eng.set_fp32_bound(0.0)
    assert torch.abs(J - J_ref).max().item() <= FOCK_TOL
    assert torch.abs(K - K_ref).max().item() <= FOCK_TOL


def test_noalloc_rejects_bases_above_the_limit():
    import torch
    f = _entry()
    mol = W.water_cluster(nx=3, ny=3, nz=1, seed=W.SEED0 + 3200)   # 9 waters, 513 functions
    eng = api.Engine(B.even_tempered(mol))
    assert eng.nbf > 512
    D = torch.zeros((eng.nbf, eng.nbf), device="cuda", dtype=torch.float64)
    rc = f(eng._h, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(D.data_ptr()))
    assert rc == api.QCG_ERR_ARG
    assert "at most 512" in api.lib().qcg_last_error(eng._h).decode()
