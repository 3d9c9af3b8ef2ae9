"""Repeated J/K builds with the same arguments are captured as a CUDA graph and replayed: the results
must equal kernel-by-kernel builds, including after the density changes and after re-screening."""
import os
import subprocess
import sys

import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W
from tests.conftest import REPO

pytestmark = pytest.mark.gpu


def _density(n, seed):
    Q, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(n, 5)))
    return 2 * Q @ Q.T


def test_replayed_builds_follow_the_density():
    import torch
    sh = B.even_tempered(W.water())
    eng = api.Engine(sh)
    eng.set_graphs(True)
    eng.schwarz(1e-10)
    n = eng.nbf
    J, K = torch.empty((n, n), dtype=torch.float64, device="cuda"), torch.empty((n, n), dtype=torch.float64, device="cuda")
    D = torch.empty((n, n), dtype=torch.float64, device="cuda")
    for it in range(5):   # builds 1 eager, 2 captured, 3-5 replayed
        Dh = _density(n, it)
        D.copy_(torch.from_numpy(Dh))
        eng.fock_jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr())
        torch.cuda.synchronize()
        Jr, Kr, _ = api.Engine(sh).fock_jk(Dh)
        assert np.abs(J.cpu().numpy() - Jr).max() <= 1e-10 and np.abs(K.cpu().numpy() - Kr).max() <= 1e-10, it
    eng.schwarz(1e-8)   # new screening: the cached graph is dropped
    Dh = _density(n, 9)
    D.copy_(torch.from_numpy(Dh))
    for _ in range(3):
        eng.fock_jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr())
    torch.cuda.synchronize()
    e2 = api.Engine(sh)
    e2.schwarz(1e-8)
    Jr, Kr, _ = e2.fock_jk(Dh)
    assert np.abs(J.cpu().numpy() - Jr).max() <= 1e-10


def test_scf_with_and_without_graphs_agree():
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from qchem_b200 import api, basis as B, workloads as W\n"
            "m = W.water(); r = api.Engine(B.even_tempered(m)).rhf(m, incremental=True)\n"
            "print(repr(r['energy']), r['iterations'])\n") % REPO
    out = {}
    for flag in ("0", "1"):
        env = dict(os.environ, QCG_GRAPHS=flag)
        p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        e, its = p.stdout.split()
        out[flag] = (float(e), int(its))
    assert abs(out["0"][0] - out["1"][0]) <= 1e-9 and abs(out["0"][1] - out["1"][1]) <= 1
