"""The learned initial guess on the GPU: the MLP kernels against the numpy oracle (BF16 operands, FP32
accumulation), training, and the guess itself on held-out water conformers, where it must cut the SCF
iteration count against the core-Hamiltonian guess while every SCF ends at the plain FP64 energy within
1e-8 Eh."""
import numpy as np
import pytest
import torch

from oracle import mlp_ref
from qchem_b200 import api, guess as G, workloads as W

pytestmark = pytest.mark.gpu

E_TOL = 1e-8


def _problem(widths, rows, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, widths[0])).astype(np.float32)
    t = rng.normal(size=(rows, widths[-1])).astype(np.float32)
    mask = (rng.random(size=(rows, widths[-1])) > 0.25).astype(np.float32)
    return x, t, mask


def _gemm_case(ta, tb, M, N, K, bias, accumulate, seed):
    """C (+)= op(A) op(B) (+ bias) through the tensor-core product, against float64 products of the same
    BF16-rounded operands."""
    g = torch.Generator().manual_seed(seed)
    A = torch.randn((K, M) if ta else (M, K), generator=g)
    B = torch.randn((N, K) if tb else (K, N), generator=g)
    C0 = torch.randn((M, N), generator=g)
    b = torch.randn(N, generator=g) if bias else None
    dA, dB, dC = A.cuda(), B.cuda(), C0.clone().cuda()
    db = b.cuda() if bias else None
    rc = api.lib().qcg_internal_gemm_bf16(int(ta), int(tb), M, N, K, dA.data_ptr(), A.shape[1], dB.data_ptr(),
                                          B.shape[1], dC.data_ptr(), N, db.data_ptr() if bias else None,
                                          int(accumulate))
    assert rc == 0
    r = lambda x: x.to(torch.bfloat16).to(torch.float64)
    opA = r(A).T if ta else r(A)
    opB = r(B).T if tb else r(B)
    ref = opA @ opB + (b.double() if bias else 0.0) + (C0.double() if accumulate else 0.0)
    scale = (opA.abs() @ opB.abs()).max().item() + 1.0
    return (dC.cpu().double() - ref).abs().max().item() / scale


@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (127, 129, 65), (300, 256, 256), (256, 1225, 256), (256, 256, 9000),
                                   (64, 16, 0)])
def test_tensor_core_product_matches_float64(ta, tb, M, N, K):
    """The MLP's matrix product on the tensor cores (tcgen05.mma, accumulator in tensor memory): every
    operand form, ragged tiles, long K (split over CTAs, atomics), K = 0, with and without bias and
    accumulation.  BF16 products are exact in FP32; only the FP32 summation order differs."""
    for bias, acc in ((False, False), (True, False), (True, True)):
        err = _gemm_case(ta, tb, M, N, K, bias, acc, seed=M * 7 + N * 3 + K + 2 * ta + tb)
        assert err < 2e-6, (bias, acc, err)


def test_mlp_forward_matches_oracle():
    widths = [23, 256, 256, 256, 300]
    net = api.Mlp(widths, seed=5)
    x, _, _ = _problem(widths, 131, 1)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty((131, widths[-1]), device="cuda")
    net.forward(131, dx.data_ptr(), dy.data_ptr())
    torch.cuda.synchronize()
    ref = mlp_ref.forward(net.params(), widths, x)
    # a BF16 operand whose FP32 value differs in the last bits between the two summation orders can round
    # to the neighbouring BF16 value (2^-8 apart); a few such flips in 10^5 operands move outputs ~1e-4
    err = np.abs(dy.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-3, err


def test_mlp_gradient_matches_oracle():
    widths = [23, 64, 80, 48, 70]
    net = api.Mlp(widths, seed=6)
    x, t, mask = _problem(widths, 77, 2)
    d = [torch.from_numpy(a).cuda() for a in (x, t, mask)]
    loss, g = net.loss_grad(77, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), want_grad=True)
    loss_r, g_r = mlp_ref.loss_grad(net.params(), widths, x, t, mask)
    assert abs(loss - loss_r) <= 1e-5 * abs(loss_r)
    rel = np.linalg.norm(g - g_r) / np.linalg.norm(g_r)
    assert rel < 5e-3, rel
    # and against the exact-arithmetic network: BF16 rounding moves the gradient by well under a percent
    _, g_x = mlp_ref.loss_grad(net.params(), widths, x, t, mask, round_bf16=False, dtype=np.float64)
    assert np.linalg.norm(g - g_x) / np.linalg.norm(g_x) < 3e-2


def test_mlp_training_reduces_loss():
    widths = [8, 64, 64, 64, 16]
    rng = np.random.default_rng(3)
    x = rng.normal(size=(512, 8)).astype(np.float32)
    t = np.tanh(x @ rng.normal(size=(8, 16))).astype(np.float32)
    mask = np.ones_like(t)
    d = [torch.from_numpy(a).cuda() for a in (x, t, mask)]
    net = api.Mlp(widths, seed=7)
    first = net.loss_grad(512, *(a.data_ptr() for a in d))
    for _ in range(300):
        net.loss_grad(512, *(a.data_ptr() for a in d))
        net.adam(lr=3e-3)
    last = net.loss_grad(512, *(a.data_ptr() for a in d))
    assert last < 0.05 * first, (first, last)


def test_mlp_rejects_bad_arguments():
    with pytest.raises(api.QcgError):
        api.Mlp([4], seed=0)
    net = api.Mlp([4, 8, 2], seed=0)
    with pytest.raises(api.QcgError):
        net.set_params(np.zeros(3, dtype=np.float32))
    with pytest.raises(api.QcgError):
        net.adam(lr=1e-3, beta1=1.5)


def test_learned_guess_cuts_iterations_on_held_out_water_conformers():
    mol = W.water()
    train = G.conformers(mol, 48, seed=W.SEED0 + 5000)
    test = G.conformers(mol, 6, seed=W.SEED0 + 5001)
    Ds, _, its_train, _, kept = G.plain_scf_dataset(train)
    model = G.LearnedGuess(mol, seed=1)
    info = model.fit([train[i] for i in kept], Ds, steps=600, batch_molecules=16)
    assert info["loss_last"] < 0.2 * info["loss_first"]
    core = G.evaluate(None, test, [0.0] * len(test), guess="core")
    E_ref = [api.Engine(model.shells_of(m)).rhf(m)["energy"] for m in test]
    learned = G.evaluate(model, test, E_ref, guess="learned")
    assert learned["all_converged"]
    assert learned["max_abs_dE"] <= E_TOL
    assert learned["iterations_mean"] < 0.75 * core["iterations_mean"], (learned, core)
