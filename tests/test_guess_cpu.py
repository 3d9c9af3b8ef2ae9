"""The learned-guess pieces that need no GPU: the MLP oracle (pinned by finite differences and by torch's
own BF16 rounding), the atom-pair block layout, and the conformer generator."""
import numpy as np
import pytest

from oracle import mlp_ref
from qchem_b200 import basis as B, guess as G, workloads as W


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(0).normal(size=4096).astype(np.float32) * np.float32(100.0)
    x[:4] = [1.0, 1.00390625, 1.01171875, -3.3e-3]      # exact, tie to even (down), tie to even (up), small
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(mlp_ref.bf16(x), ref)


def test_oracle_gradient_matches_finite_differences():
    widths = [5, 7, 6, 4]
    rng = np.random.default_rng(1)
    p = rng.normal(size=mlp_ref.nparams(widths)) * 0.5
    x = rng.normal(size=(9, 5))
    t = rng.normal(size=(9, 4))
    mask = (rng.random(size=(9, 4)) > 0.3).astype(float)
    loss, g = mlp_ref.loss_grad(p, widths, x, t, mask, round_bf16=False, dtype=np.float64)
    h = 1e-6
    fd = np.zeros_like(p)
    for k in range(p.size):
        e = np.zeros_like(p)
        e[k] = h
        lp, _ = mlp_ref.loss_grad(p + e, widths, x, t, mask, round_bf16=False, dtype=np.float64)
        lm, _ = mlp_ref.loss_grad(p - e, widths, x, t, mask, round_bf16=False, dtype=np.float64)
        fd[k] = (lp - lm) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-5, atol=1e-8)


def test_pair_layout_round_trip():
    mol = W.water()
    sh = B.even_tempered(mol)
    lay = G.PairLayout.of(mol, sh)
    assert lay.atom_nf == [35, 11, 11] and lay.atom_f0 == [0, 35, 46]
    assert len(lay.pairs) == 6 and lay.nout == 35 * 35
    A = np.random.default_rng(2).normal(size=(57, 57))
    D = A + A.T
    np.testing.assert_array_equal(lay.assemble(lay.blocks(D), 57), D)
    m = lay.mask()
    assert m.sum() == 35 * 35 + 2 * 35 * 11 + 2 * 11 * 11 + 11 * 11


def test_features_and_conformers():
    mol = W.water()
    confs = G.conformers(mol, 5, jitter=0.15, seed=3)
    assert len(confs) == 5
    for c in confs:
        assert np.abs(c.R - mol.R).max() <= 0.15
    np.testing.assert_array_equal(G.conformers(mol, 5, seed=3)[2].R, confs[2].R)
    lay = G.PairLayout.of(mol, B.even_tempered(mol))
    f = lay.features(confs[0], mol)
    assert f.shape == (6, 8 + 3 + 3 + 6 + 9)
    assert np.all(np.isfinite(f))
