"""Learned initial density for the RHF: a network trained on converged densities that the plain GPU SCF
itself produces, predicting density-matrix blocks from atom-pair geometry features.

One model serves the conformers of one molecule (same atoms, same order, geometry varying):
  rows      one per atom pair (A <= B) of a conformer;
  features  element one-hots of A and B, A == B, R_AB, exp(-R_AB / 2), the displacement R_B - R_A, the
            pair's slot one-hot, and the conformer's displacement from the template geometry (all atoms);
            standardised with training-set statistics;
  outputs   the (n_A x n_B) density block D[A functions, B functions], zero-padded to the largest block
            and standardised per slot and entry with training-set statistics (so the network predicts the
            geometry-dependent part around the mean block);
  network   api.Mlp (4 linear layers, width 256, SiLU), BF16 operands, FP32 accumulation, Adam, all on the
            GPU through the library's own kernels;
  density   the predicted blocks assembled into a symmetric nbf x nbf matrix, handed to Engine.rhf(guess=)
            in place of the core-Hamiltonian guess (src/SCFIterator/Imp/Seed.C:70-80 is the reference's
            only guess).  The SCF converges to the same energy either way; the guess changes how many
            iterations it takes.
"""
from __future__ import annotations

import dataclasses
import time
from typing import List, Optional, Sequence

import numpy as np

from . import api, basis as _basis

ELEMENTS = (1, 6, 7, 8)


def conformers(template: _basis.Molecule, n: int, jitter: float = 0.15, seed: int = 0) -> List[_basis.Molecule]:
    """n conformers of `template`: every Cartesian coordinate displaced by U[-jitter, jitter] bohr."""
    rng = np.random.default_rng(seed)
    R0 = np.asarray(template.R, dtype=float)
    return [_basis.Molecule(list(template.Z), R0 + rng.uniform(-jitter, jitter, size=R0.shape)) for _ in range(n)]


@dataclasses.dataclass
class PairLayout:
    """Atom-pair slots of one molecule and where their density blocks sit in the AO matrix."""
    Z: List[int]
    atom_f0: List[int]        # first basis function of each atom
    atom_nf: List[int]        # basis functions on each atom
    pairs: List[tuple]        # (A, B), A <= B
    bmax_a: int
    bmax_b: int

    @classmethod
    def of(cls, mol: _basis.Molecule, shells: Sequence[_basis.Shell]) -> "PairLayout":
        nat = len(mol.Z)
        f0, nf, off = [0] * nat, [0] * nat, 0
        seen = [False] * nat
        for s in shells:
            if not seen[s.atom]:
                f0[s.atom] = off
                seen[s.atom] = True
            nf[s.atom] += s.nfunc
            off += s.nfunc
        pairs = [(a, b) for a in range(nat) for b in range(a, nat)]
        return cls(list(mol.Z), f0, nf, pairs, max(nf), max(nf))

    @property
    def nout(self) -> int:
        return self.bmax_a * self.bmax_b

    def mask(self) -> np.ndarray:
        m = np.zeros((len(self.pairs), self.bmax_a, self.bmax_b), dtype=np.float32)
        for p, (a, b) in enumerate(self.pairs):
            m[p, :self.atom_nf[a], :self.atom_nf[b]] = 1.0
        return m.reshape(len(self.pairs), -1)

    def blocks(self, D: np.ndarray) -> np.ndarray:
        """(npair, nout) padded blocks of a density matrix."""
        out = np.zeros((len(self.pairs), self.bmax_a, self.bmax_b), dtype=np.float64)
        for p, (a, b) in enumerate(self.pairs):
            fa, na, fb, nb = self.atom_f0[a], self.atom_nf[a], self.atom_f0[b], self.atom_nf[b]
            out[p, :na, :nb] = D[fa:fa + na, fb:fb + nb]
        return out.reshape(len(self.pairs), -1)

    def assemble(self, blk: np.ndarray, nbf: int) -> np.ndarray:
        """Symmetric density from (npair, nout) blocks (diagonal blocks symmetrised)."""
        blk = np.asarray(blk, dtype=np.float64).reshape(len(self.pairs), self.bmax_a, self.bmax_b)
        D = np.zeros((nbf, nbf))
        for p, (a, b) in enumerate(self.pairs):
            fa, na, fb, nb = self.atom_f0[a], self.atom_nf[a], self.atom_f0[b], self.atom_nf[b]
            x = blk[p, :na, :nb]
            if a == b:
                D[fa:fa + na, fa:fa + na] = 0.5 * (x + x.T)
            else:
                D[fa:fa + na, fb:fb + nb] = x
                D[fb:fb + nb, fa:fa + na] = x.T
        return D

    def features(self, mol: _basis.Molecule, template: _basis.Molecule) -> np.ndarray:
        """One row per atom pair: element one-hots of both atoms, [a == b], R_AB, exp(-R_AB/2), R_B - R_A,
        the pair slot (one-hot) and the conformer's displacement from the template (all coordinates)."""
        R = np.asarray(mol.R, dtype=float)
        disp = (R - np.asarray(template.R, dtype=float)).ravel()
        a = np.array([p[0] for p in self.pairs])
        b = np.array([p[1] for p in self.pairs])
        Z = np.asarray(self.Z)
        el = np.asarray(ELEMENTS)
        d = R[b] - R[a]
        r = np.sqrt((d * d).sum(axis=1))
        P = len(self.pairs)
        return np.concatenate([(Z[a][:, None] == el[None, :]).astype(float), (Z[b][:, None] == el[None, :]).astype(float),
                               (a == b).astype(float)[:, None], r[:, None], np.exp(-0.5 * r)[:, None], d, np.eye(P),
                               np.broadcast_to(disp, (P, disp.size))], axis=1)


class LearnedGuess:
    """Train on (conformer, converged density) pairs; predict initial densities for new conformers."""

    def __init__(self, template: _basis.Molecule, width: int = 256, layers: int = 4, seed: int = 0,
                 shells_of=_basis.even_tempered):
        self.template = template
        self.shells_of = shells_of
        sh = shells_of(template)
        self.nbf = _basis.nbf(sh)
        self.layout = PairLayout.of(template, sh)
        self.nin = len(self.layout.features(template, template)[0])
        self.widths = [self.nin] + [width] * (layers - 1) + [self.layout.nout]
        self.net = api.Mlp(self.widths, seed=seed)
        self.x_mu = self.x_sd = self.y_mu = self.y_sd = None
        self.history = []

    # -- data ---------------------------------------------------------------------------------
    def _x(self, mols):
        return np.concatenate([self.layout.features(m, self.template) for m in mols])

    def _xn(self, mols):
        return ((self._x(mols) - self.x_mu) / self.x_sd).astype(np.float32)

    def fit(self, mols: Sequence[_basis.Molecule], densities: Sequence[np.ndarray], steps: int = 3000,
            batch_molecules: int = 128, lr: float = 2e-3, seed: int = 0, device: str = "cuda",
            y_floor: float = 1e-8) -> dict:
        """y_floor: the smallest spread an output entry is standardised by; entries that vary less are not
        amplified into the loss (1e-8: every entry counts)"""
        import torch
        P = len(self.layout.pairs)
        X = self._x(mols)
        self.x_mu = X.mean(axis=0)
        self.x_sd = X.std(axis=0) + 1e-6
        Y = np.stack([self.layout.blocks(D) for D in densities])          # (nmol, P, nout)
        self.y_mu = Y.mean(axis=0)
        self.y_sd = np.maximum(Y.std(axis=0), y_floor) + 1e-8
        mask = self.layout.mask()
        Yn = ((Y - self.y_mu) / self.y_sd * mask).astype(np.float32).reshape(-1, self.layout.nout)
        Xn = ((X - self.x_mu) / self.x_sd).astype(np.float32)
        dev = torch.device(device)
        dX = torch.from_numpy(Xn).to(dev)
        dY = torch.from_numpy(Yn).to(dev)
        dM = torch.from_numpy(np.tile(mask, (len(mols), 1))).to(dev)
        self.net.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        rng = np.random.default_rng(seed)
        nmol = len(mols)
        bm = min(batch_molecules, nmol)
        t0 = time.perf_counter()
        losses = []
        order = rng.permutation(nmol)
        pos = 0
        for step in range(steps):
            if pos + bm > nmol:
                order, pos = rng.permutation(nmol), 0
            mol_idx = torch.from_numpy(order[pos:pos + bm]).to(dev)
            pos += bm
            rows = (mol_idx[:, None] * P + torch.arange(P, device=dev)[None, :]).reshape(-1)
            xb, yb, mb = dX[rows].contiguous(), dY[rows].contiguous(), dM[rows].contiguous()
            loss = self.net.loss_grad(len(rows), xb.data_ptr(), yb.data_ptr(), mb.data_ptr())
            # cosine decay of the step size
            self.net.adam(lr=float(lr * 0.5 * (1 + np.cos(np.pi * step / steps))), weight_decay=1e-5)
            losses.append(loss)
        torch.cuda.synchronize(dev)
        info = {"steps": steps, "train_s": time.perf_counter() - t0, "loss_first": losses[0],
                "loss_last": float(np.mean(losses[-20:])), "rows": int(len(Xn)), "params": self.net.nparams}
        self.history = losses
        return info

    # -- inference ------------------------------------------------------------------------------
    def predict_blocks(self, mols: Sequence[_basis.Molecule], device: str = "cuda") -> np.ndarray:
        import torch
        P = len(self.layout.pairs)
        xn = self._xn(mols)
        rows = xn.shape[0]
        # input/output buffers (pinned host and device) and the stream binding are kept between calls: a
        # single-molecule prediction is a handful of small launches, so allocation and pageable copies
        # would cost more than the network
        key = (rows, str(device))
        if getattr(self, "_io_key", None) != key:
            dev = torch.device(device)
            self._io = (torch.empty((rows, xn.shape[1]), dtype=torch.float32).pin_memory(),
                        torch.empty((rows, xn.shape[1]), dtype=torch.float32, device=dev),
                        torch.empty((rows, self.layout.nout), dtype=torch.float32, device=dev),
                        torch.empty((rows, self.layout.nout), dtype=torch.float32).pin_memory(),
                        torch.cuda.current_stream(dev))
            self._io_key = key
            self._mask = self.layout.mask()
        hx, dx, dy, hy, stream = self._io
        self.net.set_stream(stream.cuda_stream)
        hx.numpy()[...] = xn
        dx.copy_(hx, non_blocking=True)
        self.net.forward(rows, dx.data_ptr(), dy.data_ptr())
        hy.copy_(dy, non_blocking=True)
        stream.synchronize()
        yn = hy.numpy().astype(np.float64).reshape(len(mols), P, -1)
        return (yn * self.y_sd + self.y_mu) * self._mask

    def predict(self, mol: _basis.Molecule, device: str = "cuda") -> np.ndarray:
        return self.layout.assemble(self.predict_blocks([mol], device)[0], self.nbf)

    def mean_density(self) -> np.ndarray:
        """The training-set mean density (the network's baseline, no geometry dependence)."""
        return self.layout.assemble(self.y_mu * self.layout.mask(), self.nbf)


def plain_scf_dataset(mols: Sequence[_basis.Molecule], shells_of=_basis.even_tempered, **rhf_kw):
    """Converged densities, energies and iteration counts of the plain FP64 GPU SCF (core guess), for the
    conformers whose SCF converged; `kept` lists their indices (a conformer whose core-guess SCF does not
    converge within the iteration limit gives no training target)."""
    Ds, Es, its, walls, kept = [], [], [], [], []
    for i, m in enumerate(mols):
        r = api.Engine(shells_of(m)).rhf(m, want_density=True, **rhf_kw)
        if not r["converged"]:
            continue
        kept.append(i)
        Ds.append(r["D"])
        Es.append(r["energy"])
        its.append(r["iterations"])
        walls.append(r["wall_s"])
    return Ds, np.array(Es), np.array(its), np.array(walls), kept


def plain_scf_dataset_batched(mols: Sequence[_basis.Molecule], chunk: int = 500, shells_of=_basis.even_tempered,
                              **rhf_kw):
    """plain_scf_dataset through the batched SCF: `chunk` conformers per batch handle, every SCF with the
    plain settings (core guess, the reference's DIIS rules), one J/K build per iteration over the chunk.
    The returned walls are each chunk's wall time per molecule."""
    Ds, Es, its, walls, kept = [], [], [], [], []
    for c0 in range(0, len(mols), chunk):
        part = list(mols[c0:c0 + chunk])
        t0 = time.perf_counter()
        res = api.BatchEngine([shells_of(m) for m in part]).rhf(part, want_density=True, **rhf_kw)
        per = (time.perf_counter() - t0) / len(part)
        for k, r in enumerate(res):
            if not r["converged"]:
                continue
            kept.append(c0 + k)
            Ds.append(r["D"])
            Es.append(r["energy"])
            its.append(r["iterations"])
            walls.append(per)
    return Ds, np.array(Es), np.array(its), np.array(walls), kept


def evaluate(model: Optional[LearnedGuess], mols: Sequence[_basis.Molecule], ref_energies: Sequence[float],
             shells_of=_basis.even_tempered, guess: str = "learned", **rhf_kw) -> dict:
    """SCF on held-out conformers from the learned (or mean, or core) guess: iterations, wall time (guess,
    engine set-up and SCF) and the largest energy difference to the reference energies (entries that are
    None are not compared)."""
    its, walls, dE, conv, energies = [], [], [], [], []
    for m, e_ref in zip(mols, ref_energies):
        g = None
        t0 = time.perf_counter()
        if guess == "learned":
            g = model.predict(m)
        elif guess == "mean":
            g = model.mean_density()
        r = api.Engine(shells_of(m)).rhf(m, guess=g, **rhf_kw)
        walls.append(time.perf_counter() - t0)
        its.append(r["iterations"])
        conv.append(bool(r["converged"]))
        energies.append(r["energy"])
        if e_ref is not None:
            dE.append(abs(r["energy"] - e_ref))
    return {"guess": guess, "iterations_mean": float(np.mean(its)), "iterations": [int(i) for i in its],
            "wall_s_mean": float(np.mean(walls)), "wall_s_median": float(np.median(walls)), "wall_s": walls,
            "energies": energies, "converged": conv,
            "max_abs_dE": float(np.max(dE)) if dE else None, "all_converged": bool(all(conv))}


def evaluate_batched(model: LearnedGuess, mols: Sequence[_basis.Molecule], ref_energies: Sequence[float],
                     **rhf_kw) -> dict:
    """The learned guess with batching: every conformer's guess from one network pass, every SCF in one
    batch handle (one J/K build per iteration over all molecules).  The wall time covers the guesses, the
    handle set-up and the SCF; wall_s_per_molecule is that time divided by the number of molecules (a
    throughput figure, not one molecule's latency)."""
    t0 = time.perf_counter()
    blocks = model.predict_blocks(mols)
    guesses = [model.layout.assemble(b, model.nbf) for b in blocks]
    be = api.BatchEngine([model.shells_of(m) for m in mols])
    res = be.rhf(mols, guesses=guesses, **rhf_kw)
    wall = time.perf_counter() - t0
    dE = [abs(r["energy"] - e) for r, e in zip(res, ref_energies) if e is not None and r["converged"]]
    its = [r["iterations"] for r in res]
    return {"guess": "learned", "molecules": len(mols), "wall_s": wall, "wall_s_per_molecule": wall / len(mols),
            "iterations_mean": float(np.mean(its)), "iterations_max": int(max(its)),
            "all_converged": bool(all(r["converged"] for r in res)),
            "max_abs_dE": float(np.max(dE)) if dE else None}
