"""Seeded synthetic workloads (all inputs are synthetic; there is no external dataset for this path).

  water()            one water, O at the origin, H at (+-1.43, 1.11, 0) bohr
  water_cluster()    32 waters on a jittered 4x4x2 grid of 5.5 bohr, random rotations about O
  cluster_density()  D = 2 Q Q^T with Q (N x nocc) Euclidean-orthonormal (QR of a Gaussian matrix)
  eri_class_batch()  random shell quartets of one angular class drawn from a seeded shell pool
  random_molecules() H/C/N/O heavy-atom random-walk chains capped with H, even electron count

Seeds follow numpy.random.default_rng(20261203 + config*1000 + index).
"""
from __future__ import annotations

import itertools
import math
from typing import List, Tuple

import numpy as np

from .basis import Molecule, Shell, even_tempered

SEED0 = 20261203

WATER_O = np.array([0.0, 0.0, 0.0])
WATER_H1 = np.array([1.43, 1.11, 0.0])
WATER_H2 = np.array([-1.43, 1.11, 0.0])


def water() -> Molecule:
    return Molecule([8, 1, 1], np.array([WATER_O, WATER_H1, WATER_H2]))


def _random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(nx=4, ny=4, nz=2, spacing=5.5, jitter=0.3, seed=SEED0 + 3000) -> Molecule:
    rng = np.random.default_rng(seed)
    Z, R = [], []
    for i, j, k in itertools.product(range(nx), range(ny), range(nz)):
        c = np.array([i, j, k], float) * spacing + rng.uniform(-jitter, jitter, size=3)
        rot = _random_rotation(rng)
        for z, r in ((8, WATER_O), (1, WATER_H1), (1, WATER_H2)):
            Z.append(z)
            R.append(c + rot @ r)
    return Molecule(Z, np.array(R))


def cluster_density(nbf: int, nocc: int = 160, seed=SEED0 + 3001) -> np.ndarray:
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(nbf, nocc)))
    return 2.0 * Q @ Q.T


# ------------------------------------------------------------------------------------------------
# ERI microbenchmark: 21 canonical classes (la>=lb, lc>=ld, pair(ab) >= pair(cd)), l in {s,p,d}
# ------------------------------------------------------------------------------------------------
PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]


def quartet_classes() -> List[Tuple[int, int, int, int]]:
    out = []
    for X in range(6):
        for Y in range(X + 1):
            la, lb = PAIR_CLASSES[X]
            lc, ld = PAIR_CLASSES[Y]
            out.append((la, lb, lc, ld))
    return out


def shell_pool(npool: int, seed: int, box: float = 12.0) -> List[Shell]:
    """npool random shells per L in {0,1,2}: K uniform {1,2,3}, coefficients U[0.1,1], exponents
    log-uniform in [0.05, 50], centres uniform in a 12-bohr box.  Shell index = L*npool + k."""
    rng = np.random.default_rng(seed)
    shells = []
    for L in range(3):
        for _ in range(npool):
            K = int(rng.integers(1, 4))
            ex = np.exp(rng.uniform(math.log(0.05), math.log(50.0), size=K))
            co = rng.uniform(0.1, 1.0, size=K)
            c = rng.uniform(0.0, box, size=3)
            shells.append(Shell(L, tuple(float(x) for x in c), [float(x) for x in ex], [float(x) for x in co]))
    return shells


def eri_class_batch(cls, nq: int, npool: int, seed: int) -> np.ndarray:
    """nq x 4 int32 shell indices into shell_pool(npool) for angular class cls=(la,lb,lc,ld)."""
    rng = np.random.default_rng(seed)
    q = np.empty((nq, 4), dtype=np.int32)
    for k, L in enumerate(cls):
        q[:, k] = L * npool + rng.integers(0, npool, size=nq)
    return q


# ------------------------------------------------------------------------------------------------
# Batched small molecules: heavy-atom random walk chains, H caps
# ------------------------------------------------------------------------------------------------
def random_molecule(rng, n_atoms_max=24) -> Molecule:
    while True:
        nheavy = int(rng.integers(1, max(2, n_atoms_max // 3) + 1))
        Zh = list(rng.choice([6, 7, 8], size=nheavy))
        pos = [np.zeros(3)]
        for _ in range(nheavy - 1):
            for _try in range(100):
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
                p = pos[-1] + d * rng.uniform(2.4, 2.9)
                if all(np.linalg.norm(p - q) > 2.3 for q in pos):
                    pos.append(p)
                    break
            else:
                break
        Zh = Zh[:len(pos)]
        valence = {6: 4, 7: 3, 8: 2}
        Z = list(Zh)
        R = list(pos)
        for i, (z, p) in enumerate(zip(Zh, pos)):
            nb = (i > 0) + (i < len(pos) - 1)
            for _ in range(max(0, valence[z] - nb)):
                for _try in range(100):
                    d = rng.normal(size=3)
                    d /= np.linalg.norm(d)
                    h = p + 2.0 * d
                    if all(np.linalg.norm(h - q) > 1.5 for q in R):
                        Z.append(1)
                        R.append(h)
                        break
        if sum(Z) % 2 == 1:
            # drop one H so that the electron count is even
            for k in range(len(Z) - 1, -1, -1):
                if Z[k] == 1:
                    del Z[k]
                    del R[k]
                    break
        if 2 <= len(Z) <= n_atoms_max and sum(Z) % 2 == 0:
            return Molecule(Z, np.array(R))


def random_molecules(n=256, seed=SEED0 + 4000, max_atoms=24) -> List[Molecule]:
    rng = np.random.default_rng(seed)
    return [random_molecule(rng, max_atoms) for _ in range(n)]


def basis_for(mol: Molecule) -> List[Shell]:
    return even_tempered(mol)
