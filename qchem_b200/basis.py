"""Molecular Cartesian Gaussian basis sets: shells, even-tempered construction and the Gaussian94 reader.

Shell layout follows qchem's PG_Cart basis (src/BasisSet/Molecule/PG_Cart/Imp/IrrepBasisSet.C):
  * functions are ordered shell by shell; within a shell the Cartesian components are
    for m=0..L, l=0..L-m: (L-m-l, l, m)  -> d = xx, xy, yy, xz, yz, zz   (IrrepBasisSet.C:36-54);
  * contraction coefficients are the raw file coefficients; the library folds in each primitive's
    (L,0,0) normalisation (Imp/GaussianRF.C:566-577) and renormalises every Cartesian component to unit
    self-overlap (Imp/PGData.C:17-33).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

# element symbol <-> nuclear charge for the elements the workloads use
Z_OF = {"H": 1, "HE": 2, "C": 6, "N": 7, "O": 8}
SYM_OF = {v: k for k, v in Z_OF.items()}


@dataclasses.dataclass
class Shell:
    L: int
    centre: Tuple[float, float, float]
    exps: List[float]
    coefs: List[float]
    atom: int = -1

    @property
    def nfunc(self) -> int:
        return (self.L + 1) * (self.L + 2) // 2

    @property
    def nprim(self) -> int:
        return len(self.exps)


@dataclasses.dataclass
class Molecule:
    Z: List[int]
    R: np.ndarray          # (natom, 3) bohr

    @property
    def nelec(self) -> int:
        return int(sum(self.Z))

    def nuclear_repulsion(self) -> float:
        e = 0.0
        for i in range(len(self.Z)):
            for j in range(i):
                e += self.Z[i] * self.Z[j] / float(np.linalg.norm(self.R[i] - self.R[j]))
        return e


def components(L: int) -> List[Tuple[int, int, int]]:
    """Cartesian components of one shell in PG order (IrrepBasisSet.C:36-54)."""
    return [(L - m - l, l, m) for m in range(L + 1) for l in range(L - m + 1)]


def nbf(shells: Sequence[Shell]) -> int:
    return sum(s.nfunc for s in shells)


# ------------------------------------------------------------------------------------------------
# Even-tempered uncontracted basis: alpha_k = alpha0 * beta^k, k = 0..n_L-1, one primitive per shell.
# Shells are emitted atom by atom, L ascending, exponents ascending -- the order of qchem's
# IrrepBasisSet(const rvec_t& es, size_t LMax, const Structure*) constructor (IrrepBasisSet.C:123-147),
# with per-element shell counts.
# ------------------------------------------------------------------------------------------------
EVEN_TEMPERED_COUNTS: Dict[int, Dict[int, int]] = {
    8: {0: 8, 1: 5, 2: 2},     # O: 8s 5p 2d
    7: {0: 8, 1: 5, 2: 2},     # N: same shell set as O
    6: {0: 8, 1: 5, 2: 2},     # C: same shell set as O
    1: {0: 5, 1: 2},           # H: 5s 2p
}


def even_tempered(mol: Molecule, alpha0: float = 0.1, beta: float = 2.5,
                  counts: Dict[int, Dict[int, int]] = EVEN_TEMPERED_COUNTS) -> List[Shell]:
    shells: List[Shell] = []
    for ia, (z, r) in enumerate(zip(mol.Z, mol.R)):
        for L, n in sorted(counts[z].items()):
            for k in range(n):
                shells.append(Shell(L, tuple(float(x) for x in r), [alpha0 * beta ** k], [1.0], ia))
    return shells


# ------------------------------------------------------------------------------------------------
# Gaussian94 (.bsd) reader with the semantics of qchem's Gaussian94Reader + PG_Cart IrrepBasisSet
# (src/BasisSet/Molecule/Readers/Imp/Gaussian94.C:126-179, PG_Cart/Imp/IrrepBasisSet.C:60-121):
#  * one radial per shell line; its L list is the letters on the line (e.g. "SP"), its max L sets the
#    primitive-norm folding of contracted coefficients;
#  * single-primitive shells keep coefficient 1.0 (GaussianRF(exp, R, L) constructor);
#  * radials equal within 0.01 bohr / 0.1% exponent / identical folded coefficients are merged with the
#    reference's merge rule (IrrepBasisSet.C:75-94, reproduced as is, including the inverted L test).
# ------------------------------------------------------------------------------------------------
_LETTER = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4}


def _dfact(i: int) -> float:
    r = 1.0
    while i > 1:
        r *= i
        i -= 2
    return r


def prim_norm(alpha: float, L: int) -> float:
    """GetNormalization(Polarization(L,0,0)) of one primitive (Imp/GaussianRF.C:512-521)."""
    s = (math.pi / (2 * alpha)) ** 1.5
    t = (4 * alpha) ** L
    return math.sqrt(t / (s * _dfact(2 * L - 1)))


def parse_gaussian94(text: str) -> Dict[str, List[Tuple[List[int], List[float], List[float]]]]:
    """element symbol -> list of (Ls, exponents, coefficients-of-first-L) entries."""
    out: Dict[str, list] = {}
    lines = text.splitlines()
    i = 0
    while i < len(lines) and lines[i].strip() != "!":
        i += 1
    i += 2   # the "!" line and the title line after it (Gaussian94.C TopOfFile)
    cur = None
    while i < len(lines):
        ln = lines[i].strip()
        i += 1
        if not ln:
            continue
        tok = ln.split()
        if tok[0] == "****":
            cur = None
            continue
        if cur is None:
            if len(tok) != 2 or not tok[1].lstrip("-").isdigit():
                break   # trailing prose after the last element block
            cur = tok[0].upper()
            out[cur] = []
            continue
        Ls = [_LETTER[c] for c in tok[0]]
        ncont = int(tok[1])
        exps, coefs = [], []
        for _ in range(ncont):
            vals = lines[i].split()
            i += 1
            exps.append(float(vals[0].replace("D", "E")))
            coefs.append(float(vals[1].replace("D", "E")))
        out[cur].append((Ls, exps, coefs))
    return out


def read_gaussian94(text: str, mol: Molecule) -> List[Shell]:
    data = parse_gaussian94(text)
    radials: List[Tuple[Tuple[float, float, float], int, List[float], List[float], List[float]]] = []
    Ls_all: List[List[int]] = []
    for ia, (z, r) in enumerate(zip(mol.Z, mol.R)):
        centre = tuple(float(x) for x in r)
        for Ls, exps, coefs in data[SYM_OF[z]]:
            maxL = max(Ls)
            if len(exps) == 1:
                folded = [1.0]
            else:
                folded = [c * prim_norm(a, maxL) for a, c in zip(exps, coefs)]
            dup = False
            for k, (c2, L2, e2, f2, raw2) in enumerate(radials):
                same = (math.dist(c2, centre) < 0.01 and len(e2) == len(exps)
                        and all(abs((x - y) / (x + y) * 2.0) < 0.001 for x, y in zip(e2, exps))
                        and all(x == y for x, y in zip(f2, folded)))
                if same:
                    dup = True
                    use_new = maxL > max(Ls_all[k])
                    for l in list(Ls):
                        if l in Ls_all[k]:       # reference behaviour (IrrepBasisSet.C:80-82)
                            Ls_all[k].append(l)
                    if use_new:
                        radials[k] = (centre, maxL, exps, folded, coefs)
                    break
            if not dup:
                radials.append((centre, maxL, exps, folded, coefs))
                Ls_all.append(list(Ls))
    shells: List[Shell] = []
    for (centre, maxL, exps, folded, raw), Ls in zip(radials, Ls_all):
        atom = next(i for i, r in enumerate(mol.R) if math.dist(tuple(r), centre) < 1e-12)
        for L in Ls:
            # raw coefficients re-expressed so that the library's own (L,0,0) folding reproduces the
            # radial's (maxL,0,0) folding
            if len(exps) == 1:
                c = [1.0]
            else:
                c = [f / prim_norm(a, L) for a, f in zip(exps, folded)]
            shells.append(Shell(L, centre, list(exps), c, atom))
    return shells


# ------------------------------------------------------------------------------------------------
# Flattening for the C ABI
# ------------------------------------------------------------------------------------------------
def flatten(shells: Sequence[Shell]):
    """-> (L[int32], nprim[int32], centres[f64, 3*ns], exps[f64], coefs[f64])"""
    L = np.array([s.L for s in shells], dtype=np.int32)
    npr = np.array([s.nprim for s in shells], dtype=np.int32)
    cen = np.array([c for s in shells for c in s.centre], dtype=np.float64)
    ex = np.array([e for s in shells for e in s.exps], dtype=np.float64)
    co = np.array([c for s in shells for c in s.coefs], dtype=np.float64)
    return L, npr, cen, ex, co
