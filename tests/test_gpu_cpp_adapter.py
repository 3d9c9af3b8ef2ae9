"""The C++ adapter include/qchem_b200.hpp on a GPU: a small C++ driver, compiled against the header and the
library, builds J and K of the config-1 water through every face qchem calls -- MakeAOFock (whole-system
face), AccumulateDirect / AccumulateExchange and the irrep-pair forms AccumulateDirectBoth /
AccumulateExchangeBoth (Orbital_HF_IBS face), AddAODensity / SliceAOFock -- and the results are checked
against the CPU oracle at the Fock tolerance, 1e-10.  A partner basis other than the engine is rejected."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from qchem_b200 import api, basis as B, workloads as W
from tests.conftest import REPO

pytestmark = pytest.mark.gpu

FOCK_TOL = 1e-10

DRIVER = r"""
#include <cstdio>
#include <fstream>
#include <vector>
#include "qchem_b200.hpp"
// input: nshell, then per shell L, centre, nprim, exponents, coefficients; n; D1 and D2 (n*n each).
// output (binary): J[D1], K[D1], S_J = J[D1] + J[D2] by AccumulateDirect, S_K likewise, the Both forms'
// Ji = J[D2], Jj = J[D1], Ki = K[D2], Kj = K[D1], and F = AddAODensity / SliceAOFock round trip
int main(int argc, char** argv)
{
    std::ifstream in(argv[1]);
    int ns; in >> ns;
    std::vector<qcg::ShellSpec> sh(ns);
    for (auto& s : sh)
    {
        int np; in >> s.L >> s.centre[0] >> s.centre[1] >> s.centre[2] >> np;
        s.exps.resize(np); s.coefs.resize(np);
        for (auto& x : s.exps) in >> x;
        for (auto& x : s.coefs) in >> x;
    }
    int n; in >> n;
    std::vector<double> D1(n * n), D2(n * n);
    for (auto& x : D1) in >> x;
    for (auto& x : D2) in >> x;
    qcg::FockEngine e(sh);
    if ((int)e.AODimension() != n) return 3;
    std::vector<double> J(n * n), K(n * n), SJ(n * n, 0.0), SK(n * n, 0.0), Ji(n * n, 0.0), Jj(n * n, 0.0),
        Ki(n * n, 0.0), Kj(n * n, 0.0), Dao(n * n, 0.0), F(n * n, 0.0);
    e.AddAODensity(Dao.data(), D1.data());
    e.MakeAOFock(Dao.data(), false, J.data());
    e.MakeAOFock(Dao.data(), true, K.data());
    e.SliceAOFock(F.data(), J.data());
    e.AccumulateDirect(SJ.data(), D1.data(), &e);
    e.AccumulateExchange(SK.data(), D1.data(), &e);
    e.AccumulateDirect(SJ.data(), D2.data());
    e.AccumulateExchange(SK.data(), D2.data());
    e.AccumulateDirectBoth(Ji.data(), Jj.data(), D1.data(), D2.data(), &e);
    e.AccumulateExchangeBoth(Ki.data(), Kj.data(), D1.data(), D2.data(), nullptr);
    int rejected = 0;
    qcg::FockEngine other(sh);
    try { e.AccumulateDirect(SJ.data(), D1.data(), &other); }
    catch (const qcg::Error& err) { rejected = err.code == QCG_ERR_ARG; }
    if (!rejected) return 4;
    std::FILE* f = std::fopen(argv[2], "wb");
    for (auto* v : {&J, &K, &SJ, &SK, &Ji, &Jj, &Ki, &Kj, &F}) std::fwrite(v->data(), sizeof(double), v->size(), f);
    std::fclose(f);
    return 0;
}
"""


def test_cpp_adapter_faces_match_oracle(tmp_path, oracle_mod):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    mol = W.water()
    sh = B.even_tempered(mol)
    ob = oracle_mod.OracleBasis(sh)
    n = ob.nbf
    D1 = ob.rhf(mol)["D"]
    D2 = W.cluster_density(n, nocc=5, seed=W.SEED0 + 3500)
    lines = [str(len(sh))]
    for s in sh:
        lines.append(" ".join([str(s.L)] + [repr(float(c)) for c in s.centre] + [str(len(s.exps))] +
                              [repr(float(x)) for x in s.exps] + [repr(float(x)) for x in s.coefs]))
    lines.append(str(n))
    lines.append(" ".join(repr(float(x)) for x in D1.ravel()))
    lines.append(" ".join(repr(float(x)) for x in D2.ravel()))
    inp = tmp_path / "in.txt"
    inp.write_text("\n".join(lines) + "\n")
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    libdir = os.path.dirname(api.library_path())
    exe = tmp_path / "driver"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), str(src), "-L", libdir,
                    "-lqchem_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(inp), str(out)])
    assert r.returncode == 0
    J, K, SJ, SK, Ji, Jj, Ki, Kj, F = np.fromfile(out, dtype=np.float64).reshape(9, n, n)
    J1, K1, _ = ob.jk_direct(D1)
    J2, K2, _ = ob.jk_direct(D2)
    for got, ref in ((J, J1), (K, K1), (SJ, J1 + J2), (SK, K1 + K2), (Ji, J2), (Jj, J1), (Ki, K2), (Kj, K1),
                     (F, J1)):
        assert np.abs(got - ref).max() <= FOCK_TOL


SALC_DRIVER = r"""
#include <cstdio>
#include <fstream>
#include <memory>
#include <vector>
#include "qchem_b200.hpp"
// input: the shells as above; n; the AO density D (n*n); nblock; per block m and O (n*m, row-major).
// output (binary): per block, J and K (m*m each) by the pair route: sum over every partner block h of
// AccumulateDirect / AccumulateExchange with D_h = Transform(D) in h's block
int main(int argc, char** argv)
{
    std::ifstream in(argv[1]);
    int ns; in >> ns;
    std::vector<qcg::ShellSpec> sh(ns);
    for (auto& s : sh)
    {
        int np; in >> s.L >> s.centre[0] >> s.centre[1] >> s.centre[2] >> np;
        s.exps.resize(np); s.coefs.resize(np);
        for (auto& x : s.exps) in >> x;
        for (auto& x : s.coefs) in >> x;
    }
    int n; in >> n;
    std::vector<double> D(n * n);
    for (auto& x : D) in >> x;
    int nb; in >> nb;
    qcg::FockEngine e(sh);
    std::vector<std::unique_ptr<qcg::SalcBlock>> blk;
    for (int b = 0; b < nb; ++b)
    {
        int m; in >> m;
        std::vector<double> O((size_t)n * m);
        for (auto& x : O) in >> x;
        blk.emplace_back(new qcg::SalcBlock(e, O, m));
    }
    std::vector<std::vector<double>> Db(nb);
    for (int b = 0; b < nb; ++b)
    {
        const size_t m = blk[b]->Dimension();
        Db[b].resize(m * m);
        blk[b]->Transform(D.data(), Db[b].data());
    }
    std::FILE* f = std::fopen(argv[2], "wb");
    for (int b = 0; b < nb; ++b)
    {
        const size_t m = blk[b]->Dimension();
        std::vector<double> J(m * m, 0.0), K(m * m, 0.0);
        for (int h = 0; h < nb; ++h)
        {
            blk[b]->AccumulateDirect(J.data(), Db[h].data(), blk[h].get());
            blk[b]->AccumulateExchange(K.data(), Db[h].data(), blk[h].get());
        }
        std::fwrite(J.data(), sizeof(double), J.size(), f);
        std::fwrite(K.data(), sizeof(double), K.size(), f);
    }
    std::fclose(f);
    return 0;
}
"""


def test_cpp_salc_blocks_match_oracle(tmp_path, oracle_mod):
    """The adapter's SalcBlock (qchem's SymmetryAdapted_IBS faces) on water's four C2v irrep blocks: each
    block's J and K by the pair route equal the oracle's AO J and K sliced into the block."""
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    from tests.test_gpu_salc import salc_blocks
    mol = W.water()
    sh = B.even_tempered(mol)
    ob = oracle_mod.OracleBasis(sh)
    n = ob.nbf
    D = ob.rhf(mol)["D"]
    O = list(salc_blocks(mol, sh).values())
    lines = [str(len(sh))]
    for s in sh:
        lines.append(" ".join([str(s.L)] + [repr(float(c)) for c in s.centre] + [str(len(s.exps))] +
                              [repr(float(x)) for x in s.exps] + [repr(float(x)) for x in s.coefs]))
    lines.append(str(n))
    lines.append(" ".join(repr(float(x)) for x in D.ravel()))
    lines.append(str(len(O)))
    for Ob in O:
        lines.append(str(Ob.shape[1]))
        lines.append(" ".join(repr(float(x)) for x in Ob.ravel()))
    inp = tmp_path / "in.txt"
    inp.write_text("\n".join(lines) + "\n")
    src = tmp_path / "salc.cpp"
    src.write_text(SALC_DRIVER)
    libdir = os.path.dirname(api.library_path())
    exe = tmp_path / "salc"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), str(src), "-L", libdir,
                    "-lqchem_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = tmp_path / "out.bin"
    assert subprocess.run([str(exe), str(inp), str(out)]).returncode == 0
    raw = np.fromfile(out, dtype=np.float64)
    Jo, Ko, _ = ob.jk_direct(D)
    pos = 0
    for Ob in O:
        m = Ob.shape[1]
        J = raw[pos:pos + m * m].reshape(m, m)
        K = raw[pos + m * m:pos + 2 * m * m].reshape(m, m)
        pos += 2 * m * m
        assert np.abs(J - Ob.T @ Jo @ Ob).max() <= FOCK_TOL
        assert np.abs(K - Ob.T @ Ko @ Ob).max() <= FOCK_TOL
    assert pos == raw.size
