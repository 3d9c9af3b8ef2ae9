"""Generate straight-line McMurchie-Davidson code for each of the 21 (s,p,d) quartet classes.

For class (LA LB | LC LD) the generated device function evaluates ONE primitive quartet:
  Boys F_0..F_L -> R^0_{tuv} in place, levels L..0 (registers, or a per-thread slice of shared memory
  when L >= R_SMEM_MIN_L) -> 1-D Hermite E tables of both pairs (registers) -> for every ket component
  (c,d): the ket transform X_{tuv} = sum_{h' in supp(cd)} (-1)^{|h'|} E^{cd}_{h'} R_{tuv+h'} with every
  R value read once per (c,d); then for every bra component (a,b) the factored sum
  sum_t Ex_t sum_u Ey_u sum_v Ez_v X_{tuv} and the sink call.
All indices are literals, so nvcc keeps the tables in registers without any constexpr folding work.
The code is a template on the arithmetic type RT (double, or float for the FP32 form); the primitive-pair
data, the Boys argument and the prefactor lambda are formed in FP64 and rounded to RT once.

Recursions follow qchem: R (Internal/MnD/Imp/RNLM.C:19-68), E (PG_Cart_MnD/Internal/Imp/Hermite2.C:95-139),
Boys (Internal/Boys/Imp/AuxillaryFJ.C:13-48), prefactor (PG_Cart_MnD/Imp/GaussianRF.C:446-483).

Usage: python gen_md.py <outdir>   (writes md_class_<k>.cuh for k = 0..20)
"""
import math
import os
import sys

PAIRS = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
R_SMEM_MIN_L = 6


def classes():
    out = []
    for X in range(6):
        for Y in range(X + 1):
            out.append(PAIRS[X] + PAIRS[Y])
    return out


def comps(L):
    return [(L - m - l, l, m) for m in range(L + 1) for l in range(L - m + 1)]


def hidx(L, t, u, v):
    off = 0
    for tt in range(t):
        off += (L - tt + 1) * (L - tt + 2) // 2
    for uu in range(u):
        off += (L - t - uu + 1)
    return off + v


def nherm(L):
    return (L + 1) * (L + 2) * (L + 3) // 6


def herm_list(L):
    return [(t, u, v) for t in range(L + 1) for u in range(L + 1 - t) for v in range(L + 1 - t - u)]


def inv_sqrt_dfact(k):
    d = 1.0
    for x in range(2 * k - 1, 1, -2):
        d *= x
    return 1.0 / math.sqrt(d)


def comp_norm(c):
    return inv_sqrt_dfact(c[0]) * inv_sqrt_dfact(c[1]) * inv_sqrt_dfact(c[2])


def lit(x):
    return "%.17g" % x


def gen_E(name, LA, LB, PA, PB, a12):
    """1-D E table of one direction as scalars name_i_j_t, in the build order of Hermite2.C."""
    out = [f"const RT {name}_0_0_0 = RT(1);"]

    def g(i, j, t):
        return f"{name}_{i}_{j}_{t}"

    def expr(i0, j0, t, P):
        terms = []
        if t >= 1:
            terms.append(f"{g(i0, j0, t - 1)} * {a12}")
        if t <= i0 + j0:
            terms.append(f"{g(i0, j0, t)} * {P}")
        if t + 1 <= i0 + j0:
            terms.append(f"{g(i0, j0, t + 1)} * RT({t + 1})")
        return " + ".join(terms)

    for i in range(1, LA + 1):
        for t in range(0, i + 1):
            out.append(f"const RT {name}_{i}_0_{t} = {expr(i - 1, 0, t, PA)};")
    for i in range(0, LA + 1):
        for j in range(1, LB + 1):
            for t in range(0, i + j + 1):
                out.append(f"const RT {name}_{i}_{j}_{t} = {expr(i, j - 1, t, PB)};")
    return out


CHUNK_ABOVE = 100          # classes with more outputs than this are split into __noinline__ chunks ...
CHUNK_OUTPUTS = 72         # ... of at most this many outputs (keeps each chunk's live set in registers)


def e_tables(LA, LB, LC, LD):
    out = []
    for dname, la, lb, PA, PB, a12 in (("ebx", LA, LB, "bPAx", "bPBx", "a12b"),
                                       ("eby", LA, LB, "bPAy", "bPBy", "a12b"),
                                       ("ebz", LA, LB, "bPAz", "bPBz", "a12b"),
                                       ("ekx", LC, LD, "kPAx", "kPBx", "a12k"),
                                       ("eky", LC, LD, "kPAy", "kPBy", "a12k"),
                                       ("ekz", LC, LD, "kPAz", "kPBz", "a12k")):
        out.extend(gen_E(dname, la, lb, PA, PB, a12))
    return out


def e_names(prefix, la, lb):
    names = []
    for i in range(la + 1):
        for j in range(lb + 1):
            for t in range(i + j + 1):
                names.append(f"{prefix}_{i}_{j}_{t}")
    return names


def r_prologue(L, rsm, w):
    HL = nherm(L)
    w("    const double p = ab.p, q = cd.p, pq = p + q;")
    w("    const double alpha = p * q / pq;")
    w("    const double Xd = ab.Px - cd.Px, Yd = ab.Py - cd.Py, Zd = ab.Pz - cd.Pz;")
    w(f"    RT F[{L + 1}];")
    w(f"    boys<{L}>(alpha * (Xd * Xd + Yd * Yd + Zd * Zd), bt, F);")
    w("    const RT X = RT(Xd), Y = RT(Yd), Z = RT(Zd);")
    w("    const RT m2a = RT(-2.0 * alpha);")
    w(f"    RT pwn[{L + 1}];")
    w("    pwn[0] = RT(1);")
    for n in range(1, L + 1):
        w(f"    pwn[{n}] = pwn[{n - 1}] * m2a;")
    if rsm:
        w("#define RR(i) rs[(i) * rstride]")
    else:
        w(f"    RT Rr[{HL}];")
        w("#define RR(i) Rr[i]")
    w(f"    RR(0) = pwn[{L}] * F[{L}];")
    for n in range(L - 1, -1, -1):
        for m in range(L - n, 0, -1):
            for t in range(m, -1, -1):
                for u in range(m - t, -1, -1):
                    v = m - t - u
                    if t > 0:
                        e = f"X * RR({hidx(L, t - 1, u, v)})"
                        if t > 1:
                            e += f" + RT({t - 1}) * RR({hidx(L, t - 2, u, v)})"
                    elif u > 0:
                        e = f"Y * RR({hidx(L, 0, u - 1, v)})"
                        if u > 1:
                            e += f" + RT({u - 1}) * RR({hidx(L, 0, u - 2, v)})"
                    else:
                        e = f"Z * RR({hidx(L, 0, 0, v - 1)})"
                        if v > 1:
                            e += f" + RT({v - 1}) * RR({hidx(L, 0, 0, v - 2)})"
                    w(f"    RR({hidx(L, t, u, v)}) = {e};")
        w(f"    RR(0) = pwn[{n}] * F[{n}];")
    w("    const RT lambda = RT(34.986836655249725693 / (p * q * sqrt(pq)) * ab.K * cd.K);")
    w("    const RT a12b = RT(0.5 / ab.p), a12k = RT(0.5 / cd.p);")


def ket_blocks(LA, LB, LC, LD, cds, w):
    L = LA + LB + LC + LD
    LAB = LA + LB
    A, B, C, D = comps(LA), comps(LB), comps(LC), comps(LD)
    HAB = herm_list(LAB)
    NX = len(HAB)
    for (ic, id_) in cds:
        c, d = C[ic], D[id_]
        w(f"    {{ // ket component ({ic},{id_})")
        w(f"    sink.ket_begin({ic}, {id_});")
        supp = [(tp, up, vp) for tp in range(c[0] + d[0] + 1) for up in range(c[1] + d[1] + 1)
                for vp in range(c[2] + d[2] + 1)]
        for (tp, up, vp) in supp:
            sgn = "-" if (tp + up + vp) & 1 else ""
            w(f"    const RT s{tp}{up}{vp} = {sgn}ekx_{c[0]}_{d[0]}_{tp} * eky_{c[1]}_{d[1]}_{up} * "
              f"ekz_{c[2]}_{d[2]}_{vp};")
        w("    RT " + ", ".join(f"x{i} = RT(0)" for i in range(NX)) + ";")
        contrib = {}
        for h in HAB:
            for hp in supp:
                H = hidx(L, h[0] + hp[0], h[1] + hp[1], h[2] + hp[2])
                contrib.setdefault(H, []).append((hidx(LAB, *h), hp))
        for H in sorted(contrib):
            body = " ".join(f"x{xi} = qfma(s{hp[0]}{hp[1]}{hp[2]}, r, x{xi});" for (xi, hp) in contrib[H])
            w(f"    {{ const RT r = RR({H}); {body} }}")
        w(f"    const RT lam_cd = lambda * RT({lit(comp_norm(c) * comp_norm(d))});")
        for ia, a in enumerate(A):
            for ib, b in enumerate(B):
                w("    {")
                w("      RT sx = RT(0);")
                for t in range(a[0] + b[0] + 1):
                    w("      { RT sy = RT(0);")
                    for u in range(a[1] + b[1] + 1):
                        vs = list(range(a[2] + b[2] + 1))
                        zs = f"ebz_{a[2]}_{b[2]}_0 * x{hidx(LAB, t, u, 0)}"
                        for v in vs[1:]:
                            zs = f"qfma(ebz_{a[2]}_{b[2]}_{v}, x{hidx(LAB, t, u, v)}, {zs})"
                        w(f"        sy = qfma(eby_{a[1]}_{b[1]}_{u}, {zs}, sy);")
                    w(f"        sx = qfma(ebx_{a[0]}_{b[0]}_{t}, sy, sx); }}")
                w(f"      sink({ia}, {ib}, {ic}, {id_}, sx * (lam_cd * RT({lit(comp_norm(a) * comp_norm(b))})));")
                w("    }")
        w(f"    sink.ket_end({ic}, {id_});")
        w("    }")


def gen_class(LA, LB, LC, LD, idx):
    L = LA + LB + LC + LD
    A, B, C, D = comps(LA), comps(LB), comps(LC), comps(LD)
    nab, ncd = len(A) * len(B), len(C) * len(D)
    all_cds = [(ic, id_) for ic in range(len(C)) for id_ in range(len(D))]
    chunked = nab * ncd > CHUNK_ABOVE
    # chunk functions read R through the per-thread shared-memory slice, so chunked classes keep R there
    rsm = L >= R_SMEM_MIN_L or chunked
    assert rsm or not chunked
    o = []
    w = o.append
    w(f"// class {idx}: ({'spd'[LA]}{'spd'[LB]}|{'spd'[LC]}{'spd'[LD]}), L = {L}; R table in "
      f"{'a per-thread slice of shared memory' if rsm else 'registers'}"
      f"{'; ket components split into __noinline__ chunks' if chunked else ''}")
    w(f"constexpr bool kRShared{idx} = {'true' if rsm else 'false'};")
    w(f"constexpr bool kChunked{idx} = {'true' if chunked else 'false'};")
    w(f"constexpr int kRSize{idx} = {nherm(L)};")
    chunk_names = []
    if chunked:
        per = max(1, CHUNK_OUTPUTS // nab)
        w(f"constexpr int kNChunk{idx} = {(len(all_cds) + per - 1) // per};")
    else:
        w(f"constexpr int kNChunk{idx} = 1;")
    if chunked:
        per = max(1, CHUNK_OUTPUTS // nab)
        chunks = [all_cds[i:i + per] for i in range(0, len(all_cds), per)]
        for ci, cds in enumerate(chunks):
            fn = f"prim_quartet_{idx}_chunk{ci}"
            chunk_names.append(fn)
            # each chunk rebuilds the 1-D E tables from the pair scalars (cheaper than reloading them)
            w("template <class RT, class Sink>")
            w(f"__device__ __noinline__ void {fn}(const RT* __restrict__ rs, const int rstride,")
            w("    const RT a12b, const RT bPAx, const RT bPAy, const RT bPAz, const RT bPBx,")
            w("    const RT bPBy, const RT bPBz, const RT a12k, const RT kPAx, const RT kPAy,")
            w("    const RT kPAz, const RT kPBx, const RT kPBy, const RT kPBz, const RT lambda,")
            w("    typename SinkArg<Sink>::type sink)")
            w("{")
            for s_ in e_tables(LA, LB, LC, LD):
                w("    " + s_)
            w("#define RR(i) rs[(i) * rstride]")
            ket_blocks(LA, LB, LC, LD, cds, w)
            w("#undef RR")
            w("}")
    # LOCKSTEP: the caller guarantees that every thread of the block executes this call (block-uniform
    # control flow); the barriers then keep the block's warps on the same chunk, so that the instruction
    # working set is one chunk rather than the whole class
    w("template <class RT, class Sink, bool LOCKSTEP = false>")
    w(f"__device__ __forceinline__ void prim_quartet_{idx}(const PrimPairData& ab, const PrimPairData& cd,")
    w("    const double* __restrict__ bt, RT* __restrict__ rs, const int rstride, Sink& sink)")
    w("{")
    w("    (void)rs; (void)rstride;")
    r_prologue(L, rsm, w)
    w("    const RT bPAx = RT(ab.PAx), bPAy = RT(ab.PAy), bPAz = RT(ab.PAz);")
    w("    const RT bPBx = RT(ab.PBx), bPBy = RT(ab.PBy), bPBz = RT(ab.PBz);")
    w("    const RT kPAx = RT(cd.PAx), kPAy = RT(cd.PAy), kPAz = RT(cd.PAz);")
    w("    const RT kPBx = RT(cd.PBx), kPBy = RT(cd.PBy), kPBz = RT(cd.PBz);")
    if chunked:
        for fn in chunk_names:
            w("    if constexpr (LOCKSTEP) __syncthreads();")
            w(f"    {fn}<RT, Sink>(rs, rstride, a12b, bPAx, bPAy, bPAz, bPBx, bPBy, bPBz, a12k, kPAx, kPAy, "
              f"kPAz, kPBx, kPBy, kPBz, lambda, sink);")
    else:
        for s_ in e_tables(LA, LB, LC, LD):
            w("    " + s_)
        ket_blocks(LA, LB, LC, LD, all_cds, w)
    w("#undef RR")
    w("}")
    # chunk c alone (after Boys and R): lets several warps share one quartet's ket components when a class
    # has too few quartets to fill the GPU; an unchunked class has the single chunk 0
    w("template <class RT, class Sink>")
    w(f"__device__ __forceinline__ void prim_quartet_chunk_{idx}(const int c, const PrimPairData& ab,")
    w("    const PrimPairData& cd, const double* __restrict__ bt, RT* __restrict__ rs, const int rstride,")
    w("    Sink& sink)")
    w("{")
    if chunked:
        r_prologue(L, True, w)
        w("    const RT bPAx = RT(ab.PAx), bPAy = RT(ab.PAy), bPAz = RT(ab.PAz);")
        w("    const RT bPBx = RT(ab.PBx), bPBy = RT(ab.PBy), bPBz = RT(ab.PBz);")
        w("    const RT kPAx = RT(cd.PAx), kPAy = RT(cd.PAy), kPAz = RT(cd.PAz);")
        w("    const RT kPBx = RT(cd.PBx), kPBy = RT(cd.PBy), kPBz = RT(cd.PBz);")
        w("    switch (c)")
        w("    {")
        for ci, fn in enumerate(chunk_names):
            w(f"    case {ci}: {fn}<RT, Sink>(rs, rstride, a12b, bPAx, bPAy, bPAz, bPBx, bPBy, bPBz, a12k, kPAx, "
              f"kPAy, kPAz, kPBx, kPBy, kPBz, lambda, sink); break;")
        w("    default: break;")
        w("    }")
        w("#undef RR")
    else:
        w("    (void)c;")
        w(f"    prim_quartet_{idx}<RT, Sink>(ab, cd, bt, rs, rstride, sink);")
    w("}")
    return o


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for k, (la, lb, lc, ld) in enumerate(classes()):
        body = gen_class(la, lb, lc, ld, k)
        text = ("// generated by gen_md.py -- do not edit\n#pragma once\n#include \"../md_core.cuh\"\n"
                "namespace qcg {\nnamespace gen {\n" + "\n".join(body) + "\n}  // namespace gen\n}  // namespace qcg\n")
        path = os.path.join(outdir, f"md_class_{k}.cuh")
        old = open(path).read() if os.path.exists(path) else None
        if old != text:
            with open(path, "w") as f:
                f.write(text)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "gen"))


# ------------------------------------------------------------------------------------------------------
# Horizontal-recurrence (HRR) form, generated on request only (main_hrr): the primitive quartets produce
# [e0|f0] for e over the Cartesian components of L = LA..LA+LB on centre A and f over L = LC..LC+LD on
# centre C (E^{e0} tables, one index per pair), accumulated over the primitives of a contracted quartet;
# the contracted block is then carried to (ab|cd) by
#     (x, y + 1_i) = (x + 1_i, y) + D_i (x, y),   D = C - D on the ket, A - B on the bra,
# once per contracted quartet instead of once per primitive quartet.  The library's kernels do not use it
# yet; tests/test_gen_md_host.py checks it against the oracle on the host.
# ------------------------------------------------------------------------------------------------------
# f components per chunk of the chunked HRR classes: with one, no (dd|dd) chunk spills under ptxas for
# sm_100a (two spill 2.3 KB over the class); each chunk rebuilds its E tables (~90 operations against
# ~500 for one f of (dd|dd)), which a B200 measurement has to weigh
HRR_F_PER_CHUNK = 1


def comps_range(L0, L1):
    return [c for L in range(L0, L1 + 1) for c in comps(L)]


def hrr_code(Lx, Ly, src, dst, D, w, prefix):
    """Straight-line HRR for all (x, y), x in comps(Lx), y in comps(Ly), from src(k) = the value of
    (comps_range(Lx, Lx + Ly)[k], 0); every intermediate (x, y) node is computed once.  All sources are
    loaded before the first result is stored, so the results may overwrite the sources (in place)."""
    F = comps_range(Lx, Lx + Ly)
    fidx = {c: k for k, c in enumerate(F)}
    for k in range(len(F)):
        w(f"    const RT {prefix}s{k} = {src(k)};")
    memo = {}

    def node(x, y):
        key = (x, y)
        if key in memo:
            return memo[key]
        if sum(y) == 0:
            memo[key] = f"{prefix}s{fidx[x]}"
            return memo[key]
        i = next(a for a in range(3) if y[a] > 0)
        y1 = tuple(y[a] - (a == i) for a in range(3))
        x1 = tuple(x[a] + (a == i) for a in range(3))
        hi, lo = node(x1, y1), node(x, y1)
        name = f"{prefix}{len(memo)}"
        w(f"    const RT {name} = qfma({D[i]}, {lo}, {hi});")
        memo[key] = name
        return name

    for ix, x in enumerate(comps(Lx)):
        for iy, y in enumerate(comps(Ly)):
            w(dst(ix, iy, node(x, y), comp_norm(x) * comp_norm(y)))


def hrr_f_blocks(LAB, L, E, F, fsel, w):
    """[e0|f0] for the f of F listed in fsel (indices into F), every e of E; R read through RR()."""
    HAB = herm_list(LAB)
    NX = len(HAB)
    for jf in fsel:
        f = F[jf]
        w(f"    {{ // f = {f}")
        supp = [(tp, up, vp) for tp in range(f[0] + 1) for up in range(f[1] + 1) for vp in range(f[2] + 1)]
        for (tp, up, vp) in supp:
            sgn = "-" if (tp + up + vp) & 1 else ""
            w(f"    const RT s{tp}{up}{vp} = {sgn}ekx_{f[0]}_0_{tp} * eky_{f[1]}_0_{up} * ekz_{f[2]}_0_{vp};")
        w("    RT " + ", ".join(f"x{i} = RT(0)" for i in range(NX)) + ";")
        contrib = {}
        for h in HAB:
            for hp in supp:
                H = hidx(L, h[0] + hp[0], h[1] + hp[1], h[2] + hp[2])
                contrib.setdefault(H, []).append((hidx(LAB, *h), hp))
        for H in sorted(contrib):
            body = " ".join(f"x{xi} = qfma(s{hp[0]}{hp[1]}{hp[2]}, r, x{xi});" for (xi, hp) in contrib[H])
            w(f"    {{ const RT r = RR({H}); {body} }}")
        for je, e in enumerate(E):
            w("    {")
            w("      RT sx = RT(0);")
            for t in range(e[0] + 1):
                w("      { RT sy = RT(0);")
                for u in range(e[1] + 1):
                    zs = f"ebz_{e[2]}_0_0 * x{hidx(LAB, t, u, 0)}"
                    for v in range(1, e[2] + 1):
                        zs = f"qfma(ebz_{e[2]}_0_{v}, x{hidx(LAB, t, u, v)}, {zs})"
                    w(f"        sy = qfma(eby_{e[1]}_0_{u}, {zs}, sy);")
                w(f"        sx = qfma(ebx_{e[0]}_0_{t}, sy, sx); }}")
            w(f"      sink({je}, {jf}, sx * lambda);")
            w("    }")
        w("    }")


def hrr_e_tables(LAB, LCD):
    out = []
    for dname, Lmax, PA, a12 in (("ebx", LAB, "bPAx", "a12b"), ("eby", LAB, "bPAy", "a12b"),
                                 ("ebz", LAB, "bPAz", "a12b"), ("ekx", LCD, "kPAx", "a12k"),
                                 ("eky", LCD, "kPAy", "a12k"), ("ekz", LCD, "kPAz", "a12k")):
        out.extend(gen_E(dname, Lmax, 0, PA, "0", a12))
    return out


def gen_class_hrr(LA, LB, LC, LD, idx):
    L = LA + LB + LC + LD
    LAB, LCD = LA + LB, LC + LD
    E, F = comps_range(LA, LAB), comps_range(LC, LCD)
    chunked = len(E) * len(F) > CHUNK_ABOVE
    rsm = L >= R_SMEM_MIN_L or chunked
    o = []
    w = o.append
    w(f"// class {idx} in HRR form: [e0|f0] has {len(E)} x {len(F)} entries"
      f"{'; f split into __noinline__ chunks' if chunked else ''}")
    w(f"constexpr int kHrrE{idx} = {len(E)};")
    w(f"constexpr int kHrrF{idx} = {len(F)};")
    w(f"constexpr bool kHrrRShared{idx} = {'true' if rsm else 'false'};")
    chunk_names = []
    if chunked:
        per = HRR_F_PER_CHUNK
        groups = [list(range(len(F)))[i:i + per] for i in range(0, len(F), per)]
        for ci, fsel in enumerate(groups):
            fn = f"prim_quartet_hrr_{idx}_chunk{ci}"
            chunk_names.append(fn)
            w("template <class RT, class Sink>")
            w(f"__device__ __noinline__ void {fn}(const RT* __restrict__ rs, const int rstride, const RT a12b,")
            w("    const RT bPAx, const RT bPAy, const RT bPAz, const RT a12k, const RT kPAx, const RT kPAy,")
            w("    const RT kPAz, const RT lambda, typename SinkArg<Sink>::type sink)")
            w("{")
            for s_ in hrr_e_tables(LAB, LCD):
                w("    " + s_)
            w("#define RR(i) rs[(i) * rstride]")
            hrr_f_blocks(LAB, L, E, F, fsel, w)
            w("#undef RR")
            w("}")
    # primitive quartet -> sink(ie, if, value)
    w("template <class RT, class Sink>")
    w(f"__device__ __forceinline__ void prim_quartet_hrr_{idx}(const PrimPairData& ab, const PrimPairData& cd,")
    w("    const double* __restrict__ bt, RT* __restrict__ rs, const int rstride, Sink& sink)")
    w("{")
    w("    (void)rs; (void)rstride;")
    r_prologue(L, rsm, w)
    w("    const RT bPAx = RT(ab.PAx), bPAy = RT(ab.PAy), bPAz = RT(ab.PAz);")
    w("    const RT kPAx = RT(cd.PAx), kPAy = RT(cd.PAy), kPAz = RT(cd.PAz);")
    if chunked:
        for fn in chunk_names:
            w(f"    {fn}<RT, Sink>(rs, rstride, a12b, bPAx, bPAy, bPAz, a12k, kPAx, kPAy, kPAz, lambda, sink);")
    else:
        for s_ in hrr_e_tables(LAB, LCD):
            w("    " + s_)
        hrr_f_blocks(LAB, L, E, F, range(len(F)), w)
    w("#undef RR")
    w("}")
    # ket HRR of one e row: p[f] -> y[c * ND + d], times the (c, d) component norms (y may be p)
    nd = len(comps(LD))
    w("template <class RT>")
    w(f"__device__ __forceinline__ void hrr_ket_{idx}(const RT* p, RT* y, const RT CDx,")
    w("    const RT CDy, const RT CDz)")
    w("{")
    hrr_code(LC, LD, lambda k: f"ld_l2(p + {k})", lambda ix, iy, v, nrm: f"    y[{ix * nd + iy}] = {v} * RT({lit(nrm)});",
             ("CDx", "CDy", "CDz"), w, "t")
    w("}")
    # bra HRR of one (c, d) column: y[e * ys] -> o[(a * NB + b) * os], times the (a, b) component norms
    # (o may be y, with os == ys)
    nb = len(comps(LB))
    w("template <class RT>")
    w(f"__device__ __forceinline__ void hrr_bra_{idx}(const RT* y, const int ys, RT* o,")
    w("    const int os, const RT ABx, const RT ABy, const RT ABz)")
    w("{")
    hrr_code(LA, LB, lambda k: f"ld_l2(y + {k} * ys)",
             lambda ix, iy, v, nrm: f"    o[{ix * nb + iy} * os] = {v} * RT({lit(nrm)});", ("ABx", "ABy", "ABz"), w,
             "t")
    w("}")
    return o


def main_hrr(outdir):
    """Writes md_hrr_<k>.cuh (the HRR form of class k) for k = 0..20 into outdir."""
    os.makedirs(outdir, exist_ok=True)
    for k, (la, lb, lc, ld) in enumerate(classes()):
        body = gen_class_hrr(la, lb, lc, ld, k)
        text = ("// generated by gen_md.py (HRR form) -- do not edit\n#pragma once\n#include \"../md_core.cuh\"\n"
                "namespace qcg {\nnamespace gen {\n" + "\n".join(body) + "\n}  // namespace gen\n}  // namespace qcg\n")
        with open(os.path.join(outdir, f"md_hrr_{k}.cuh"), "w") as f:
            f.write(text)


# ------------------------------------------------------------------------------------------------------
# Team form (main_team): the code of the warp-specialised ERI-batch kernel (eri_team.cuh).  A CTA holds 32
# contracted quartets, one per lane.  Per primitive quartet a producer warp writes a shared-memory stage
# per lane: R^0_{tuv} scaled by the prefactor lambda, and the single-centre Hermite tables E^{i0}_t of the
# ket pair (and, after the last ket primitive of a bra primitive pair, of the bra pair).  Consumer warp w
# owns one ket component f of the HRR form ([e0|f0], f over L = LC..LC+LD on centre C) and keeps in
# registers
#     Y_f[h] = sum over the ket primitives of sum_{h' in supp(f)} (-1)^{|h'|} E^{f0}_{h'} R_{h+h'}
# for h over the bra's Hermite indices, and, once per bra primitive pair, adds
#     acc_f[e] += sum_t E^{ex 0}_t sum_u E^{ey 0}_u sum_v E^{ez 0}_v Y_f[tuv]
# so the bra contraction runs once per bra primitive pair instead of once per primitive quartet.  The
# ket and bra horizontal recurrences of the HRR form then give (ab|cd).  All indices are literals.
# ------------------------------------------------------------------------------------------------------
def ne1(Lmax):
    """stored 1-D entries E^{i0}_t, 1 <= i <= Lmax, t <= i (E^{00}_0 = 1 is not stored)"""
    return (Lmax + 1) * (Lmax + 2) // 2 - 1


def e1_slot(i, t):
    return i * (i + 1) // 2 - 1 + t


def r_stream(L, w, store):
    """Boys -> R^0_{tuv} for t+u+v <= L, each stored once through store(H, name) as soon as it exists.
    Same recursion and branch order as r_prologue (x first, then y, then z), evaluated column by column
    (v, then u, then t) so that only the columns the next ones need stay live; lambda is folded into
    R^n_{000}, so every R value carries it."""
    w("    const double p = ab.p, q = cd.p, pq = p + q;")
    w("    const double alpha = p * q / pq;")
    w("    const double Xd = ab.Px - cd.Px, Yd = ab.Py - cd.Py, Zd = ab.Pz - cd.Pz;")
    w(f"    RT F[{L + 1}];")
    w(f"    boys<{L}>(alpha * (Xd * Xd + Yd * Yd + Zd * Zd), bt, F);")
    w("    const RT X = RT(Xd), Y = RT(Yd), Z = RT(Zd);")
    w("    const RT m2a = RT(-2.0 * alpha);")
    w("    const RT lambda = RT(34.986836655249725693 / (p * q * sqrt(pq)) * ab.K * cd.K);")
    w("    const RT g0 = lambda;")
    for n in range(1, L + 1):
        w(f"    const RT g{n} = g{n - 1} * m2a;")

    def nm(n, t, u, v):
        return f"r{n}_{t}_{u}_{v}"

    for v in range(L + 1):
        for n in range(L - v + 1):
            if v == 0:
                w(f"    const RT {nm(n, 0, 0, 0)} = g{n} * F[{n}];")
            else:
                e = f"Z * {nm(n + 1, 0, 0, v - 1)}"
                if v > 1:
                    e += f" + RT({v - 1}) * {nm(n + 1, 0, 0, v - 2)}"
                w(f"    const RT {nm(n, 0, 0, v)} = {e};")
        for u in range(L - v + 1):
            if u >= 1:
                for n in range(L - u - v + 1):
                    e = f"Y * {nm(n + 1, 0, u - 1, v)}"
                    if u > 1:
                        e += f" + RT({u - 1}) * {nm(n + 1, 0, u - 2, v)}"
                    w(f"    const RT {nm(n, 0, u, v)} = {e};")
            for t in range(L - u - v + 1):
                if t >= 1:
                    for n in range(L - t - u - v + 1):
                        e = f"X * {nm(n + 1, t - 1, u, v)}"
                        if t > 1:
                            e += f" + RT({t - 1}) * {nm(n + 1, t - 2, u, v)}"
                        w(f"    const RT {nm(n, t, u, v)} = {e};")
                w(store(hidx(L, t, u, v), nm(0, t, u, v)))


def gen_class_team(LA, LB, LC, LD, idx):
    L = LA + LB + LC + LD
    LAB, LCD = LA + LB, LC + LD
    E, F = comps_range(LA, LAB), comps_range(LC, LCD)
    HAB = herm_list(LAB)
    NR, NH = nherm(L), nherm(LAB)
    NEB, NEK = 3 * ne1(LAB), 3 * ne1(LCD)
    BOFF, KOFF = NR, NR + NEB
    o = []
    w = o.append
    w(f"// class {idx} in team form: R has {NR} entries, Y_f {NH}, [e0|f0] {len(E)} x {len(F)}")
    w(f"constexpr int kTeamNR{idx} = {NR};")
    w(f"constexpr int kTeamNH{idx} = {NH};")
    w(f"constexpr int kTeamNE{idx} = {len(E)};")
    w(f"constexpr int kTeamNF{idx} = {len(F)};")
    w(f"constexpr int kTeamStage{idx} = {NR + NEB + NEK};   // stage entries per lane")
    # ket-step instruction estimate (loads, products, fused multiply-adds) of the largest component: the
    # launcher sizes its warp count so that the ket code running at once fits the instruction cache
    sizes = []
    for f in F:
        supp = (f[0] + 1) * (f[1] + 1) * (f[2] + 1)
        idxs = set((h[0] + a, h[1] + b, h[2] + c) for h in HAB for a in range(f[0] + 1) for b in range(f[1] + 1)
                   for c in range(f[2] + 1))
        sizes.append(len(HAB) * supp + len(idxs) + 2 * supp + sum(f) + 3)
    w(f"constexpr int kTeamKetInstr{idx} = {max(sizes)};")
    # producer
    w("// one lane's stage for one primitive quartet: entry i at st[i * 32]; the bra tables only when bra_e")
    w("template <class RT>")
    w(f"__device__ __forceinline__ void team_produce_{idx}(RT* __restrict__ st, const PrimPairData& ab,")
    w("    const PrimPairData& cd, const double* __restrict__ bt, const bool bra_e)")
    w("{")
    r_stream(L, w, lambda H, name: f"    st[{H} * 32] = {name};")
    if LCD > 0:
        w("    {")
        w("    const RT a12k = RT(0.5 / cd.p);")
        w("    const RT kPAx = RT(cd.PAx), kPAy = RT(cd.PAy), kPAz = RT(cd.PAz);")
        for d, (dn, PA) in enumerate((("ekx", "kPAx"), ("eky", "kPAy"), ("ekz", "kPAz"))):
            for s_ in gen_E(dn, LCD, 0, PA, "0", "a12k"):
                w("    " + s_)
            for i in range(1, LCD + 1):
                for t in range(i + 1):
                    w(f"    st[{KOFF + d * ne1(LCD) + e1_slot(i, t)} * 32] = {dn}_{i}_0_{t};")
        w("    }")
    if LAB > 0:
        w("    if (bra_e)")
        w("    {")
        w("    const RT a12b = RT(0.5 / ab.p);")
        w("    const RT bPAx = RT(ab.PAx), bPAy = RT(ab.PAy), bPAz = RT(ab.PAz);")
        for d, (dn, PA) in enumerate((("ebx", "bPAx"), ("eby", "bPAy"), ("ebz", "bPAz"))):
            for s_ in gen_E(dn, LAB, 0, PA, "0", "a12b"):
                w("    " + s_)
            for i in range(1, LAB + 1):
                for t in range(i + 1):
                    w(f"    st[{BOFF + d * ne1(LAB) + e1_slot(i, t)} * 32] = {dn}_{i}_0_{t};")
        w("    }")
    else:
        w("    (void)bra_e;")
    w("}")
    # consumer: ket step of component jf
    w("// Y_f[h] += sum_{h' in supp(f)} (-1)^{|h'|} E^{f0}_{h'} R_{h+h'} for ket component jf (warp-uniform)")
    w("template <class RT>")
    w(f"__device__ __forceinline__ void team_ket_{idx}(const int jf, const RT* __restrict__ st, RT (&Yf)[{NH}])")
    w("{")
    w("    switch (jf)")
    w("    {")
    for jf, f in enumerate(F):
        w(f"    case {jf}: {{ // f = {f}")
        for d, dn in enumerate(("ekx", "eky", "ekz")):
            for t in range(f[d] + 1):
                if f[d] == 0:
                    w(f"    const RT {dn}_0_0_0 = RT(1);")
                else:
                    w(f"    const RT {dn}_{f[d]}_0_{t} = st[{KOFF + d * ne1(LCD) + e1_slot(f[d], t)} * 32];")
        supp = [(tp, up, vp) for tp in range(f[0] + 1) for up in range(f[1] + 1) for vp in range(f[2] + 1)]
        for (tp, up, vp) in supp:
            sgn = "-" if (tp + up + vp) & 1 else ""
            w(f"    const RT s{tp}{up}{vp} = {sgn}ekx_{f[0]}_0_{tp} * eky_{f[1]}_0_{up} * ekz_{f[2]}_0_{vp};")
        contrib = {}
        for h in HAB:
            for hp in supp:
                H = hidx(L, h[0] + hp[0], h[1] + hp[1], h[2] + hp[2])
                contrib.setdefault(H, []).append((hidx(LAB, *h), hp))
        for H in sorted(contrib):
            body = " ".join(f"Yf[{xi}] = qfma(s{hp[0]}{hp[1]}{hp[2]}, r, Yf[{xi}]);" for (xi, hp) in contrib[H])
            w(f"    {{ const RT r = st[{H} * 32]; {body} }}")
        w("    } break;")
    w("    default: break;")
    w("    }")
    w("}")
    # consumer: bra step (the same for every f)
    w("// acc[e] += sum_t E^{ex 0}_t sum_u E^{ey 0}_u sum_v E^{ez 0}_v Y_f[tuv], bra tables from the stage")
    w("template <class RT>")
    w(f"__device__ __forceinline__ void team_bra_{idx}(const RT* __restrict__ st, const RT (&Yf)[{NH}],")
    w(f"    RT (&acc)[{len(E)}])")
    w("{")
    for d, dn in enumerate(("ebx", "eby", "ebz")):
        w(f"    const RT {dn}_0_0_0 = RT(1);")
        for i in range(1, LAB + 1):
            for t in range(i + 1):
                w(f"    const RT {dn}_{i}_0_{t} = st[{BOFF + d * ne1(LAB) + e1_slot(i, t)} * 32];")
    for je, e in enumerate(E):
        w("    {")
        w("      RT sx = RT(0);")
        for t in range(e[0] + 1):
            w("      { RT sy = RT(0);")
            for u in range(e[1] + 1):
                zs = f"ebz_{e[2]}_0_0 * Yf[{hidx(LAB, t, u, 0)}]"
                for v in range(1, e[2] + 1):
                    zs = f"qfma(ebz_{e[2]}_0_{v}, Yf[{hidx(LAB, t, u, v)}], {zs})"
                w(f"        sy = qfma(eby_{e[1]}_0_{u}, {zs}, sy);")
            w(f"        sx = qfma(ebx_{e[0]}_0_{t}, sy, sx); }}")
        w(f"      acc[{je}] += sx;")
        w("    }")
    w("}")
    # the recurrences on the per-CTA scratch, whose layout is lane-minor (element k of lane l at [k * 32 + l]):
    # ket of one e row: p[f] -> y[c * ND + d]; bra of one (c d) column: y[e * NCD] -> o[(a * NB + b) * os]
    nd, nb, ncd = len(comps(LD)), len(comps(LB)), len(comps(LC)) * len(comps(LD))
    w("template <class RT>")
    w(f"__device__ __forceinline__ void team_hrr_ket_{idx}(const RT* p, RT* y, const RT CDx, const RT CDy,")
    w("    const RT CDz)")
    w("{")
    hrr_code(LC, LD, lambda k: f"p[{k} * 32]", lambda ix, iy, v, nrm: f"    y[{ix * nd + iy} * 32] = {v} * RT({lit(nrm)});",
             ("CDx", "CDy", "CDz"), w, "t")
    w("}")
    w("template <class RT>")
    w(f"__device__ __forceinline__ void team_hrr_bra_{idx}(const RT* y, RT* o, const int os, const RT ABx,")
    w("    const RT ABy, const RT ABz)")
    w("{")
    hrr_code(LA, LB, lambda k: f"y[{k * ncd} * 32]",
             lambda ix, iy, v, nrm: f"    o[{ix * nb + iy} * os] = {v} * RT({lit(nrm)});", ("ABx", "ABy", "ABz"), w, "t")
    w("}")
    return o


def main_team(outdir, classes_=None):
    """Writes md_team_<k>.cuh (the team form of class k) for the classes listed (default: all 21)."""
    os.makedirs(outdir, exist_ok=True)
    for k, (la, lb, lc, ld) in enumerate(classes()):
        if classes_ is not None and k not in classes_:
            continue
        body = gen_class_team(la, lb, lc, ld, k)
        text = ("// generated by gen_md.py (team form) -- do not edit\n#pragma once\n#include \"../md_core.cuh\"\n"
                "namespace qcg {\nnamespace gen {\n" + "\n".join(body) + "\n}  // namespace gen\n}  // namespace qcg\n")
        path = os.path.join(outdir, f"md_team_{k}.cuh")
        old = open(path).read() if os.path.exists(path) else None
        if old != text:
            with open(path, "w") as f:
                f.write(text)
