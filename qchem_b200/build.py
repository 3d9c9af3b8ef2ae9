"""Build libqchem_b200.so (the C ABI of include/qchem_b200.h) for sm_100a, in-tree.

  python -m qchem_b200.build [--force] [-j N]

Steps: generate the per-class MD code (csrc/gen_md.py), compile the 2 x 21 class objects (FP64 and
FP32) plus the
runtime in parallel with nvcc (-gencode arch=compute_100a,code=sm_100a -lineinfo), link a shared
library into qchem_b200/_lib/.  Objects are cached in qchem_b200/_build/ keyed by a hash of their
inputs, so unchanged classes are not recompiled.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "gen")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libqchem_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")   # cuSOLVER / cuBLAS of the SCF step
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
NCLASS = 21
HOST_OMP = ["-Xcompiler", "-fopenmp", "-Xcompiler", "-march=x86-64-v3"]   # the SCF's host linear algebra (eigensolver, products) is threaded


def _read(p):
    with open(p, "rb") as f:
        return f.read()


def _hash(parts):
    h = hashlib.sha256()
    for p in parts:
        h.update(p if isinstance(p, bytes) else p.encode())
    return h.hexdigest()[:20]


def _headers(names):
    return [_read(os.path.join(CSRC, n)) for n in names]


# FP64 ERI-batch classes built in the horizontal-recurrence form: measured on a B200 at 10^6 quartets per
# class, (dp|dp) 1.36x, (dd|pp) 1.23x, (dd|dp) 1.41x and (dd|dd) 1.52x faster than the direct form; every
# other class was slower (its read-back and recurrence work outweigh the smaller saving)
HRR_CLASSES = (14, 17, 19, 20)


def _eri_hrr(k: int) -> bool:
    """Whether class k's FP64 ERI batches use the horizontal-recurrence form: HRR_CLASSES, or every class
    with QCG_ERI_HRR=1 in the environment, or none with QCG_ERI_HRR=0."""
    env = os.environ.get("QCG_ERI_HRR")
    if env == "1":
        return True
    if env == "0":
        return False
    return k in HRR_CLASSES


# FP64 ERI-batch classes that run in the team form (eri_team.cu) by default: every class whose ket pair is not
# (ss).  Measured on a B200 at 10^6 quartets per class, the team form was 1.15-6.8x faster on these 15 classes
# ((dd|dd) 2.8x, (dd|pp) 6.8x); on the (xx|ss) classes, whose single ket component gives a one-warp CTA, it was
# 0.6-1.0x.  Every class has a team launcher; QCG_ERI_TEAM_MASK in the environment selects others at run time.
TEAM_CLASSES = tuple(k for k in range(NCLASS) if k not in (0, 1, 3, 6, 10, 15))


def _team_mask() -> int:
    return sum(1 << k for k in TEAM_CLASSES)


# classes whose direct J/K build runs in the team form by default (QCG_JK_TEAM_MASK selects others at run time):
# (dd|dd), (dd|dp), (dd|ds), (dd|pp), (dd|ps), (dp|dp).  Measured class by class on a B200 on the
# uncontracted 32-water build (1824 functions), the team form took 0.47-0.93x the thread-per-quartet kernel's
# time on these six ((dd|dd) 43 vs 92 ms, (dp|dp) 528 vs 826 ms) and 0.31-0.76x the warp-shared form's; on
# (dp|pp) the warp-shared form is faster still (999 vs 1231 ms), and on the others the team form took
# 1.07-4.7x the thread-per-quartet time.
JK_TEAM_CLASSES = (14, 16, 17, 18, 19, 20)


def _jk_team_mask() -> int:
    return sum(1 << k for k in JK_TEAM_CLASSES)


# classes whose direct J/K build runs in the warp-shared form by default (QCG_JK_WARP_MASK selects others):
# (ps|ss), (ps|ps), (pp|ss), (pp|ps), (ds|ss), (ds|ps), (ds|pp), (ds|ds), (dp|ss), (dp|ps), (dp|pp), (dp|ds).
# Measured class by class on a B200 on the uncontracted 32-water build (half-warp sets), the warp-shared form
# took 0.51-0.82x the thread-per-quartet kernel's time on these twelve ((ds|ps) 219 vs 428 ms, (dp|ds) 625
# vs 872 ms, (dp|pp) 994 vs 1345 ms, where the team form took 1231 ms); on (ss|ss), (pp|pp) and (dd|ss) it
# was level (1.00-1.02x), and those stay thread-per-quartet.
JK_WARP_CLASSES = (1, 2, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13)


def _jk_warp_mask() -> int:
    return sum(1 << k for k in JK_WARP_CLASSES)


def _jobs():
    core = _headers(["md_core.cuh", "qcg_internal.h"])
    jobs = []
    src = os.path.join(CSRC, "eri_class.cu")
    for prec in (64, 32):
        for k in range(NCLASS):
            defs = [f"-DQCG_CLASS={k}", f"-DQCG_PREC={prec}"]
            parts = [_read(src), _read(os.path.join(GEN, f"md_class_{k}.cuh"))]
            if _eri_hrr(k) and prec == 64:
                defs.append("-DQCG_ERI_HRR=1")
                parts.append(_read(os.path.join(GEN, f"md_hrr_{k}.cuh")))
            key = _hash(parts + core + _headers(["eri_kernels.cuh", "smem_attr.h"]) + FLAGS + defs)
            jobs.append((src, defs, os.path.join(BUILD, f"eri_class_{k}_f{prec}_{key}.o")))
    team_src = os.path.join(CSRC, "eri_team.cu")
    for k in range(NCLASS):
        defs = [f"-DQCG_CLASS={k}"]
        parts = [_read(team_src), _read(os.path.join(GEN, f"md_team_{k}.cuh"))]
        key = _hash(parts + core + _headers(["eri_kernels.cuh", "eri_team.cuh", "eri_team_iface.h", "team_sync.cuh", "smem_attr.h"])
                    + FLAGS + defs)
        jobs.append((team_src, defs, os.path.join(BUILD, f"eri_team_{k}_{key}.o")))
    extra = {"runtime.cu": _headers(["boys_table.h", "eri_team_iface.h"]) + [_read(os.path.join(INCLUDE, "qchem_b200.h"))],
             "registry.cu": _headers(["eri_team_iface.h"]),
             "fock_kernels.cu": _headers(["team_sync.cuh"]),
             "mlp.cu": [_read(os.path.join(INCLUDE, "qchem_b200.h"))] + _headers(["smem_attr.h", "team_sync.cuh"])}
    for name in ("registry.cu", "fock_kernels.cu", "runtime.cu", "mlp.cu"):
        s = os.path.join(CSRC, name)
        defs = HOST_OMP + [f"-DQCG_TEAM_DEFAULT_MASK={_team_mask():#x}u",
                           f"-DQCG_JK_TEAM_DEFAULT_MASK={_jk_team_mask():#x}u",
                           f"-DQCG_JK_WARP_DEFAULT_MASK={_jk_warp_mask():#x}u"] if name == "runtime.cu" else []
        key = _hash([_read(s)] + core + extra.get(name, []) + FLAGS + defs)
        jobs.append((s, defs, os.path.join(BUILD, f"{name[:-3]}_{key}.o")))
    return jobs


def _compile(job):
    src, defs, obj = job
    if os.path.exists(obj):
        return obj, False
    tmp = obj + ".tmp.o"
    cmd = [NVCC] + FLAGS + defs + ["-I", CSRC, "-c", src, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=CSRC)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)} {defs}:\n{r.stderr[-4000:]}")
    os.replace(tmp, obj)
    return obj, True


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    sys.path.insert(0, CSRC)
    try:
        import gen_md  # noqa: E402
    finally:
        sys.path.pop(0)
    gen_md.main(GEN)
    gen_md.main_hrr(GEN)
    gen_md.main_team(GEN)
    if not os.path.exists(os.path.join(CSRC, "boys_table.h")):
        raise RuntimeError("csrc/boys_table.h is missing (python csrc/gen_boys_table.py regenerates it)")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    todo = _jobs()
    if force:
        for _, _, obj in todo:
            if os.path.exists(obj):
                os.remove(obj)
    # biggest classes first so that the slowest compiles start early
    todo.sort(key=lambda j: -os.path.getsize(os.path.join(GEN, f"md_class_{j[1][0].split('=')[1]}.cuh"))
              if j[1] and j[1][0].startswith("-DQCG_CLASS") else 0)
    n = jobs or max(1, os.cpu_count() or 1)
    built = []
    with cf.ThreadPoolExecutor(max_workers=n) as ex:
        for obj, fresh in ex.map(_compile, todo):
            built.append(obj)
            if verbose and fresh:
                print("compiled", os.path.basename(obj), flush=True)
    objs = [o for _, _, o in todo]
    key = _hash([os.path.basename(o) for o in sorted(objs)])
    stamp = LIB + ".key"
    if force or not os.path.exists(LIB) or not os.path.exists(stamp) or open(stamp).read() != key:
        tmp = LIB + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + [
            "-lgomp", "-L", CUDA_LIB, "-lcusolver", "-lcublas", "-Xlinker", "-rpath=" + CUDA_LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr[-4000:])
        os.replace(tmp, LIB)
        with open(stamp, "w") as f:
            f.write(key)
    # drop stale objects of older source versions
    keep = set(objs)
    for f in os.listdir(BUILD):
        p = os.path.join(BUILD, f)
        if p.endswith(".o") and p not in keep:
            os.remove(p)
    return LIB


if __name__ == "__main__":
    j = None
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    print(build(force="--force" in sys.argv, jobs=j, verbose=True))
