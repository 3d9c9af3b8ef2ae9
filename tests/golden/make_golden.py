"""Write the golden fixtures of tests/golden/ from the reference sources (JanReimers/qchem).

Run where the reference source tree is available, naming its root in QCHEM_REF:
    QCHEM_REF=<path to the qchem checkout> python tests/golden/make_golden.py

Outputs (committed):
  boys_reference_sample.json  -- entries of the reference's Boys table (Internal/Boys/Imp/AuxillaryData.C)
                                 at sampled rows, all 23 orders, plus the maximum relative difference of
                                 the whole reference table from this project's generated table
  dzvp_HNO.bsd                -- the H, N and O entries of BasisSetData/dzvp.bsd (DZVP orbital basis data)
  anchors.json                -- the reference's RHF energy anchors with geometries and tolerances
                                 (IntegrationTests/M_HF_U.C:21-51)
The tests only read these files; nothing at test time touches the reference tree.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("QCHEM_REF")
if not REF:
    sys.exit("set QCHEM_REF to the root of the qchem source tree")


def reference_boys_table():
    path = os.path.join(REF, "src/BasisSet/Molecule/Evaluators/Internal/Boys/Imp/AuxillaryData.C")
    text = open(path).read()
    body = text[text.index("theLookUp[121][23]"):]
    nums = [float(x) for x in re.findall(r"[-+]?\d\.\d+E[-+]\d+", body)]
    assert len(nums) == 121 * 23, len(nums)
    return [nums[i * 23:(i + 1) * 23] for i in range(121)]


def product_boys_table():
    text = open(os.path.join(REPO, "qchem_b200/csrc/boys_table.h")).read()
    body = text[text.index("{") + 1:text.index("}")]
    nums = [float(x) for x in body.replace("\n", " ").split(",") if x.strip()]
    return [nums[i * 23:(i + 1) * 23] for i in range(121)]


def main():
    ref = reference_boys_table()
    prod = product_boys_table()
    maxrel = 0.0
    for i in range(121):
        for j in range(23):
            maxrel = max(maxrel, abs(ref[i][j] - prod[i][j]) / abs(ref[i][j]))
    rows = [0, 1, 7, 33, 60, 99, 119, 120]
    sample = {"source": "src/BasisSet/Molecule/Evaluators/Internal/Boys/Imp/AuxillaryData.C",
              "rows": rows, "T": [0.1 * r for r in rows], "values": [ref[r] for r in rows],
              "max_rel_diff_full_table_vs_generated": maxrel}
    with open(os.path.join(HERE, "boys_reference_sample.json"), "w") as f:
        json.dump(sample, f, indent=1)

    bsd = open(os.path.join(REF, "BasisSetData/dzvp.bsd")).read().splitlines()
    out = []
    i = 0
    while i < len(bsd) and bsd[i].strip() != "!":
        out.append(bsd[i])
        i += 1
    out.extend(bsd[i:i + 2])
    i += 2
    keep = {"H", "N", "O"}
    cur = None
    for ln in bsd[i:]:
        tok = ln.split()
        if not tok:
            continue
        if cur is None:
            if len(tok) == 2 and tok[1].lstrip("-").isdigit():
                cur = tok[0].upper()
                if cur in keep:
                    out.append(ln)
            else:
                break
            continue
        if cur in keep:
            out.append(ln)
        if tok[0] == "****":
            cur = None
    with open(os.path.join(HERE, "dzvp_HNO.bsd"), "w") as f:
        f.write("\n".join(out) + "\n")

    anchors = {
        "source": "IntegrationTests/M_HF_U.C:21-51 (RHF/DZVP, Cartesian d, core guess, DIIS)",
        "water": {"Z": [8, 1, 1], "R": [[0, 0, 0], [0, 1.431, 1.107], [0, -1.431, 1.107]],
                  "energy": -76.022903, "rel_tol": 1e-5},
        "n2": {"Z": [7, 7], "R": [[-1.03, 0, 0], [1.04, 0, 0]], "energy": -108.94524, "rel_tol": 1e-4},
    }
    with open(os.path.join(HERE, "anchors.json"), "w") as f:
        json.dump(anchors, f, indent=1)
    print("max relative difference, reference Boys table vs generated:", maxrel)


if __name__ == "__main__":
    sys.exit(main())
