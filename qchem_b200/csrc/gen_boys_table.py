"""Generate boys_table.h: F_j(T) for T = 0.0, 0.1, ..., 12.0 (121 rows) and j = 0..22 (23 orders).

The table has the shape and spacing the reference's T < 12 branch expects
(src/BasisSet/Molecule/Evaluators/Internal/Boys/Imp/AuxillaryData.C:8-10: 121 x 23, step 0.1), but the
values are computed here from the definition F_j(T) = int_0^1 u^{2j} exp(-T u^2) du via the lower
incomplete gamma function, F_j(T) = gamma(j+1/2, T) / (2 T^{j+1/2}), at 40 significant digits with
mpmath, then rounded to double.
"""
import os
import sys

import mpmath

ROWS, COLS = 121, 23


def table():
    mpmath.mp.dps = 40
    out = []
    for it in range(ROWS):
        T = mpmath.mpf(it) / 10
        row = []
        for j in range(COLS):
            if it == 0:
                v = mpmath.mpf(1) / (2 * j + 1)
            else:
                a = j + mpmath.mpf(1) / 2
                v = mpmath.gammainc(a, 0, T) / (2 * T ** a)
            row.append(float(v))
        out.append(row)
    return out


def main(path):
    t = table()
    lines = ["// generated by gen_boys_table.py -- Boys function F_j(T), T = 0.1*i (i=0..120), j = 0..22",
             "#pragma once", "static const double kBoysTable[121 * 23] = {"]
    for row in t:
        lines.append("    " + ", ".join("%.17g" % v for v in row) + ",")
    lines.append("};")
    text = "\n".join(lines) + "\n"
    with open(path, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "boys_table.h"))
