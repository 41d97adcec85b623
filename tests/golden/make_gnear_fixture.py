"""Writes tests/golden/gnear_alpha0.1.txt from the reference's real-space Coulomb tables.

The reference tabulates G(r) = erfc(sqrt(a) r) / r^2 + 2 sqrt(a) exp(-a r^2) / (sqrt(pi) r) at
a = 0.1 in res/json_files/Gnear_table_leq2_2.txt (0.1 <= r < 2) and Gnear_table_geq2_2.txt
(2 <= r < 12); the same numbers are compiled into framework/model/ERFTable.h.  Columns: index
(FP32 exponent and top 8 mantissa bits of r), r, the interpolation step width, G(r), and the
interpolation slope.  This script keeps every third row of each file (and the last), as printed.

Run from the repository root where the reference tree is present:
    python tests/golden/make_gnear_fixture.py [reference root]
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def rows(path):
    out = []
    for ln in open(path):
        w = ln.split()
        if len(w) == 5:
            out.append(w)
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RBMD_REFERENCE_ROOT", "/root/reference")
    lines = ["# r G(r) slope  -- every third row of res/json_files/Gnear_table_{leq2,geq2}_2.txt (alpha = 0.1),",
             "# as the reference prints them; written by tests/golden/make_gnear_fixture.py"]
    for name in ("Gnear_table_leq2_2.txt", "Gnear_table_geq2_2.txt"):
        rr = rows(os.path.join(root, "res", "json_files", name))
        keep = list(range(0, len(rr), 3))
        if keep[-1] != len(rr) - 1:
            keep.append(len(rr) - 1)
        for k in keep:
            lines.append(f"{rr[k][1]} {rr[k][3]} {rr[k][4]}")
    with open(os.path.join(HERE, "gnear_alpha0.1.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"{len(lines) - 2} rows")


if __name__ == "__main__":
    main()
