"""Extract the L137 hybrid-coordinate table from the reference's SCM namelist.

The OpenIFS single-column test ships the 138 half-level coefficients A (Pa)
and B (dimensionless) of the operational L137 grid as namelist NAMVV1
(ifs-test/tests/scm/common/namelists:90-366, DVALH(0:137) and DVBH(0:137)).
This script copies those numbers, unchanged, into l137_ab.txt beside it, so that
the input generator can build PAPH = A + B * p_surface without the reference
tree being present.  Run it from a checkout that has the reference mounted:

    python openifs_b200/data/make_l137.py /path/to/openifs
"""
import os
import re
import sys

NUM = r"[-+]?\d+\.\d*(?:[eE][-+]?\d+)?"


def extract(namelist_text):
    i = namelist_text.index("DVALH(0)")
    j = namelist_text.index("DVBH(0)")
    k = namelist_text.index("/", j)
    a = re.findall(NUM, namelist_text[i + len("DVALH(0)"):j])
    b = re.findall(NUM, namelist_text[j + len("DVBH(0)"):k])
    if len(a) != 138 or len(b) != 138:
        raise ValueError(f"expected 138 A and B values, got {len(a)} and {len(b)}")
    return a, b


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python make_l137.py <root of the OpenIFS source tree>")
    root = sys.argv[1]
    src = os.path.join(root, "ifs-test/tests/scm/common/namelists")
    a, b = extract(open(src).read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "l137_ab.txt")
    with open(out, "w") as f:
        f.write("# L137 half-level hybrid coefficients, k = 0..137 (top to surface)\n")
        f.write("# copied from ifs-test/tests/scm/common/namelists NAMVV1 DVALH/DVBH\n")
        f.write("# k A_Pa B\n")
        for kk, (x, y) in enumerate(zip(a, b)):
            f.write(f"{kk} {x} {y}\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
