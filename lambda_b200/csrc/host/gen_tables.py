"""Regenerates the two data tables the render loop needs, from the reference tree.

  - CIE 1931 2-degree colour-matching functions, 1 nm steps 360..830 nm (471 x 3):
    the standard observer data the reference integrates spectra against
    (src/core/constants.h:30, used by xyz31 in src/core/utils.h:195-203).
  - The 256-entry improved-noise permutation (Perlin 2002) the reference's Perlin
    texture hashes with (src/core/constants.h:28, utils.h:98).

Both are published data and must hold the same values for results to match.
Output: tables.inc (C++ arrays) and ../../_tables.py (the permutation, for the
scene generator). Run once: python gen_tables.py <reference>/src/core/constants.h
(or set LAMBDA_REF_SRC to the reference's src/ directory).
"""
import os
import re
import sys

if len(sys.argv) > 1:
    path = sys.argv[1]
elif os.environ.get("LAMBDA_REF_SRC"):
    path = os.path.join(os.environ["LAMBDA_REF_SRC"], "core", "constants.h")
else:
    sys.exit("usage: python gen_tables.py <reference>/src/core/constants.h (or set LAMBDA_REF_SRC)")
src = open(path).read()

perm_txt = re.search(r"h_PERMUTATION\[\]\s*=\s*\{([^}]*)\}", src).group(1)
perm = [int(x) for x in perm_txt.replace("\n", " ").split(",") if x.strip()]
assert len(perm) == 256 and sorted(perm) == list(range(256))

cie_txt = re.search(r"h_CIE_XYZ_1931\[\]\[3\]\s*=\s*\{(.*?)\};", src, re.S).group(1)
rows = re.findall(r"\{([^}]*)\}", cie_txt)
cie = [[float(x) for x in r.split(",")] for r in rows]
assert len(cie) == 471 and all(len(r) == 3 for r in cie)

here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "tables.inc"), "w") as f:
    f.write("// Generated by gen_tables.py. CIE 1931 2-degree observer (x, y, z) at 1 nm from 360 nm,\n")
    f.write("// and the improved-noise permutation. Published data; values must not change.\n")
    f.write("static const double kCieXyz1931[471][3] = {\n")
    for r in cie:
        f.write("    {" + ", ".join(repr(x) for x in r) + "},\n")
    f.write("};\n")
    f.write("static const int kPerlinPermutation[256] = {\n")
    for i in range(0, 256, 16):
        f.write("    " + ", ".join(str(x) for x in perm[i:i + 16]) + ",\n")
    f.write("};\n")
with open(os.path.join(here, "..", "..", "_tables.py"), "w") as f:
    f.write('"""Generated by csrc/host/gen_tables.py: the improved-noise permutation (Perlin 2002)."""\n\n')
    f.write("PERLIN_PERMUTATION = (\n")
    for i in range(0, 256, 16):
        f.write("    " + ", ".join(str(x) for x in perm[i:i + 16]) + ",\n")
    f.write(")\n")
print("ok", len(perm), len(cie))
