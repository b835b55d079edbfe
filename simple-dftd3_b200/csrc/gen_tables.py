#!/usr/bin/env python3
"""Generate ``d3_tables.c``: the D3 model's per-element parameter tables.

The tables are the parameters of the D3 model itself, so they must be the
reference's values, not a re-derivation.  This script transcribes them
mechanically from the reference's Fortran data modules (the array literals are
parsed, nothing is typed by hand) and writes a C translation unit that both the
CUDA library and the CPU oracle compile:

* ``src/dftd3/reference.f90``  number_of_references (:30-45), reference_cn
  (:47-151) and the reference C6 table filled in ``copy_c6`` (:207-66221),
  indexed as ``reference_c6(iref, jref, ic)`` with ``ic = atj + ati*(ati-1)/2``
  for ``ati >= atj`` (``get_c6``, :160-171).
* ``src/dftd3/data/r4r2.f90``  r4_over_r2 (:44-67); the model uses
  ``sqrt(0.5*r4_over_r2*sqrt(Z))`` (:69-70), evaluated at load time.
* ``src/dftd3/data/vdwrad.f90`` pairwise van-der-Waals radii in Angstrom
  (:38-1111); the model multiplies them by ``aatoau``.

The D3 covalent radii used by the coordination number come from mctc-lib
(``mctc_data_covrad``, pinned at 06db4d8 by ``subprojects/mctc-lib.wrap``),
which the reference does not vendor.  They are restated here from the
published D3 radius set: the single-bond covalent radii of Pyykkoe and Atsumi
(Chem. Eur. J. 15, 186 (2009)) with the values for metals reduced by 10 %, as
used by Grimme et al., J. Chem. Phys. 132, 154104 (2010); the D3 counting
function scales them by 4/3.  The golden-vector tests pin every element that
occurs in the reference's own fixtures.

All literals are written out with the decimal digits of the source, so the C
compiler rounds them exactly as the Fortran compiler did.

Usage: python gen_tables.py REFERENCE_ROOT > d3_tables.c
"""
import re
import sys
from pathlib import Path

# D3 covalent radii in Angstrom for Z = 1..118 (see module docstring).
RCOV_ANGSTROM = [
    0.32, 0.46, 1.20, 0.94, 0.77, 0.75, 0.71, 0.63, 0.64, 0.67,
    1.40, 1.25, 1.13, 1.04, 1.10, 1.02, 0.99, 0.96, 1.76, 1.54,
    1.33, 1.22, 1.21, 1.10, 1.07, 1.04, 1.00, 0.99, 1.01, 1.09,
    1.12, 1.09, 1.15, 1.10, 1.14, 1.17, 1.89, 1.67, 1.47, 1.39,
    1.32, 1.24, 1.15, 1.13, 1.13, 1.08, 1.15, 1.23, 1.28, 1.26,
    1.26, 1.23, 1.32, 1.31, 2.09, 1.76, 1.62, 1.47, 1.58, 1.57,
    1.56, 1.55, 1.51, 1.52, 1.51, 1.50, 1.49, 1.49, 1.48, 1.53,
    1.46, 1.37, 1.31, 1.23, 1.18, 1.16, 1.11, 1.12, 1.13, 1.32,
    1.30, 1.30, 1.36, 1.31, 1.38, 1.42, 2.01, 1.81, 1.67, 1.58,
    1.52, 1.53, 1.54, 1.55, 1.49, 1.49, 1.51, 1.51, 1.48, 1.50,
    1.56, 1.58, 1.45, 1.41, 1.34, 1.29, 1.27, 1.21, 1.16, 1.15,
    1.09, 1.22, 1.36, 1.43, 1.46, 1.58, 1.48, 1.57,
]

NUM = r"([-+]?\d+\.\d*(?:[eEdD][-+]?\d+)?)_wp"


def literals(text):
    return [s.replace("d", "e").replace("D", "e") for s in re.findall(NUM, text)]


def parse_reference(root):
    src = (root / "src/dftd3/reference.f90").read_text()
    m = re.search(r"number_of_references\(max_elem\)\s*=\s*\[(.*?)\]", src, re.S)
    body = re.sub(r"!.*", "", m.group(1))
    nref = [int(x) for x in re.findall(r"\d+", body.replace("&", " "))]
    assert len(nref) == 103, len(nref)
    m = re.search(r"reference_cn\(max_ref, max_elem\)\s*=\s*reshape\(\[(.*?)\],", src, re.S)
    refcn = literals(m.group(1))
    assert len(refcn) == 7 * 103, len(refcn)
    c6 = [None] * (7 * 7 * 5356)
    for a, b, body in re.findall(r"c6ab_view\((\d+):(\d+)\)\s*=\s*\[(.*?)\]", src, re.S):
        vals = literals(body)
        lo, hi = int(a), int(b)
        assert len(vals) == hi - lo + 1
        c6[lo - 1:hi] = vals
    assert all(v is not None for v in c6)
    return nref, refcn, c6


def parse_r4r2(root):
    src = (root / "src/dftd3/data/r4r2.f90").read_text()
    m = re.search(r"r4_over_r2\(max_elem\)\s*=\s*\[(.*?)\]", src, re.S)
    vals = literals(m.group(1))
    assert len(vals) == 118, len(vals)
    return vals


def parse_vdwrad(root):
    src = (root / "src/dftd3/data/vdwrad.f90").read_text()
    m = re.search(r"vdwrad\(max_elem\*\(1\+max_elem\)/2\)\s*=\s*aatoau\s*\*\s*\[(.*?)\]", src, re.S)
    vals = literals(m.group(1))
    assert len(vals) == 103 * 104 // 2, len(vals)
    return vals


def emit_array(out, ctype, name, vals, per_line=8):
    out.append(f"const {ctype} {name}[{len(vals)}] = {{")
    for k in range(0, len(vals), per_line):
        out.append("  " + ", ".join(vals[k:k + per_line]) + ",")
    out.append("};")


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python gen_tables.py <reference root>")
    root = Path(sys.argv[1])
    nref, refcn, c6 = parse_reference(root)
    r4r2 = parse_r4r2(root)
    vdw = parse_vdwrad(root)
    assert len(RCOV_ANGSTROM) == 118
    # zeros are written compactly; every other literal keeps its source digits
    c6 = ["0" if float(v) == 0.0 else v for v in c6]
    out = [
        "/* Generated by gen_tables.py from the reference's Fortran data modules.",
        " * Do not edit: regenerate instead.  Layouts (0-based):",
        " *   d3_nref[Z-1], d3_refcn[(Z-1)*7 + iref]",
        " *   d3_c6ab[ic*49 + jref*7 + iref] with ic = atj + ati*(ati+1)/2, ati >= atj",
        " *   d3_vdwrad_aa[ic] (Angstrom), same pair index",
        " *   d3_r4_over_r2[Z-1], d3_rcov_aa[Z-1] (Angstrom) */",
        '#include "d3_tables.h"',
        "",
    ]
    emit_array(out, "unsigned char", "d3_nref", [str(v) for v in nref], 20)
    emit_array(out, "double", "d3_refcn", refcn, 7)
    emit_array(out, "double", "d3_r4_over_r2", r4r2, 8)
    emit_array(out, "double", "d3_rcov_aa", [f"{v:.2f}" for v in RCOV_ANGSTROM], 10)
    emit_array(out, "double", "d3_vdwrad_aa", vdw, 8)
    emit_array(out, "double", "d3_c6ab", c6, 7)
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
