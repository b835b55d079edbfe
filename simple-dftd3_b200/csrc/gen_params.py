#!/usr/bin/env python3
"""Generate d3_params.c, the damping parameter database behind the
dftd3_load_*_damping entries, from the reference's Fortran source.

Mechanical transcription (nothing typed by hand) of src/dftd3/param.f90:
  * the method names and aliases of get_method_id (param.f90:96-299),
  * the d3_param defaults (param.f90:38-48),
  * the parameter records of get_rational_damping (param.f90:302-802),
    get_zero_damping (:805-1088), get_mrational_damping (:1091-1136),
    get_mzero_damping (:1139-1184), get_optimizedpower_damping (:1187-1244),
    get_cso_damping (:1248-1293) and get_z_damping (:1297-1326, no records).
Method names are looked up as get_method_id does: '-' removed, lower case.

Usage: python gen_params.py <reference root> > d3_params.c
"""
import re
import sys
from pathlib import Path

FAMILIES = ("rational", "zero", "mrational", "mzero", "optimizedpower", "cso", "z")
FIELDS = ("s6", "s8", "s9", "rs6", "rs8", "a1", "a2", "alp", "bet")


def joined_statements(text):
    """Fortran source with continuation lines joined and comments removed."""
    out = []
    for line in text.splitlines():
        code = line.split("!", 1)[0] if '"' not in line else line
        out.append(code.rstrip())
    src = "\n".join(out)
    src = re.sub(r"&\s*\n\s*&?", " ", src)
    return src


def parse(root: Path):
    text = (root / "src/dftd3/param.f90").read_text()
    src = joined_statements(text)
    # defaults of the record type
    m = re.search(r"type\s*::\s*d3_param(.*?)end type d3_param", src, re.S)
    defaults = {k: float(v) for k, v in re.findall(r"real\(wp\)\s*::\s*(\w+)\s*=\s*([-\d.]+)_wp", m.group(1))}
    assert set(defaults) == set(FIELDS), defaults
    # method names
    body = re.search(r"function get_method_id(.*?)end function get_method_id", src, re.S).group(1)
    aliases, ids = [], {}
    for names, ident in re.findall(r'case\(([^)]*)\);\s*id\s*=\s*(p_\w+)', body):
        if ident not in ids:
            ids[ident] = len(ids) + 1
        for name in re.findall(r'"([^"]*)"', names):
            aliases.append((name, ids[ident]))
    # parameter records
    records = {}
    for fam in FAMILIES:
        sub = re.search(r"subroutine get_%s_damping\((.*?)end subroutine get_%s_damping" % (fam, fam), src, re.S)
        assert sub, fam
        recs = []
        for cases, args in re.findall(r"case\s*\(\s*(p_[\w,\s]*?)\)\s*\n\s*param\s*=\s*d3_param\(([^)]*)\)",
                                      sub.group(1)):
            values = dict(defaults)
            for k, v in re.findall(r"(\w+)\s*=\s*([-\d.eE+]+)_wp", args):
                values[k] = float(v)
            for ident in re.findall(r"p_\w+", cases):
                recs.append((ids[ident], values))
        records[fam] = recs
    return aliases, records


def emit(aliases, records):
    out = ["/* Generated by gen_params.py from the reference parameter database",
           " * (src/dftd3/param.f90); do not edit. */",
           '#include "d3_params.h"', ""]
    out.append("const d3_method_alias d3_method_aliases[] = {")
    for name, ident in aliases:
        out.append('    {"%s", %d},' % (name, ident))
    out.append("};")
    out.append("const int d3_n_method_aliases = %d;" % len(aliases))
    out.append("")
    for fam in FAMILIES:
        out.append("/* method id, %s */" % ", ".join(FIELDS))
        out.append("const d3_param_record d3_%s_params[] = {" % fam)
        for ident, v in records[fam]:
            out.append("    {%d, {%s}}," % (ident, ", ".join(repr(v[k]) for k in FIELDS)))
        if not records[fam]:
            out.append("    {0, {0}},   /* no records; the count below is 0 */")
        out.append("};")
        out.append("const int d3_n_%s_params = %d;" % (fam, len(records[fam])))
        out.append("")
    return "\n".join(out)


if __name__ == "__main__":
    aliases, records = parse(Path(sys.argv[1]))
    print(emit(aliases, records))
