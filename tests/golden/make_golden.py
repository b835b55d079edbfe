#!/usr/bin/env python3
"""Extract golden vectors from the reference's own test files.

Reads the reference source tree (its root given on the command line) as text and writes
small JSON fixtures next to this script.  Every fixture records the file it
came from, the damping parameters the reference test used (with the
parameter-table line they come from) and the tolerance the reference test
applies.  Geometries keep the units of their source files ("angstrom" or
"bohr"); the tests convert Angstrom with the same Bohr radius the reference
readers use.

Run it only where the reference is present:
    python tests/golden/make_golden.py REFERENCE_ROOT
"""
import ast
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu "
    "Zn Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba "
    "La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb "
    "Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr"
).split()


def znum(sym):
    sym = sym.strip()
    return SYMBOLS.index(sym[0].upper() + sym[1:].lower()) + 1


def read_xyz(path):
    lines = path.read_text().splitlines()
    nat = int(lines[0].split()[0])
    nums, xyz = [], []
    for ln in lines[2:2 + nat]:
        p = ln.split()
        nums.append(znum(p[0]))
        xyz.append([float(x) for x in p[1:4]])
    return nums, xyz, "angstrom"


def read_gen(path):
    lines = [ln for ln in path.read_text().splitlines() if ln.strip()]
    nat, kind = lines[0].split()[:2]
    assert kind.upper() == "C", "only cluster gen files are used"
    species = lines[1].split()
    nums, xyz = [], []
    for ln in lines[2:2 + int(nat)]:
        p = ln.split()
        nums.append(znum(species[int(p[1]) - 1]))
        xyz.append([float(x) for x in p[2:5]])
    return nums, xyz, "angstrom"


def read_tmol(path):
    nums, xyz, on = [], [], False
    for ln in path.read_text().splitlines():
        if ln.startswith("$coord"):
            on = True
            continue
        if ln.startswith("$"):
            on = False
            continue
        if on and ln.strip():
            p = ln.split()
            xyz.append([float(x) for x in p[:3]])
            nums.append(znum(p[3]))
    return nums, xyz, "bohr"


def read_molfile(path):
    lines = path.read_text().splitlines()
    nat = int(lines[3][:3])
    nums, xyz = [], []
    for ln in lines[4:4 + nat]:
        p = ln.split()
        xyz.append([float(x) for x in p[:3]])
        nums.append(znum(p[3]))
    return nums, xyz, "angstrom"


def read_pdb(path):
    """ATOM/HETATM records: coordinates in columns 31-54, element in 77-78."""
    nums, xyz = [], []
    for ln in path.read_text().splitlines():
        if ln.startswith(("ATOM", "HETATM")):
            xyz.append([float(ln[30:38]), float(ln[38:46]), float(ln[46:54])])
            nums.append(znum(ln[76:78].strip() or ln[12:16].strip()))
    return nums, xyz, "angstrom"


# 10-gradient-d3-op reads its .log file with `--input xyz`
READERS = {".xyz": read_xyz, ".gen": read_gen, ".tmol": read_tmol,
           ".coord": read_tmol, ".sdf": read_molfile, ".mol": read_molfile,
           ".pdb": read_pdb, ".log": read_xyz}

PARAM_DEFAULTS = {"rational": dict(s6=1.0, s8=1.0, s9=0.0, a1=0.4, a2=5.0, alp=14.0),
                  "zero": dict(s6=1.0, s8=1.0, s9=0.0, rs6=1.0, rs8=1.0, alp=14.0)}
PARAM_DEFAULTS["mrational"] = PARAM_DEFAULTS["rational"]
PARAM_DEFAULTS["mzero"] = dict(PARAM_DEFAULTS["zero"], bet=0.0)
PARAM_DEFAULTS["optimizedpower"] = dict(PARAM_DEFAULTS["rational"], bet=0.0)
PARAM_DEFAULTS["z"] = dict(s6=1.0, s8=1.0, s9=0.0, a1=0.4, alp=14.0)

_PARAM_DB = None


def param_db(root):
    """The records of src/dftd3/param.f90 as parsed for the library's
    parameter table (simple-dftd3_b200/csrc/gen_params.py)."""
    global _PARAM_DB
    if _PARAM_DB is None:
        sys.path.insert(0, str(HERE.parents[1] / "simple-dftd3_b200" / "csrc"))
        import gen_params
        aliases, records = gen_params.parse(root)
        _PARAM_DB = (dict(aliases), records, gen_params.FIELDS)
    return _PARAM_DB


def param_f90(root, family, method, atm, **extra):
    """get_<family>_damping(method) with s9 = 1 when atm (param.f90)."""
    names, records, fields = param_db(root)
    ident = names[method.replace("-", "").lower()]
    values = next(v for i, v in records[family] if i == ident)
    p = {k: values[k] for k in fields}
    if atm:
        p["s9"] = 1.0
    p.update(extra)
    p["damping"] = family
    p["source"] = f"param.f90 get_{family}_damping ({method}){' + atm' if atm else ''}"
    return p


def param_toml(root, method, key):
    """A record of assets/parameters.toml over its [default.parameter]
    record and the d3_param defaults, as app/toml.f90:138-240 merges them."""
    import tomllib
    db = tomllib.loads((root / "assets/parameters.toml").read_text())
    _, _, fields = param_db(root)
    p = dict(s6=1.0, s8=1.0, s9=0.0, rs6=1.0, rs8=1.0, a1=0.4, a2=5.0, alp=14.0, bet=0.0)
    p.update(db["default"]["parameter"]["d3"][key])
    p.update(db["parameter"][method]["d3"][key])
    p.pop("doi", None)
    family = {"rational": "rational", "zero": "zero", "mzero": "mzero",
              "optimizedpower": "optimizedpower", "cso": "cso"}[p.pop("damping")]
    p = {k: float(p[k]) for k in fields}
    p["damping"] = family
    p["source"] = f"assets/parameters.toml [parameter.{method}] d3.{key} over [default.parameter]"
    return p


def param(damping, source, **kw):
    """d3_param defaults (src/dftd3/param.f90:38-48) overridden by kw."""
    p = dict(PARAM_DEFAULTS[damping])
    p.update(kw)
    p["damping"] = damping
    p["source"] = source
    return p


# Validation fixtures: (name, geometry file, damping parameters).  The
# parameters are those the CLI arguments in the matching .resp select.
VALIDATION = [
    ("01-energy-d3-bj", "01-tyr-xab.xyz",
     param("rational", "param.f90:343-345 (pbe) + --atm", a1=0.4289, s8=0.7875, a2=4.4407, s9=1.0)),
    ("02-energy-d3-zero", "02-ser-xad.gen",
     param("zero", "param.f90 get_zero_damping (b3lyp)", rs6=1.261, s8=1.703)),
    ("06-gradient-d3-bj", "06-229.xyz",
     param("rational", "param.f90:391-392 (olyp)", a1=0.5299, s8=2.6205, a2=2.8065)),
    ("07-gradient-d3-zero", "07-bih3-nh3.tmol",
     param("zero", "param.f90 get_zero_damping (m06l) + --atm", rs6=1.581, s8=0.0, s9=1.0)),
    ("11-pairwise-d3-bj", "11-cf3br-benzene.xyz",
     param("rational", "--bj-param 1.0 2.9491 0.4466 6.1742", s6=1.0, s8=2.9491, a1=0.4466, a2=6.1742)),
    ("12-pairwise-d3-zero", "12-butane.gen",
     param("zero", "--zero-param 1.0 1.764 0.806 --atm", s6=1.0, s8=1.764, rs6=0.806, s9=1.0)),
    ("16-db-d3-bj", "16-i10e.gen",
     param("rational", "fixture damping parameters (b1lyp from assets/parameters.toml)",
           s6=1.0, s8=2.1167, s9=1.0, a1=0.1986, a2=5.3875, alp=14.0)),
    ("17-db-d3-zero", "17-li2-ch4.sdf",
     param("zero", "assets/parameters.toml:5-6,418-419 (pkzb, table default s9=1)",
           rs6=0.6327, s8=0.0, s9=1.0, rs8=1.0)),
    # the pairwise sets 13-15 give their parameters on the command line
    # (app/cli.f90: --bjm-param s6 s8 a1 a2, --zerom-param s6 s8 rs6 bet,
    # --op-param s6 s8 a1 a2 bet, --atm-scale s9)
    ("13-pairwise-d3-bjm", "13-c60.coord",
     param("mrational", "--bjm-param 1.0 1.206988 0.240184 3.864426 --atm-scale 2.0",
           s6=1.0, s8=1.206988, a1=0.240184, a2=3.864426, s9=2.0)),
    ("14-pairwise-d3-zerom", "14-anthracene2.xyz",
     param("mzero", "--zerom-param 1.0 1.841686 1.279637 0.014370 --atm-scale 0.5",
           s6=1.0, s8=1.841686, rs6=1.279637, bet=0.014370, s9=0.5)),
    ("15-pairwise-d3-op", "15-pxylene.mol",
     param("optimizedpower", "--op-param 1.0 0.27632 0.700 2.500 8.0",
           s6=1.0, s8=0.27632, a1=0.700, a2=2.500, bet=8.0)),
]


def validation_families(root):
    """The fixtures of the modified rational, modified zero and optimized
    power families; their parameters come from the reference's tables."""
    return [
        ("03-energy-d3-bjm", "03-met-xag.coord", param_f90(root, "mrational", "b97d", False)),
        ("04-energy-d3-zerom", "04-val-xad.mol", param_f90(root, "mzero", "bp", False)),
        ("05-energy-d3-op", "05-cys-xag.sdf", param_f90(root, "optimizedpower", "tpss", False)),
        ("08-gradient-d3-bjm", "08-teh2-hbr.mol", param_f90(root, "mrational", "pbe0", False)),
        ("09-gradient-d3-zerom", "09-0a.pdb", param_f90(root, "mzero", "lcwpbe", False)),
        ("10-gradient-d3-op", "10-but14diol.log", param_f90(root, "optimizedpower", "revpbe0", False)),
        ("18-db-d3-bjm", "18-c1.pdb", param_toml(root, "blyp", "bjm")),
        ("19-db-d3-zerom", "19-g1.mol", param_toml(root, "b2plyp", "zerom")),
        ("20-db-d3-op", "20-i21p.tmol", param_toml(root, "ms2", "op")),
    ]


def validation(root):
    out = []
    vdir = root / "test/validation"
    for name, geo, par in VALIDATION + validation_families(root):
        path = vdir / geo
        nums, xyz, unit = READERS[path.suffix](path)
        ref = json.loads((vdir / f"{name}.json").read_text())
        case = {"name": name, "numbers": nums, "positions": xyz, "unit": unit,
                "param": par, "energy": ref["energy"], "tol_abs": 1.0e-6,
                "source": f"test/validation/{name}.json, tester.py:61 (abs 1e-6)"}
        if "gradient" in ref:
            case["gradient"] = ref["gradient"]
            case["virial"] = ref["virial"]
        if "additive pairwise energy" in ref:
            case["pairwise2"] = ref["additive pairwise energy"]
            case["pairwise3"] = ref["non-additive pairwise energy"]
        out.append(case)
    return out


def _np_arrays(func):
    """All list literals passed to np.array(...) inside a function body."""
    arrays = []
    for node in ast.walk(func):
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute)
                and node.func.attr == "array" and node.args):
            try:
                arrays.append(ast.literal_eval(node.args[0]))
            except ValueError:
                pass
    return arrays


def _dict_entry(func, key):
    """Literal value stored under ``key`` in the first dict display of func."""
    node = next(n for n in ast.walk(func) if isinstance(n, ast.Dict))
    for k, v in zip(node.keys, node.values):
        if isinstance(k, ast.Constant) and k.value == key:
            return ast.literal_eval(v)
    raise KeyError(key)


def python_tests(root):
    pydir = root / "python/dftd3"
    src = (pydir / "test_interface.py").read_text()
    tree = ast.parse(src)
    funcs = {f.name: f for f in tree.body if isinstance(f, ast.FunctionDef)}
    numbers, positions = _np_arrays(funcs["model"])
    # energies quoted in the tests (ref = X if atm else Y)
    def refs(fname):
        m = re.search(r"ref = (-?[\d.e-]+) if atm else (-?[\d.e-]+)", ast.get_source_segment(src, funcs[fname]))
        return float(m.group(1)), float(m.group(2))
    pbe0 = refs("test_pbe0_d3_bj")
    b3lyp = refs("test_b3lyp_d3_zero")
    cases = []
    for atm, e in ((True, pbe0[0]), (False, pbe0[1])):
        cases.append({"param": param("rational", "param.f90:364-365 (pbe0)", a1=0.4145, s8=1.2177,
                                     a2=4.8593, s9=1.0 if atm else 0.0), "energy": e})
    for atm, e in ((True, b3lyp[0]), (False, b3lyp[1])):
        cases.append({"param": param("zero", "param.f90 get_zero_damping (b3lyp)", rs6=1.261, s8=1.703,
                                     s9=1.0 if atm else 0.0), "energy": e})
    for fname, family, method in (("test_pbe_d3_bjm", "mrational", "pbe"), ("test_bp_d3_zerom", "mzero", "bp"),
                                  ("test_b97d_d3_op", "optimizedpower", "b97d")):
        e_atm, e_two = refs(fname)
        cases.append({"param": param_f90(root, family, method, True), "energy": e_atm})
        cases.append({"param": param_f90(root, family, method, False), "energy": e_two})
    # ZDampingParam(a1=200770.0, s9=...) with the constructor defaults s6 = s8 = 1, alp = 14
    e_atm, e_two = refs("test_pbe_d3_z")
    for atm, e in ((True, e_atm), (False, e_two)):
        cases.append({"param": param("z", "test_interface.py test_pbe_d3_z (interface.py ZDampingParam)",
                                     a1=200770.0, s9=1.0 if atm else 0.0), "energy": e})
    # the water dimer of test_hessian / test_hessian_ghost_atoms (analytic
    # Hessian against central differences of the gradient, step 1e-6, abs 1e-7)
    hnum, hpos = _np_arrays(funcs["test_hessian"])
    hseg = ast.get_source_segment(src, funcs["test_hessian_ghost_atoms"])
    hghost = ast.literal_eval(re.search(r"set_ghost_atoms\((\[[^\]]*\])\)", hseg).group(1))
    hessian_case = {"name": "test_interface.hessian", "numbers": hnum, "positions": hpos, "unit": "bohr",
                    "param": param_f90(root, "rational", "pbe0", True), "ghost": hghost, "step": 1.0e-6,
                    "tol_abs": 1.0e-7, "tol_sym": 1.0e-12,
                    "source": "python/dftd3/test_interface.py test_hessian, test_hessian_ghost_atoms"}
    interface = {"name": "test_interface.model", "numbers": numbers, "positions": positions,
                 "unit": "bohr", "cases": cases, "tol_rel": 1.0e-6,
                 "source": "python/dftd3/test_interface.py:77-100,231-235,322-358 (pytest.approx rel 1e-6)"}

    src = (pydir / "test_qcschema.py").read_text()
    tree = ast.parse(src)
    funcs = {f.name: f for f in tree.body if isinstance(f, ast.FunctionDef)}
    mol = {"geometry": _dict_entry(funcs["get_molecule"], "geometry")}
    seg = ast.get_source_segment(src, funcs["get_molecule"])
    m = re.search(r'"symbols": "([^"]+)"\.split\(" "\)', seg)
    nums = [znum(s) for s in m.group(1).split(" ")]
    geom = mol["geometry"]
    grads = _np_arrays(funcs["test_gradient_b97d_d3bj"])
    def qrefs(fname):
        m = re.search(r"ref = (-?[\d.e-]+) if atm else (-?[\d.e-]+)", ast.get_source_segment(src, funcs[fname]))
        return float(m.group(1)), float(m.group(2))
    r2 = qrefs("test_energy_r2scan_d3bj")
    bp = qrefs("test_energy_bp_d3zero")
    mcases = []
    for atm, e in ((True, r2[0]), (False, r2[1])):
        mcases.append({"param": param("rational", "param.f90 get_rational_damping (r2scan)", a1=0.49484001,
                                      s8=0.78981345, a2=5.73083694, s9=1.0 if atm else 0.0), "energy": e})
    for atm, e in ((True, bp[0]), (False, bp[1])):
        mcases.append({"param": param("zero", "test_qcschema.py params_tweaks (bp)", s8=1.683, rs6=1.139,
                                      s9=1.0 if atm else 0.0), "energy": e})
    for atm, g in ((True, grads[0]), (False, grads[1])):
        mcases.append({"param": param("rational", "param.f90:337-338 (b97d)", a1=0.5545, s8=2.2609,
                                      a2=3.2297, s9=1.0 if atm else 0.0), "gradient": g})
    molecule1 = {"name": "test_qcschema.molecule1", "numbers": nums, "positions": geom, "unit": "bohr",
                 "cases": mcases, "tol_abs": 1.0e-9,
                 "source": "python/dftd3/test_qcschema.py:37-57,166-427 (abs 1e-9)"}

    seg = ast.get_source_segment(src, funcs["test_gradient_tpss_d3zero"])
    mdict = {"geometry": _dict_entry(funcs["test_gradient_tpss_d3zero"], "geometry")}
    m = re.search(r'"symbols": "([^"]+)"\.split\(\)', seg)
    tnums = [znum(s) for s in m.group(1).split()]
    tgrad = _np_arrays(funcs["test_gradient_tpss_d3zero"])[0]
    tpss = {"name": "test_qcschema.tpss_d3zero", "numbers": tnums, "positions": mdict["geometry"],
            "unit": "bohr", "cases": [{"param": param("zero", "params_tweaks sr6/s8/alpha6, qcschema.py:60 s9=1",
                                                      rs6=1.166, s8=1.105, alp=14.0, s9=1.0),
                                       "gradient": tgrad}],
            "tol_abs": 1.0e-9, "source": "python/dftd3/test_qcschema.py:500-547 (abs 1e-9)"}
    return [interface, molecule1, tpss, hessian_case]


def fortran_array(body):
    return [float(x) for x in re.findall(r"([-+]?\d+\.\d*(?:[eEdD][-+]?\d+)?)_wp", body)]


def unit_tests(root):
    src = (root / "test/unit/test_regression.f90").read_text()
    syms = re.findall(r'"(\w+)"', re.search(r"sym\(nat\) = \[(.*?)\]", src, re.S).group(1))
    xyz = fortran_array(re.search(r"xyz\(3, nat\) = reshape\(\[(.*?)\]", src, re.S).group(1))
    lat = fortran_array(re.search(r"lattice\(3, 3\) = reshape\(\[(.*?)\]", src, re.S).group(1))
    e = float(re.search(r"check\(error, energy, ([-\d.E+]+)_wp", src).group(1))
    gn = float(re.search(r"check\(error, norm2\(gradient\), ([-\d.E+]+)_wp", src).group(1))
    ta = {"name": "test_regression.dftbplus_871", "numbers": [znum(s) for s in syms],
          "positions": [xyz[3 * k:3 * k + 3] for k in range(len(syms))], "unit": "bohr",
          "lattice": [lat[0:3], lat[3:6], lat[6:9]], "periodic": [True, True, True], "wrapped": False,
          "param": param("rational", "test_regression.f90:55-56", s6=1.0, s8=2.34, a1=6.30, a2=5.00,
                         s9=0.0, alp=14.0),
          "energy": e, "gradient_norm": gn, "tol_abs": 100 * 2.220446049250313e-16,
          "source": "test/unit/test_regression.f90:49-75,87-196 (thr 100*eps)"}

    src = (root / "test/unit/test_model.f90").read_text()
    seg = re.search(r"subroutine test_gw_amf3.*?end subroutine test_gw_amf3", src, re.S).group(0)
    ref = fortran_array(re.search(r"ref\(6, 4\) = reshape\(\[(.*?)\]", seg, re.S).group(1))
    ids = [int(x) for x in re.search(r"mol%id = \[(.*?)\]", seg).group(1).split(",")]
    num = [int(x) for x in re.search(r"mol%num = \[(.*?)\]", seg).group(1).split(",")]
    xyz = fortran_array(re.search(r"mol%xyz = reshape\(\[(.*?)\]", seg, re.S).group(1))
    amf3 = {"name": "test_model.gw_amf3", "numbers": [num[i - 1] for i in ids],
            "positions": [xyz[3 * k:3 * k + 3] for k in range(len(ids))], "unit": "bohr",
            "cn_cutoff": 30.0, "weights": [ref[6 * k:6 * k + 6] for k in range(len(ids))],
            "tol_abs": 100 * 2.220446049250313e-16,
            "source": "test/unit/test_model.f90:62-87,279-310 (thr 100*eps)"}
    return [ta, amf3]


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python make_golden.py <reference root>")
    root = Path(sys.argv[1])
    fixtures = {"validation": validation(root), "python": python_tests(root), "unit": unit_tests(root)}
    for key, cases in fixtures.items():
        (HERE / f"{key}.json").write_text(json.dumps(cases, indent=1) + "\n")
        print(f"{key}.json: {len(cases)} fixtures")


if __name__ == "__main__":
    main()
