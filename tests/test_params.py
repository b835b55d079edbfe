"""Damping parameters loaded by method name (dftd3_load_*_damping; reference
api.f90:588-1018 over param.f90), checked against the parameter values the
golden fixtures were transcribed with, and the reference's name
normalisation and errors."""
import json
import re
from pathlib import Path

import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _fixture_params():
    out = []
    for fname in ("validation.json", "python.json"):
        data = json.loads((GOLDEN / fname).read_text())
        for entry in data:
            for case in entry.get("cases", [entry]):
                par = case.get("param")
                if not par:
                    continue
                m = re.search(r"\((\w+)\)", par.get("source", ""))
                if m:
                    out.append((m.group(1), par))
    return out


CASES = _fixture_params()


def test_fixtures_name_methods():
    assert len({m for m, _ in CASES}) >= 5


# the values each family's evaluation reads
FAMILY_KEYS = {"rational": ("s6", "s8", "s9", "a1", "a2", "alp"),
               "mrational": ("s6", "s8", "s9", "a1", "a2", "alp"),
               "zero": ("s6", "s8", "s9", "rs6", "rs8", "alp"),
               "mzero": ("s6", "s8", "s9", "rs6", "rs8", "alp", "bet"),
               "optimizedpower": ("s6", "s8", "s9", "a1", "a2", "alp", "bet")}


@pytest.mark.parametrize("method,par", CASES, ids=[f"{m}-{p['damping']}-s9={p['s9']}" for m, p in CASES])
def test_loaded_values_match_fixtures(method, par):
    from dftd3 import library
    load = getattr(library, f"load_{par['damping']}_damping")
    got = library.get_param_values(load(method, par["s9"] != 0.0))
    assert got["damping"] == {"mrational": "rational"}.get(par["damping"], par["damping"])
    for k in FAMILY_KEYS[par["damping"]]:
        assert got[k] == pytest.approx(par.get(k, {"rs8": 1.0}.get(k)), abs=0, rel=1e-15), k


def test_name_normalisation():
    from dftd3 import library
    ref = library.get_param_values(library.load_rational_damping("b3lyp", False))
    for name in ("B3LYP", "b3-lyp", "B3-LYP", "b3lyp5"):
        assert library.get_param_values(library.load_rational_damping(name, False)) == ref


def test_atm_flag_sets_s9():
    from dftd3 import library
    assert library.get_param_values(library.load_rational_damping("pbe", True))["s9"] == 1.0
    assert library.get_param_values(library.load_rational_damping("pbe", False))["s9"] == 0.0
    assert library.get_param_values(library.load_zero_damping("pbe", True))["s9"] == 1.0


def test_unknown_method_and_family():
    from dftd3 import library
    with pytest.raises(RuntimeError, match="No entry for 'not-a-functional' present"):
        library.load_rational_damping("not-a-functional", False)
    assert library.get_param_values(library.load_mrational_damping("pbe", False))["damping"] == "rational"
    # get_z_damping holds no records (param.f90:1297-1326)
    with pytest.raises(RuntimeError, match="No entry for 'pbe' present"):
        library.load_z_damping("pbe", False)


def test_other_families_by_method():
    """Records of get_mzero_damping, get_optimizedpower_damping and
    get_cso_damping (param.f90:1139-1293) as the loaders return them."""
    from dftd3 import library
    m = library.get_param_values(library.load_mzero_damping("b3lyp", True))
    assert (m["damping"], m["rs6"], m["s8"], m["bet"], m["s9"]) == ("mzero", 1.338153, 1.532981, 0.013988, 1.0)
    o = library.get_param_values(library.load_optimizedpower_damping("tpssh", False))
    assert (o["damping"], o["s8"], o["a1"], o["a2"], o["bet"]) == ("optimizedpower", 0.43185, 0.575, 3.0, 8.0)
    c = library.get_param_values(library.load_cso_damping("pw6b95", False))
    assert (c["damping"], c["a1"], c["a2"], c["rs6"], c["rs8"]) == ("cso", -0.15, 2.5, 0.0, 6.25)


def test_family_constructors():
    """dftd3_new_*_damping of every family (api.f90:748-982)."""
    from dftd3 import library
    v = library.get_param_values(library.new_mzero_damping(1.0, 0.5, 0.0, 1.2, 1.0, 14.0, 0.1))
    assert (v["damping"], v["rs6"], v["bet"]) == ("mzero", 1.2, 0.1)
    v = library.get_param_values(library.new_optimizedpower_damping(0.9, 0.0, 1.0, 0.15, 4.75, 14.0, 6.0))
    assert (v["damping"], v["a2"], v["bet"], v["s9"]) == ("optimizedpower", 4.75, 6.0, 1.0)
    v = library.get_param_values(library.new_cso_damping(1.0, 0.0, 0.86, 2.5, 0.1, 6.0, 14.0))
    assert (v["damping"], v["a1"], v["rs6"], v["rs8"]) == ("cso", 0.86, 0.1, 6.0)
    v = library.get_param_values(library.new_z_damping(1.0, 1.0, 0.0, 200770.0, 14.0))
    assert (v["damping"], v["a1"], v["a2"]) == ("z", 200770.0, 0.0)


def test_python_interface_by_method():
    from dftd3.interface import RationalDampingParam, ZeroDampingParam
    from dftd3 import library
    p = RationalDampingParam(method="pbe0")
    assert library.get_param_values(p._param)["a2"] == 4.8593
    z = ZeroDampingParam(method="b3lyp", atm=True)
    assert library.get_param_values(z._param)["rs6"] == 1.261
