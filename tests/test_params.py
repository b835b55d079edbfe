"""Damping parameters loaded by method name (dftd3_load_rational_damping,
dftd3_load_zero_damping, dftd3_load_mrational_damping; reference api.f90:588-745
over param.f90), checked against the parameter values the golden fixtures
were transcribed with, and the reference's name normalisation and errors."""
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


@pytest.mark.parametrize("method,par", CASES, ids=[f"{m}-{p['damping']}-s9={p['s9']}" for m, p in CASES])
def test_loaded_values_match_fixtures(method, par):
    from dftd3 import library
    load = library.load_rational_damping if par["damping"] == "rational" else library.load_zero_damping
    got = library.get_param_values(load(method, par["s9"] != 0.0))
    assert got["damping"] == par["damping"]
    keys = ("s6", "s8", "s9", "a1", "a2", "alp") if par["damping"] == "rational" else \
        ("s6", "s8", "s9", "rs6", "rs8", "alp")
    for k in keys:
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
    with pytest.raises(RuntimeError, match="not supported"):
        library.load_mzero_damping("pbe", False)


def test_python_interface_by_method():
    from dftd3.interface import RationalDampingParam, ZeroDampingParam
    from dftd3 import library
    p = RationalDampingParam(method="pbe0")
    assert library.get_param_values(p._param)["a2"] == 4.8593
    z = ZeroDampingParam(method="b3lyp", atm=True)
    assert library.get_param_values(z._param)["rs6"] == 1.261
