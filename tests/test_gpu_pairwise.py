"""GPU parity of the pairwise decomposition (dftd3_get_pairwise_dispersion,
get_pairwise_dispersion_v2 in disp.f90:403-457) against the FP64 oracle and
the reference's pairwise validation sets 11-15.

The pair matrices are FP64 in every precision setting; entries are compared
to 1e-12 of the largest entry, and the matrices must sum to the energy of
dftd3_get_dispersion."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_ref as O
from test_gpu_twobody import _param_obj, _positions

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1.0e-12
PAIRWISE = [c for c in json.loads((GOLDEN / "validation.json").read_text()) if "pairwise2" in c]


def gpu_pairwise(numbers, positions, param, lattice=None, periodic=None, cutoff=None, ghost=None,
                 precision="fp64", partition=None):
    from dftd3.interface import DispersionModel
    model = DispersionModel(np.asarray(numbers), np.asarray(positions, dtype=float),
                            None if lattice is None else np.asarray(lattice, dtype=float),
                            None if periodic is None else np.asarray(periodic, dtype=bool))
    if cutoff is not None:
        model.set_realspace_cutoff(*cutoff)
    if ghost is not None:
        model.set_ghost_atoms(ghost)
    if partition is not None:
        model.set_work_partition(*partition)
    model.set_precision(precision)
    pw = model.get_pairwise_dispersion(_param_obj(param))
    energy = float(model.get_dispersion(_param_obj(param), grad=False)["energy"])
    return pw, energy


def assert_pairs(pw, ref):
    for key in ("additive pairwise energy", "non-additive pairwise energy"):
        got, want = np.asarray(pw[key]), np.asarray(ref[key])
        scale = max(np.abs(want).max(), 1e-300)
        assert np.abs(got - want).max() <= TOL * scale, (key, np.abs(got - want).max(), scale)


def assert_sums_to(pw, energy):
    total = pw["additive pairwise energy"].sum() + pw["non-additive pairwise energy"].sum()
    assert abs(total - energy) <= 1e-11 * abs(energy), (total, energy)


@pytest.mark.parametrize("case", PAIRWISE, ids=[c["name"] for c in PAIRWISE])
def test_pairwise_fixtures(case):
    """test/validation/1[1-5]-pairwise-*: oracle parity and the fixture's
    matrices at its tolerance (abs 1e-6, tester.py:61)."""
    pos = _positions(case)
    n = len(case["numbers"])
    pw, energy = gpu_pairwise(case["numbers"], pos, case["param"])
    assert_pairs(pw, O.pairwise_dispersion(case["numbers"], pos, case["param"]))
    np.testing.assert_allclose(pw["additive pairwise energy"], np.reshape(case["pairwise2"], (n, n)), rtol=0,
                               atol=case["tol_abs"])
    np.testing.assert_allclose(pw["non-additive pairwise energy"], np.reshape(case["pairwise3"], (n, n)), rtol=0,
                               atol=case["tol_abs"])
    assert_sums_to(pw, energy)


FAMILIES = {
    "rational": dict(damping="rational", s6=1.0, s8=1.2177, a1=0.4145, a2=4.8593, s9=1.0, alp=14.0),
    "zero": dict(damping="zero", s6=1.0, s8=1.703, rs6=1.261, rs8=1.0, s9=1.0, alp=14.0),
    "mzero": dict(damping="mzero", s6=1.0, s8=1.532981, rs6=1.338153, rs8=1.0, bet=0.013988, s9=1.0, alp=14.0),
    "optimizedpower": dict(damping="optimizedpower", s6=1.0, s8=0.43185, a1=0.575, a2=3.0, bet=8.0, s9=1.0,
                           alp=14.0),
    "cso": dict(damping="cso", s6=1.0, a1=0.86, a2=2.5, a3=0.0, a4=6.25, s9=1.0, alp=14.0),
    "z": dict(damping="z", s6=1.0, s8=1.0, a1=200770.0, s9=1.0, alp=14.0),
}


@pytest.mark.parametrize("name", sorted(FAMILIES))
def test_pairwise_families_molecule(name):
    from dftd3 import synthetic as S
    d = S.molecule100(seed=21)
    par = FAMILIES[name]
    cut = (50.0, 25.0, 40.0, 0.0, 0.0)
    pw, energy = gpu_pairwise(d["numbers"], d["positions"], par, cutoff=cut)
    assert_pairs(pw, O.pairwise_dispersion(d["numbers"], d["positions"], par, cutoff=cut))
    assert_sums_to(pw, energy)


@pytest.mark.parametrize("name", ["rational", "zero"])
def test_pairwise_periodic_smooth(name):
    """A small triclinic cell with smooth cutoffs: self-image pairs on the
    diagonal and image triples."""
    from dftd3 import synthetic as S
    rng = np.random.default_rng(9)
    lat = S.triclinic(11.0, 11.5, 12.0, 87.0, 92.0, 94.0)
    num = rng.choice([1, 6, 8], size=24).astype(np.int32)
    pos = S.pack_cell(rng, 24, lat, 2.0)
    par = FAMILIES[name]
    cut = (25.0, 12.0, 20.0, 4.0, 3.0)
    pw, energy = gpu_pairwise(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut)
    assert_pairs(pw, O.pairwise_dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut))
    assert_sums_to(pw, energy)
    assert np.any(np.diag(pw["additive pairwise energy"]) != 0.0)


def test_pairwise_ghosts_partition_precision():
    """Ghost atoms give zero rows; the work partition and the mixed form of
    the model leave the FP64 pair matrices of the whole system unchanged."""
    from dftd3 import synthetic as S
    d = S.molecule100(seed=22)
    par = FAMILIES["rational"]
    ghost = [1, 4, 9]
    ref = O.pairwise_dispersion(d["numbers"], d["positions"], par, ghost=ghost)
    pw, _ = gpu_pairwise(d["numbers"], d["positions"], par, ghost=ghost)
    assert_pairs(pw, ref)
    assert not np.any(pw["additive pairwise energy"][ghost])
    full = O.pairwise_dispersion(d["numbers"], d["positions"], par)
    pw_part, _ = gpu_pairwise(d["numbers"], d["positions"], par, partition=(1, 3), precision="mixed")
    assert_pairs(pw_part, full)
