"""GPU parity of the analytic Hessian (dftd3_get_dispersion_hessian,
get_dispersion_hessian in disp.f90:236-308) against the FP64 oracle, and the
reference's own check of it: symmetry and central differences of the
gradient (test_interface.py test_hessian, test_hessian_ghost_atoms)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_ref as O
from test_gpu_twobody import _param_obj, _positions

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASE = next(e for e in json.loads((GOLDEN / "python.json").read_text()) if e["name"] == "test_interface.hessian")
TOL = 1.0e-12


def _model(numbers, positions, lattice=None, periodic=None, cutoff=None, ghost=None, partition=None):
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
    return model


def assert_hessian(h, ref):
    scale = np.abs(ref).max()
    assert np.abs(h - ref).max() <= TOL * scale, (np.abs(h - ref).max(), scale)
    assert np.abs(h - h.T).max() <= TOL * scale


@pytest.mark.parametrize("ghost", [False, True])
def test_hessian_fixture(ghost):
    """The water dimer of the reference's Hessian tests: oracle parity, and
    central differences of the GPU gradient (step 1e-6, abs 1e-7)."""
    nums, pos = np.array(CASE["numbers"]), _positions(CASE)
    gh = CASE["ghost"] if ghost else None
    model = _model(nums, pos, ghost=gh)
    param = _param_obj(CASE["param"])
    res = model.get_hessian(param)
    h = np.asarray(res["hessian"])
    assert not np.isnan(h).any()
    assert_hessian(h, O.hessian(nums, pos, CASE["param"], ghost=gh))
    assert float(res["energy"]) == pytest.approx(float(model.get_dispersion(param, grad=False)["energy"]),
                                                 rel=1e-13)
    step = CASE["step"]
    num = np.zeros_like(h)
    for i in range(len(nums)):
        for c in range(3):
            p = pos.copy(); p[i, c] += step
            model.update(p)
            gr = model.get_dispersion(param, grad=True)["gradient"]
            p[i, c] -= 2 * step
            model.update(p)
            gl = model.get_dispersion(param, grad=True)["gradient"]
            num[3 * i + c] = 0.5 * (gr - gl).ravel() / step
    model.update(pos)
    assert np.abs(h - num).max() <= CASE["tol_abs"]


FAMILIES = {
    "rational": dict(damping="rational", s6=1.0, s8=1.2177, a1=0.4145, a2=4.8593, s9=1.0, alp=14.0),
    "zero": dict(damping="zero", s6=1.0, s8=1.703, rs6=1.261, rs8=1.0, s9=1.0, alp=14.0),
    "mzero": dict(damping="mzero", s6=1.0, s8=1.532981, rs6=1.338153, rs8=1.0, bet=0.013988, s9=1.0, alp=14.0),
    "optimizedpower": dict(damping="optimizedpower", s6=1.0, s8=0.43185, a1=0.575, a2=3.0, bet=8.0, s9=1.0,
                           alp=14.0),
    "cso": dict(damping="cso", s6=1.0, a1=0.24, a2=2.5, a3=0.0, a4=6.25, s9=1.0, alp=14.0),
    "z": dict(damping="z", s6=1.0, s8=1.0, a1=1.0, s9=0.0, alp=14.0),
}


@pytest.mark.parametrize("name", sorted(FAMILIES))
def test_hessian_families(name):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(7)
    nums = rng.choice([1, 6, 7, 8], size=24).astype(np.int32)
    pos = S.pack_box(rng, 24, 0.0, 9.0, 2.0)
    par = FAMILIES[name]
    h = np.asarray(_model(nums, pos).get_hessian(_param_obj(par))["hessian"])
    assert_hessian(h, O.hessian(nums, pos, par))


def test_hessian_periodic_partition():
    """A periodic cell with smooth cutoffs; parts of the work partition match
    the oracle's parts and sum to the complete Hessian."""
    from dftd3 import synthetic as S
    rng = np.random.default_rng(5)
    lat = S.triclinic(9.0, 9.5, 10.0, 88.0, 91.0, 93.0)
    nums = rng.choice([1, 6, 8], size=10).astype(np.int32)
    pos = S.pack_cell(rng, 10, lat, 2.0)
    par = FAMILIES["rational"]
    cut = (20.0, 12.0, 15.0, 3.0, 2.0)
    full = np.asarray(_model(nums, pos, lat, [True] * 3, cut).get_hessian(_param_obj(par))["hessian"])
    assert_hessian(full, O.hessian(nums, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut))
    total = np.zeros_like(full)
    for k in range(3):
        part = np.asarray(_model(nums, pos, lat, [True] * 3, cut, partition=(k, 3)).get_hessian(
            _param_obj(par))["hessian"])
        ref = O.hessian(nums, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut, part=k, nparts=3)
        assert np.abs(part - ref).max() <= TOL * np.abs(full).max()
        total += part
    assert np.abs(total - full).max() <= TOL * np.abs(full).max()

