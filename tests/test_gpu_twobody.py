"""GPU parity of the CN -> weights -> C6 -> two-body -> CN chain-rule path.

Calls the library through the C ABI (dftd3.interface over cffi) and compares
with the FP64 oracle on the same inputs: the FP64 form to 1e-12 relative, the
mixed form to the 1e-7 energy / 1e-7 Eh/Bohr gradient budget.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_ref as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
RTOL64 = 1.0e-12          # FP64 form: energy, relative
GTOL64 = 1.0e-12          # FP64 form: gradient/virial, relative to the largest component
ETOL_MIXED = 1.0e-7       # mixed form: energy, relative
GTOL_MIXED = 1.0e-7       # mixed form: gradient, Hartree/Bohr


def _positions(case):
    p = np.array(case["positions"], dtype=float)
    return p * O.AATOAU if case["unit"] == "angstrom" else p


def _param_obj(p):
    """The interface's parameter object of a fixture parameter dict."""
    from dftd3 import interface as I
    kind = p["damping"]
    if kind in ("rational", "mrational"):
        cls = I.RationalDampingParam if kind == "rational" else I.ModifiedRationalDampingParam
        return cls(s6=p["s6"], s8=p["s8"], s9=p["s9"], a1=p["a1"], a2=p["a2"], alp=p["alp"])
    if kind == "zero":
        return I.ZeroDampingParam(s6=p["s6"], s8=p["s8"], s9=p["s9"], rs6=p["rs6"], rs8=p["rs8"], alp=p["alp"])
    if kind == "mzero":
        return I.ModifiedZeroDampingParam(s6=p["s6"], s8=p["s8"], s9=p["s9"], rs6=p["rs6"], rs8=p["rs8"],
                                          alp=p["alp"], bet=p["bet"])
    if kind == "optimizedpower":
        return I.OptimizedPowerDampingParam(s6=p["s6"], s8=p["s8"], s9=p["s9"], a1=p["a1"], a2=p["a2"],
                                            alp=p["alp"], bet=p["bet"])
    if kind == "cso":
        return I.CSODampingParam(s6=p["s6"], s9=p["s9"], a1=p["a1"], a2=p["a2"], a3=p["a3"], a4=p["a4"],
                                 alp=p["alp"])
    return I.ZDampingParam(s6=p["s6"], s8=p["s8"], s9=p["s9"], a1=p["a1"], alp=p["alp"])


def gpu_dispersion(numbers, positions, param, lattice=None, periodic=None, grad=True, cutoff=None,
                   precision="fp64", ghost=None, partition=None, tuning=None):
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
    if tuning is not None:
        model.set_tuning(*tuning)
    return model.get_dispersion(_param_obj(param), grad=grad)


def assert_close(res, ref, rtol, gtol):
    e, er = float(res["energy"]), ref["energy"]
    assert abs(e - er) <= rtol * abs(er), (e, er, (e - er) / er)
    if "gradient" in res:
        scale = max(np.abs(ref["gradient"]).max(), 1e-300)
        err = np.abs(res["gradient"] - ref["gradient"]).max()
        assert err <= gtol * scale, (err, scale)
        vscale = max(np.abs(ref["virial"]).max(), 1e-300)
        verr = np.abs(np.ravel(res["virial"]) - np.ravel(ref["virial"])).max()
        assert verr <= gtol * vscale, (verr, vscale)


def _cases():
    out = []
    for c in json.loads((GOLDEN / "validation.json").read_text()):
        out.append((c["name"], c["numbers"], _positions(c), c["param"]))
    for c in [e for e in json.loads((GOLDEN / "python.json").read_text()) if "cases" in e]:
        for k, sub in enumerate(c["cases"]):
            out.append((f"{c['name']}[{k}]", c["numbers"], _positions(c), sub["param"]))
    return out


TWO_BODY = [c for c in _cases() if c[3]["s9"] == 0.0]


@pytest.mark.parametrize("case", TWO_BODY, ids=[c[0] for c in TWO_BODY])
def test_golden_geometries_fp64(case):
    name, numbers, pos, param = case
    ref = O.dispersion(numbers, pos, param)
    res = gpu_dispersion(numbers, pos, param)
    assert_close(res, ref, RTOL64, GTOL64)


def test_energy_only_path():
    name, numbers, pos, param = TWO_BODY[0]
    ref = O.dispersion(numbers, pos, param, grad=False)
    res = gpu_dispersion(numbers, pos, param, grad=False)
    assert set(res) == {"energy"}
    assert abs(float(res["energy"]) - ref["energy"]) <= RTOL64 * abs(ref["energy"])


def test_periodic_regression_ta():
    """The 90-atom Ta cell of test_regression.f90 (wrapped by the API)."""
    case = json.loads((GOLDEN / "unit.json").read_text())[0]
    ref = O.dispersion(case["numbers"], _positions(case), case["param"], lattice=case["lattice"],
                       periodic=case["periodic"])
    res = gpu_dispersion(case["numbers"], _positions(case), case["param"], lattice=case["lattice"],
                         periodic=case["periodic"])
    assert_close(res, ref, RTOL64, 1.0e-10)


def test_molecule100_fp64():
    from dftd3 import synthetic as S
    d = S.molecule100()
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    ref = O.dispersion(d["numbers"], d["positions"], par)
    res = gpu_dispersion(d["numbers"], d["positions"], par)
    assert_close(res, ref, RTOL64, GTOL64)


@pytest.fixture(scope="module")
def cell2000():
    from dftd3 import synthetic as S
    d = S.cell2000()
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    ref = O.dispersion(d["numbers"], d["positions"], par, lattice=d["lattice"], periodic=d["periodic"])
    return d, par, ref


def test_cell2000_fp64(cell2000):
    d, par, ref = cell2000
    res = gpu_dispersion(d["numbers"], d["positions"], par, lattice=d["lattice"], periodic=d["periodic"])
    assert_close(res, ref, RTOL64, GTOL64)


def test_cell2000_mixed(cell2000):
    d, par, ref = cell2000
    res = gpu_dispersion(d["numbers"], d["positions"], par, lattice=d["lattice"], periodic=d["periodic"],
                         precision="mixed")
    e, er = float(res["energy"]), ref["energy"]
    assert abs(e - er) <= ETOL_MIXED * abs(er), (e - er) / er
    assert np.abs(res["gradient"] - ref["gradient"]).max() <= GTOL_MIXED


def test_zero_damping_periodic_smooth():
    """Zero damping, smooth cutoffs and a small triclinic cell."""
    from dftd3 import synthetic as S
    rng = np.random.default_rng(3)
    lat = S.triclinic(14.0, 15.0, 16.0, 88.0, 92.0, 95.0)
    num = rng.choice([1, 6, 8, 17], size=60).astype(np.int32)
    pos = S.pack_cell(rng, 60, lat, 2.0)
    par = dict(damping="zero", s6=1.0, s8=1.703, s9=0.0, rs6=1.261, rs8=1.0, alp=14.0)
    cut = (30.0, 20.0, 25.0, 5.0, 4.0)
    ref = O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut)
    res = gpu_dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut)
    assert_close(res, ref, RTOL64, GTOL64)


@pytest.mark.parametrize("periodic", [[True, False, False], [True, True, False]])
def test_low_dimensional_periodicity(periodic):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(5)
    lat = np.diag([12.0, 13.0, 40.0])
    num = rng.choice([1, 6, 7], size=40).astype(np.int32)
    pos = S.pack_box(rng, 40, 0.0, 11.0, 1.9)
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    cut = (25.0, 20.0, 20.0, 0.0, 0.0)
    ref = O.dispersion(num, pos, par, lattice=lat, periodic=periodic, cutoff=cut)
    res = gpu_dispersion(num, pos, par, lattice=lat, periodic=periodic, cutoff=cut)
    assert_close(res, ref, RTOL64, GTOL64)


def test_ghost_atoms():
    name, numbers, pos, param = TWO_BODY[0]
    ghost = [0, 3, 5]
    ref = O.dispersion(numbers, pos, param, ghost=ghost)
    res = gpu_dispersion(numbers, pos, param, ghost=ghost)
    assert_close(res, ref, RTOL64, GTOL64)


def test_work_partition_sums_to_full():
    """test_interface.py:440-465: parts reproduce the complete result."""
    from dftd3 import synthetic as S
    d = S.molecule100(seed=4)
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    full = gpu_dispersion(d["numbers"], d["positions"], par)
    tot_e, tot_g, tot_s = 0.0, 0.0, 0.0
    for part in range(3):
        r = gpu_dispersion(d["numbers"], d["positions"], par, partition=(part, 3))
        ref = O.dispersion(d["numbers"], d["positions"], par, part=part, nparts=3)
        assert_close(r, ref, 1.0e-11, 1.0e-11)
        tot_e += float(r["energy"]); tot_g = tot_g + r["gradient"]; tot_s = tot_s + r["virial"]
    assert abs(tot_e - float(full["energy"])) < 1.0e-12
    assert np.abs(tot_g - full["gradient"]).max() < 1.0e-12
    assert np.abs(tot_s - full["virial"]).max() < 1.0e-12


def test_deterministic():
    from dftd3 import synthetic as S
    d = S.molecule100(seed=7)
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    a = gpu_dispersion(d["numbers"], d["positions"], par)
    b = gpu_dispersion(d["numbers"], d["positions"], par)
    assert float(a["energy"]) == float(b["energy"])
    assert np.array_equal(a["gradient"], b["gradient"])
    assert np.array_equal(a["virial"], b["virial"])


def test_batched_matches_single():
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion, RationalDampingParam
    d = S.batch4096(nmol=12, seed=2)
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    bat = BatchedDispersion(d["numbers"], d["positions"])
    res = bat.get_dispersion(RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp")}, s9=0.0),
                             grad=True)
    for k in range(12):
        ref = O.dispersion(d["numbers"][k], d["positions"][k], par)
        assert abs(res["energy"][k] - ref["energy"]) <= RTOL64 * abs(ref["energy"])
        assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max()


@pytest.fixture(scope="module")
def large_batch():
    """Six molecules and a 4500-atom cluster in one batch."""
    from dftd3 import synthetic as S
    mols = S.batch4096(nmol=6, seed=31, nmin=20, nmax=120)
    big = S.cluster5000(seed=32, natoms=4500)
    nums = list(mols["numbers"]) + [big["numbers"]]
    pos = list(mols["positions"]) + [big["positions"]]
    par = dict(S.PBE_BJ, damping="rational", s9=0.0)
    refs = [O.dispersion(n, p, par, cutoff=(40.0, 40.0, 25.0, 0.0, 0.0)) for n, p in zip(nums, pos)]
    return nums, pos, par, refs


@pytest.mark.parametrize("order", [0.0, 3.0])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spatial_orders_large_batch(large_batch, order, precision):
    """Column order (0) and Morton order (3 Bohr cells) give the oracle's results."""
    from dftd3.interface import BatchedDispersion, RationalDampingParam
    nums, pos, par, refs = large_batch
    bat = BatchedDispersion(nums, pos)
    bat.set_realspace_cutoff(40.0, 40.0, 25.0)
    bat.set_precision(precision)
    bat.set_tuning(order, 0)
    res = bat.get_dispersion(RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp")}, s9=0.0),
                             grad=True)
    for k, ref in enumerate(refs):
        if precision == "fp64":
            assert abs(res["energy"][k] - ref["energy"]) <= RTOL64 * abs(ref["energy"])
            assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max()
        else:
            assert abs(res["energy"][k] - ref["energy"]) <= ETOL_MIXED * abs(ref["energy"])
            assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL_MIXED


def test_spatial_orders_agree():
    """Column order and Morton orders reproduce each other on a molecule
    batch and on the periodic 2000-atom cell (FP64)."""
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion, RationalDampingParam
    param = RationalDampingParam(**S.PBE_BJ, s9=0.0)
    d = S.batch4096(nmol=40, seed=33)
    c = S.cell2000(natoms=600)
    for nums, pos, lat, per in ((d["numbers"], d["positions"], None, None),
                                ([c["numbers"]], [c["positions"]], np.asarray(c["lattice"])[None],
                                 np.asarray(c["periodic"])[None])):
        out = []
        for order in (0.0, 2.0, 4.5):
            bat = BatchedDispersion(nums, pos, lat, per)
            bat.set_tuning(order, 0)
            out.append(bat.get_dispersion(param, grad=True))
        for r in out[1:]:
            np.testing.assert_allclose(r["energy"], out[0]["energy"], rtol=1e-13, atol=0)
            for g, g0 in zip(r["gradient"], out[0]["gradient"]):
                assert np.abs(g - g0).max() <= 1e-12 * np.abs(g0).max()
