"""GPU parity of the Axilrod-Teller-Muto three-body term (with the two-body
sum and the CN chain rule it feeds), through the C ABI, against the FP64
oracle: the FP64 form to 1e-12 relative, the mixed form to 1e-7."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_ref as O
from test_gpu_twobody import (GOLDEN, GTOL64, GTOL_MIXED, ETOL_MIXED, RTOL64, _cases, _positions,
                              assert_close, gpu_dispersion)

pytestmark = pytest.mark.gpu

THREE_BODY = [c for c in _cases() if c[3]["s9"] != 0.0]


@pytest.mark.parametrize("case", THREE_BODY, ids=[c[0] for c in THREE_BODY])
def test_golden_geometries_atm_fp64(case):
    name, numbers, pos, param = case
    ref = O.dispersion(numbers, pos, param)
    res = gpu_dispersion(numbers, pos, param)
    assert_close(res, ref, RTOL64, GTOL64)


def test_atm_energy_only():
    name, numbers, pos, param = THREE_BODY[0]
    ref = O.dispersion(numbers, pos, param, grad=False)
    res = gpu_dispersion(numbers, pos, param, grad=False)
    assert abs(float(res["energy"]) - ref["energy"]) <= RTOL64 * abs(ref["energy"])


@pytest.fixture(scope="module")
def cluster():
    from dftd3 import synthetic as S
    d = S.cluster5000(seed=3, natoms=700)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    ref = O.dispersion(d["numbers"], d["positions"], par)
    return d, par, ref


def test_cluster_atm_fp64(cluster):
    d, par, ref = cluster
    res = gpu_dispersion(d["numbers"], d["positions"], par)
    assert_close(res, ref, RTOL64, GTOL64)


def test_cluster_atm_mixed(cluster):
    d, par, ref = cluster
    res = gpu_dispersion(d["numbers"], d["positions"], par, precision="mixed")
    e, er = float(res["energy"]), ref["energy"]
    assert abs(e - er) <= ETOL_MIXED * abs(er), (e - er) / er
    assert np.abs(res["gradient"] - ref["gradient"]).max() <= GTOL_MIXED


@pytest.mark.parametrize("damping", ["rational", "zero"])
def test_periodic_atm(damping):
    """ATM under 3D periodicity: self images and repeated atoms (triple_scale)."""
    from dftd3 import synthetic as S
    rng = np.random.default_rng(9)
    lat = S.triclinic(9.5, 10.0, 10.5, 87.0, 91.0, 94.0)
    num = rng.choice([1, 6, 8], size=24).astype(np.int32)
    pos = S.pack_cell(rng, 24, lat, 2.0)
    if damping == "rational":
        par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    else:
        par = dict(damping="zero", s6=1.0, s8=1.703, s9=1.0, rs6=1.261, rs8=1.0, alp=14.0)
    cut = (25.0, 14.0, 20.0, 0.0, 0.0)
    ref = O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut)
    res = gpu_dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=cut)
    assert_close(res, ref, RTOL64, GTOL64)


def test_atm_smooth_cutoff_and_ghosts():
    from dftd3 import synthetic as S
    d = S.molecule100(seed=5)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    cut = (30.0, 12.0, 25.0, 4.0, 3.0)
    ghost = [1, 7, 33]
    ref = O.dispersion(d["numbers"], d["positions"], par, cutoff=cut, ghost=ghost)
    res = gpu_dispersion(d["numbers"], d["positions"], par, cutoff=cut, ghost=ghost)
    assert_close(res, ref, RTOL64, GTOL64)


def test_atm_work_partition():
    from dftd3 import synthetic as S
    d = S.molecule100(seed=6)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    full = gpu_dispersion(d["numbers"], d["positions"], par)
    tot_e, tot_g = 0.0, 0.0
    for part in range(3):
        r = gpu_dispersion(d["numbers"], d["positions"], par, partition=(part, 3))
        ref = O.dispersion(d["numbers"], d["positions"], par, part=part, nparts=3)
        assert_close(r, ref, 1.0e-11, 1.0e-11)
        tot_e += float(r["energy"]); tot_g = tot_g + r["gradient"]
    assert abs(tot_e - float(full["energy"])) < 1.0e-12
    assert np.abs(tot_g - full["gradient"]).max() < 1.0e-12


def test_batched_atm_matches_single():
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion, RationalDampingParam
    d = S.batch4096(nmol=16, seed=4)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    bat = BatchedDispersion(d["numbers"], d["positions"])
    res = bat.get_dispersion(RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp", "s9")}),
                             grad=True)
    for k in range(16):
        ref = O.dispersion(d["numbers"][k], d["positions"][k], par)
        assert abs(res["energy"][k] - ref["energy"]) <= RTOL64 * abs(ref["energy"])
        assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max()


def test_named_methods_reproduce_fixtures():
    """Parameters loaded by method name, as the reference's Python tests do
    (RationalDampingParam(method="pbe0"), test_interface.py), give the
    fixture energies at the fixtures' tolerance and exactly the energies of
    the same parameters given explicitly."""
    import re
    from dftd3 import interface as I
    classes = {"rational": I.RationalDampingParam, "zero": I.ZeroDampingParam,
               "mrational": I.ModifiedRationalDampingParam, "mzero": I.ModifiedZeroDampingParam,
               "optimizedpower": I.OptimizedPowerDampingParam}
    entry = json.loads((GOLDEN / "python.json").read_text())[0]
    model = I.DispersionModel(np.array(entry["numbers"]), np.array(entry["positions"]))
    checked = 0
    for case in entry["cases"]:
        par = case["param"]
        m = re.search(r"\((\w+)\)", par["source"])
        if not m:          # given by value (the Z damping case)
            continue
        cls = classes[par["damping"]]
        by_name = model.get_dispersion(cls(method=m.group(1), atm=par["s9"] != 0.0), grad=False)["energy"]
        explicit = gpu_dispersion(entry["numbers"], entry["positions"], par, grad=False)["energy"]
        assert float(by_name) == float(explicit)
        assert abs(float(by_name) - case["energy"]) <= entry.get("tol_rel", 1e-6) * abs(case["energy"])
        checked += 1
    assert checked >= 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixed_batch_molecules_and_clusters(precision):
    """One batch with molecules (block-per-molecule kernel) and systems above
    its size or periodic (neighbour-list kernel), compared per system."""
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion, RationalDampingParam
    mols = S.batch4096(nmol=6, seed=21)
    big = S.cluster5000(seed=22, natoms=280)
    nums = list(mols["numbers"]) + [big["numbers"]]
    pos = list(mols["positions"]) + [big["positions"]]
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    bat = BatchedDispersion(nums, pos)
    bat.set_precision(precision)
    res = bat.get_dispersion(RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp", "s9")}),
                             grad=True)
    etol, gtol = (RTOL64, GTOL64) if precision == "fp64" else (ETOL_MIXED, None)
    for k in range(len(nums)):
        ref = O.dispersion(nums[k], pos[k], par)
        assert abs(res["energy"][k] - ref["energy"]) <= etol * abs(ref["energy"]), k
        if gtol:
            assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= gtol * np.abs(ref["gradient"]).max(), k
            assert np.abs(res["virial"][k] - ref["virial"]).max() <= gtol * np.abs(ref["virial"]).max(), k
        else:
            assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL_MIXED, k


def test_molecule_kernel_energy_only_and_mixed():
    """Energy-only evaluation and the mixed form of the block-per-molecule kernel."""
    from dftd3 import synthetic as S
    d = S.molecule100(seed=8)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    ref = O.dispersion(d["numbers"], d["positions"], par)
    e = gpu_dispersion(d["numbers"], d["positions"], par, grad=False)
    assert abs(float(e["energy"]) - ref["energy"]) <= RTOL64 * abs(ref["energy"])
    r = gpu_dispersion(d["numbers"], d["positions"], par, precision="mixed")
    assert abs(float(r["energy"]) - ref["energy"]) <= ETOL_MIXED * abs(ref["energy"])
    assert np.abs(r["gradient"] - ref["gradient"]).max() <= GTOL_MIXED


MOL = (3.0, 4, 0, 1)     # launch shapes forcing the block-per-molecule triple kernel


@pytest.mark.parametrize("case", THREE_BODY[:3], ids=[c[0] for c in THREE_BODY[:3]])
def test_golden_atm_molecule_kernel(case):
    name, numbers, pos, param = case
    ref = O.dispersion(numbers, pos, param)
    res = gpu_dispersion(numbers, pos, param, tuning=MOL)
    assert_close(res, ref, RTOL64, GTOL64)


def test_molecule_kernel_smooth_ghosts_partition():
    from dftd3 import synthetic as S
    d = S.molecule100(seed=5)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    cut = (30.0, 12.0, 25.0, 4.0, 3.0)
    ghost = [1, 7, 33]
    ref = O.dispersion(d["numbers"], d["positions"], par, cutoff=cut, ghost=ghost)
    res = gpu_dispersion(d["numbers"], d["positions"], par, cutoff=cut, ghost=ghost, tuning=MOL)
    assert_close(res, ref, RTOL64, GTOL64)
    for part in range(3):
        r = gpu_dispersion(d["numbers"], d["positions"], par, partition=(part, 3), tuning=MOL)
        rp = O.dispersion(d["numbers"], d["positions"], par, part=part, nparts=3)
        assert_close(r, rp, 1.0e-11, 1.0e-11)
    e = gpu_dispersion(d["numbers"], d["positions"], par, grad=False, tuning=MOL)
    ref0 = O.dispersion(d["numbers"], d["positions"], par)
    assert abs(float(e["energy"]) - ref0["energy"]) <= RTOL64 * abs(ref0["energy"])
    m = gpu_dispersion(d["numbers"], d["positions"], par, precision="mixed", tuning=MOL)
    assert abs(float(m["energy"]) - ref0["energy"]) <= ETOL_MIXED * abs(ref0["energy"])
    assert np.abs(m["gradient"] - ref0["gradient"]).max() <= GTOL_MIXED


def test_molecule_kernel_by_count():
    """At least one molecule per SM selects the block-per-molecule kernel by
    itself; the batch agrees with the oracle either way."""
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion, RationalDampingParam
    d = S.batch4096(nmol=200, seed=23, nmax=40)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    bat = BatchedDispersion(d["numbers"], d["positions"])
    p = RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp", "s9")})
    auto = bat.get_dispersion(p, grad=True)
    bat.set_tuning(3.0, 4, 0, 2)
    roots = bat.get_dispersion(p, grad=True)
    assert np.allclose(auto["energy"], roots["energy"], rtol=1e-12, atol=0)
    for k in (0, 77, 199):
        ref = O.dispersion(d["numbers"][k], d["positions"][k], par)
        assert abs(auto["energy"][k] - ref["energy"]) <= RTOL64 * abs(ref["energy"])
        assert np.abs(auto["gradient"][k] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max()
