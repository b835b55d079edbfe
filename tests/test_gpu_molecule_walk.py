"""GPU parity of the molecule-batch diagonal walks (k_two_body_rot, k_cn_rot,
k_cn_chain_rot) against the FP64 oracle and against the general tile sweeps.

A batch of 40 molecules of 8-160 atoms (about 2500 atoms, so the batch takes
the tile path rather than the small-system kernels) has the single lattice
point T = 0 everywhere, which selects the diagonal walks for the two-body sum,
the CN and the stored chain rule (FP64 as well, every molecule having at most
256 atoms).  Rational damping with and without the three-body term and zero
damping are compared per molecule with the oracle (ncoord.f90:86-228,
rational.f90:378-514, zero.f90:409-553): FP64 to 1e-12, mixed to 1e-7
relative energy (3e-7 for zero damping) and 1e-7 Hartree/Bohr gradient.  The same batch with two work
items per tile pair (which the walks do not take) gives the general sweeps'
results, which the walks must match to 1e-12 in FP64.
"""
import numpy as np
import pytest

import oracle_ref as O

pytestmark = pytest.mark.gpu

RTOL64 = 1.0e-12
ETOL_MIXED = 1.0e-7
# zero damping's factor goes as (R0/r)^14, which multiplies the FP32 rounding
# of r^2 sevenfold: on molecules of ten atoms the mixed energy is up to 2e-7
# off in the general sweeps as well
ETOL_MIXED_ZERO = 3.0e-7
GTOL_MIXED = 1.0e-7       # Hartree/Bohr

PARAMS = {
    "rational": dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, alp=14.0, s9=0.0),
    "rational-atm": dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, alp=14.0, s9=1.0),
    "zero": dict(damping="zero", s6=1.0, s8=0.722, rs6=1.217, rs8=1.0, alp=14.0, s9=0.0),
}


def _param(p):
    from dftd3 import interface as I
    if p["damping"] == "zero":
        return I.ZeroDampingParam(s6=p["s6"], s8=p["s8"], s9=p["s9"], rs6=p["rs6"], rs8=p["rs8"], alp=p["alp"])
    return I.RationalDampingParam(s6=p["s6"], s8=p["s8"], s9=p["s9"], a1=p["a1"], a2=p["a2"], alp=p["alp"])


@pytest.fixture(scope="module")
def batch():
    from dftd3 import synthetic as S
    d = S.batch4096(seed=41, nmol=40, nmin=8, nmax=160)
    assert sum(len(n) for n in d["numbers"]) > 2048
    return d["numbers"], d["positions"]


def _run(nums, pos, par, precision, split=0):
    from dftd3.interface import BatchedDispersion
    bat = BatchedDispersion(nums, pos)
    bat.set_precision(precision)
    bat.set_tuning(0.0, split)
    return bat.get_dispersion(_param(par), grad=True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(PARAMS))
def test_walks_match_oracle(batch, name, precision):
    nums, pos = batch
    par = PARAMS[name]
    res = _run(nums, pos, par, precision)
    # a sample of the molecules, the largest among them
    order = np.argsort([-len(n) for n in nums])
    for k in list(order[:3]) + list(range(0, len(nums), 7)):
        ref = O.dispersion(nums[k], pos[k], par)
        e, g, v = float(res["energy"][k]), np.asarray(res["gradient"][k]), np.asarray(res["virial"][k])
        if precision == "fp64":
            assert abs(e - ref["energy"]) <= RTOL64 * abs(ref["energy"]), (k, e, ref["energy"])
            assert np.abs(g - ref["gradient"]).max() <= RTOL64 * np.abs(ref["gradient"]).max()
            assert np.abs(v - ref["virial"]).max() <= RTOL64 * np.abs(ref["virial"]).max()
        else:
            etol = ETOL_MIXED_ZERO if par["damping"] == "zero" else ETOL_MIXED
            assert abs(e - ref["energy"]) <= etol * abs(ref["energy"]), (k, e, ref["energy"])
            assert np.abs(g - ref["gradient"]).max() <= GTOL_MIXED


@pytest.mark.parametrize("name", sorted(PARAMS))
def test_walks_match_general_sweeps(batch, name):
    nums, pos = batch
    par = PARAMS[name]
    walk = _run(nums, pos, par, "fp64")
    general = _run(nums, pos, par, "fp64", split=2)
    e_w, e_g = np.asarray(walk["energy"]), np.asarray(general["energy"])
    assert np.all(np.abs(e_w - e_g) <= RTOL64 * np.abs(e_g))
    for k in range(len(nums)):
        gw, gg = np.asarray(walk["gradient"][k]), np.asarray(general["gradient"][k])
        assert np.abs(gw - gg).max() <= RTOL64 * max(np.abs(gg).max(), 1e-300)
        vw, vg = np.asarray(walk["virial"][k]), np.asarray(general["virial"][k])
        assert np.abs(vw - vg).max() <= RTOL64 * max(np.abs(vg).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_walks_with_ghost_atoms(precision):
    """A 300-atom molecule (tile path: the mixed form takes the walks, FP64 the
    general sweeps above 256 atoms) with ghost atoms, which keep their CN
    share but have no C6 (model.f90:166-174, 398-401)."""
    from dftd3 import synthetic as S
    from dftd3.interface import DispersionModel
    c = S.cluster5000(seed=43, natoms=300)
    par = PARAMS["rational"]
    ghost = [0, 17, 64, 150, 299]
    ref = O.dispersion(c["numbers"], c["positions"], par, ghost=ghost)
    model = DispersionModel(c["numbers"], c["positions"])
    model.set_precision(precision)
    model.set_ghost_atoms(ghost)
    res = model.get_dispersion(_param(par), grad=True)
    e, g = float(res["energy"]), np.asarray(res["gradient"])
    if precision == "fp64":
        assert abs(e - ref["energy"]) <= RTOL64 * abs(ref["energy"])
        assert np.abs(g - ref["gradient"]).max() <= RTOL64 * np.abs(ref["gradient"]).max()
    else:
        assert abs(e - ref["energy"]) <= ETOL_MIXED * abs(ref["energy"])
        assert np.abs(g - ref["gradient"]).max() <= GTOL_MIXED
