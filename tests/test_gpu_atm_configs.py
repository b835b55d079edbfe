"""GPU parity of the three-body workloads at their full sizes against the FP64
oracle (get_atm_dispersion_derivs, atm.f90:625-825, with the two-body sum and
the CN chain rule of disp.f90:56-185).

  * the whole 5000-atom cluster of seed 0 (D3(BJ) + ATM, 40 Bohr three-body
    cutoff, about 1.7e9 accepted triples);
  * frames 0 and 1 of the periodic 512-atom frame set of seed 0 (125 images,
    about 1e9 triples per frame), evaluated as one batch;
  * 64 molecules of the 4096-molecule batch of seed 0, its eight largest
    (256 atoms) among them, with the block-per-molecule triple kernel and with
    the neighbour-list kernel.

The oracle needs minutes for the first two, so its results were stored once
by tests/golden/make_atm_fixtures.py (atm_configs.npz, with a checksum of the
generated positions); the molecule sample is evaluated by the oracle here.
Tolerances: FP64 1e-12 (energy relative, gradient and virial relative to their
largest component); mixed 1e-7 relative energy, 1e-7 Hartree/Bohr largest
gradient error and 1e-6 of the largest virial component (the FP32 pair terms
of the smallest molecules leave their virial about 7e-7 off).
"""
from pathlib import Path

import numpy as np
import pytest

import oracle_ref as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
RTOL64 = 1.0e-12
ETOL_MIXED = 1.0e-7
GTOL_MIXED = 1.0e-7            # Hartree/Bohr
VTOL_MIXED = 1.0e-6


def _param():
    from dftd3 import synthetic as S
    return dict(S.PBE_BJ, damping="rational", s9=1.0)


def _rp(par):
    from dftd3.interface import RationalDampingParam
    return RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp", "s9")})


@pytest.fixture(scope="module")
def fixtures():
    return dict(np.load(GOLDEN / "atm_configs.npz"))


def _checksum(pos):
    return float(np.sum(np.asarray(pos, dtype=float) * np.arange(1, 4)))


def _compare(e, g, v, e_ref, g_ref, v_ref, precision, periodic=False):
    g_ref, v_ref = np.asarray(g_ref), np.asarray(v_ref)
    if precision == "fp64":
        assert abs(e - e_ref) <= RTOL64 * abs(e_ref), (e - e_ref) / e_ref
        assert np.abs(g - g_ref).max() <= RTOL64 * np.abs(g_ref).max()
        assert np.abs(v - v_ref).max() <= RTOL64 * np.abs(v_ref).max()
    else:
        assert abs(e - e_ref) <= ETOL_MIXED * abs(e_ref), (e - e_ref) / e_ref
        assert np.abs(g - g_ref).max() <= GTOL_MIXED, np.abs(g - g_ref).max()
        assert np.abs(v - v_ref).max() <= VTOL_MIXED * np.abs(v_ref).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cluster5000_full(fixtures, precision):
    from dftd3 import synthetic as S
    from dftd3.interface import DispersionModel
    d = S.cluster5000(seed=0)
    assert _checksum(d["positions"]) == float(fixtures["cluster5000_checksum"])
    model = DispersionModel(d["numbers"], d["positions"])
    model.set_precision(precision)
    res = model.get_dispersion(_rp(_param()), grad=True)
    _compare(float(res["energy"]), res["gradient"], res["virial"], float(fixtures["cluster5000_energy"]),
             fixtures["cluster5000_gradient"], fixtures["cluster5000_virial"], precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_periodic_frames(fixtures, precision):
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion
    f = S.frames256(seed=0, nframes=2)
    for k in range(2):
        assert _checksum(f["positions"][k]) == float(fixtures[f"frame{k}_checksum"])
    bat = BatchedDispersion(f["numbers"], f["positions"], f["lattices"], f["periodic"])
    bat.set_precision(precision)
    res = bat.get_dispersion(_rp(_param()), grad=True)
    for k in range(2):
        _compare(float(res["energy"][k]), res["gradient"][k], res["virial"][k], float(fixtures[f"frame{k}_energy"]),
                 fixtures[f"frame{k}_gradient"], fixtures[f"frame{k}_virial"], precision, periodic=True)


@pytest.fixture(scope="module")
def molecule_sample():
    from dftd3 import synthetic as S
    d = S.batch4096(seed=0)
    pick = S.batch4096_sample([len(n) for n in d["numbers"]])
    nums = [d["numbers"][k] for k in pick]
    pos = [d["positions"][k] for k in pick]
    assert max(len(n) for n in nums) == 256
    refs = [O.dispersion(n, p, _param()) for n, p in zip(nums, pos)]
    return nums, pos, refs


@pytest.mark.parametrize("kernel", ["molecule", "roots"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch4096_sample(molecule_sample, kernel, precision):
    from dftd3.interface import BatchedDispersion
    nums, pos, refs = molecule_sample
    bat = BatchedDispersion(nums, pos)
    bat.set_precision(precision)
    bat.set_tuning(0.0, 0, 0, 1 if kernel == "molecule" else 2)
    res = bat.get_dispersion(_rp(_param()), grad=True)
    for k, ref in enumerate(refs):
        _compare(float(res["energy"][k]), res["gradient"][k], res["virial"][k], ref["energy"], ref["gradient"],
                 ref["virial"], precision)
