"""Bit-reproducible results: the same input evaluated twice gives identical
energy, gradient and virial, with the three-body term on (s9 = 1).

The reference merges its thread partials in OpenMP critical sections
(atm.f90:813), so its own sums depend on the thread schedule; here every sum
has a fixed order (shared-memory and register sums in a fixed sequence, the
neighbour-list kernel's per-atom sums in fixed point), so both forms repeat
bit for bit.  Covered: the block-per-molecule kernel and the neighbour-list
kernel on a 16-molecule batch, a 700-atom cluster, and a small periodic cell
whose images are repeated atoms (triple_scale, atm.f90:954-980).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _param():
    from dftd3 import synthetic as S
    from dftd3.interface import RationalDampingParam
    return RationalDampingParam(**dict(S.PBE_BJ, s9=1.0))


def _twice(make):
    out = []
    for _ in range(2):
        r = make()
        out.append([np.array(r["energy"], dtype=float).copy(),
                    np.concatenate([np.ravel(g) for g in r["gradient"]]) if isinstance(r["gradient"], list)
                    else np.array(r["gradient"]).copy(),
                    np.array(r["virial"]).copy()])
    return out


def _assert_identical(out):
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kernel", [1, 2], ids=["molecule", "roots"])
def test_batch_repeats_bit_for_bit(precision, kernel):
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion
    d = S.batch4096(seed=0, nmol=16)

    def make():
        bat = BatchedDispersion(d["numbers"], d["positions"])
        bat.set_precision(precision)
        bat.set_tuning(0.0, 0, 0, kernel)
        return bat.get_dispersion(_param(), grad=True)

    _assert_identical(_twice(make))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cluster_repeats_bit_for_bit(precision):
    from dftd3 import synthetic as S
    from dftd3.interface import DispersionModel
    c = S.cluster5000(seed=0, natoms=700)

    def make():
        m = DispersionModel(c["numbers"], c["positions"])
        m.set_precision(precision)
        return m.get_dispersion(_param(), grad=True)

    _assert_identical(_twice(make))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_periodic_cell_repeats_bit_for_bit(precision):
    from dftd3 import synthetic as S
    from dftd3.interface import DispersionModel
    rng = np.random.default_rng(9)
    lat = S.triclinic(9.5, 10.0, 10.5, 87.0, 91.0, 94.0)
    num = rng.choice([1, 6, 8], size=24).astype(np.int32)
    pos = S.pack_cell(rng, 24, lat, 2.0)

    def make():
        m = DispersionModel(num, pos, lat, np.array([True, True, True]))
        m.set_precision(precision)
        m.set_realspace_cutoff(25.0, 20.0, 20.0)
        return m.get_dispersion(_param(), grad=True)

    _assert_identical(_twice(make))
