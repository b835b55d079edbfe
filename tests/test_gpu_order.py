"""The one-block column order gives the atoms the same places as the rank passes.

Batches of at least 32 systems of at most 4096 atoms are put in column order
by one block per system (three bitonic sorts of the order words in shared
memory); a batch holding a larger system takes the multi-launch rank passes
for all its systems.  The words are distinct, so both give every atom the same
place, the same tiles and the same tile spheres, and, with every sum in a
fixed order, the same results bit for bit.  A batch of a test system and 31
molecules (block order) is evaluated again with a 4200-atom cluster appended
(rank passes): every system shared by the two must agree exactly.  Covered: a
1500-atom cluster with the three-body term and a periodic 300-atom cell, FP64
and mixed.  (The average system size stays below 512 atoms in both batches, so
the per-system sums use the same block width.)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _param(s9):
    from dftd3 import synthetic as S
    from dftd3.interface import RationalDampingParam
    return RationalDampingParam(**dict(S.PBE_BJ, s9=s9))


def _molecules():
    from dftd3 import synthetic as S
    d = S.batch4096(seed=7, nmol=31, nmax=96)
    return d["numbers"], d["positions"]


def _compare(a, b, nsys):
    for k in range(nsys):
        assert np.array_equal(np.asarray(a["energy"])[k], np.asarray(b["energy"])[k]), k
        assert np.array_equal(np.ravel(a["gradient"][k]), np.ravel(b["gradient"][k])), k
        assert np.array_equal(np.asarray(a["virial"][k]), np.asarray(b["virial"][k])), k


def _run(nums, pos, lats, pers, precision, s9):
    from dftd3.interface import BatchedDispersion
    bat = BatchedDispersion(nums, pos, None if lats is None else np.array(lats),
                            None if pers is None else np.array(pers))
    bat.set_precision(precision)
    bat.set_tuning(0.0, 2)          # the same work split in both batches
    return bat.get_dispersion(_param(s9), grad=True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cluster_block_order_matches_rank_passes(precision):
    from dftd3 import synthetic as S
    small = S.cluster5000(seed=3, natoms=1500)
    large = S.cluster5000(seed=4, natoms=4200)
    mn, mp = _molecules()
    nums = [small["numbers"]] + mn
    pos = [small["positions"]] + mp
    a = _run(nums, pos, None, None, precision, 1.0)
    b = _run(nums + [large["numbers"]], pos + [large["positions"]], None, None, precision, 1.0)
    _compare(a, b, len(nums))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cell_block_order_matches_rank_passes(precision):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(5)
    lat = S.triclinic(15.0, 16.0, 17.0, 88.0, 92.0, 95.0)
    num = rng.choice([1, 6, 7, 8, 14], size=300).astype(np.int32)
    cell = S.pack_cell(rng, 300, lat, 2.0)
    large = S.cluster5000(seed=6, natoms=4200)
    mn, mp = _molecules()
    nums = [num] + mn
    pos = [cell] + mp
    lats = [lat] + [np.eye(3) * 1000.0] * len(mn)
    pers = [[True] * 3] + [[False] * 3] * len(mn)
    a = _run(nums, pos, lats, pers, precision, 0.0)
    b = _run(nums + [large["numbers"]], pos + [large["positions"]], lats + [np.eye(3) * 1000.0],
             pers + [[False] * 3], precision, 0.0)
    _compare(a, b, len(nums))
