"""GPU parity of the tile-pair sweeps for every work split of a tile pair
(tuning[1]: 1 the whole pair, 2 halves of the j tile, 4 also halves of the
translation list) in both forms, on periodic cells whose CN lattice points
fit one chunk of 128 (the CN pass stores the chain-rule sums) and cells that
need several chunks (the chain rule evaluates the terms again).  The work
counters of the counting launches must not depend on the split."""
import numpy as np
import pytest

import oracle_ref as O
from test_gpu_twobody import ETOL_MIXED, GTOL_MIXED, GTOL64, RTOL64, _param_obj, assert_close

pytestmark = pytest.mark.gpu

PAR = dict(damping="rational", s6=1.0, s8=1.2177, a1=0.4145, a2=4.8593, s9=0.0, alp=14.0)
PAR_ZERO = dict(damping="zero", s6=1.0, s8=1.703, rs6=1.261, rs8=1.0, s9=0.0, alp=14.0)
VTOL_MIXED = 1.0e-6        # mixed form: virial, relative to its largest component


def _cell(seed, n, edge):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(seed)
    lat = S.triclinic(edge, 1.05 * edge, 0.95 * edge, 88.0, 92.0, 95.0)
    num = rng.choice([1, 6, 7, 8], size=n).astype(np.int32)
    pos = S.pack_cell(rng, n, lat, 2.0)
    return num, pos, lat


def _model(num, pos, lat, cut, precision, split):
    from dftd3.interface import DispersionModel
    model = DispersionModel(num, pos, lat, np.array([True, True, True]))
    model.set_realspace_cutoff(*cut[:3])
    model.set_precision(precision)
    model.set_tuning(0.0, split)
    return model


# (seed, atoms, cell edge, cutoffs disp2 / disp3 / CN): the first cell's CN
# lattice points fit one chunk, the second's do not
CELLS = {"one_chunk": (31, 150, 18.0, (30.0, 20.0, 25.0)), "chunks": (32, 44, 12.0, (35.0, 20.0, 30.0))}


@pytest.mark.parametrize("cell", sorted(CELLS))
@pytest.mark.parametrize("split", [1, 2, 4])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_parity(cell, split, precision):
    seed, n, edge, cut = CELLS[cell]
    num, pos, lat = _cell(seed, n, edge)
    ocut = (cut[0], cut[1], cut[2], 0.0, 0.0)
    ref = O.dispersion(num, pos, PAR, lattice=lat, periodic=[True] * 3, cutoff=ocut)
    res = _model(num, pos, lat, cut, precision, split).get_dispersion(_param_obj(PAR), grad=True)
    if precision == "fp64":
        assert_close(res, ref, RTOL64, GTOL64)
    else:
        e, er = float(res["energy"]), ref["energy"]
        assert abs(e - er) <= ETOL_MIXED * abs(er), (e - er) / er
        assert np.abs(res["gradient"] - ref["gradient"]).max() <= GTOL_MIXED
        # the mixed form's budget covers energy and gradient; its virial is
        # checked at 1e-6 of the largest component (4e-7 measured on the
        # one-chunk cell)
        vscale = np.abs(ref["virial"]).max()
        assert np.abs(res["virial"] - ref["virial"]).max() <= VTOL_MIXED * vscale


@pytest.mark.parametrize("split", [1, 2, 4])
def test_split_zero_damping_ghosts(split):
    """Zero damping with ghost atoms (zero species vectors) on the one-chunk cell."""
    from dftd3.interface import DispersionModel
    seed, n, edge, cut = CELLS["one_chunk"]
    num, pos, lat = _cell(seed, n, edge)
    ghost = [0, 5, 17, 64]
    ref = O.dispersion(num, pos, PAR_ZERO, lattice=lat, periodic=[True] * 3,
                       cutoff=(cut[0], cut[1], cut[2], 0.0, 0.0), ghost=ghost)
    model = DispersionModel(num, pos, lat, np.array([True, True, True]))
    model.set_realspace_cutoff(*cut)
    model.set_ghost_atoms(ghost)
    model.set_tuning(0.0, split)
    res = model.get_dispersion(_param_obj(PAR_ZERO), grad=True)
    assert_close(res, ref, RTOL64, GTOL64)


@pytest.mark.parametrize("cell", sorted(CELLS))
def test_split_counts_batch(cell):
    """A batch of the cell and a shifted copy: every split gives each
    system the oracle's result, and the pair, triple and CN term counts of
    the counting launches are properties of the structures."""
    from dftd3 import library
    from dftd3.interface import BatchedDispersion
    seed, n, edge, cut = CELLS[cell]
    num, pos, lat = _cell(seed, n, edge)
    pos2 = pos + np.array([0.7, -1.1, 0.4])
    ocut = (cut[0], cut[1], cut[2], 0.0, 0.0)
    refs = [O.dispersion(num, p, PAR, lattice=lat, periodic=[True] * 3, cutoff=ocut) for p in (pos, pos2)]
    counts = []
    for precision in ("fp64", "mixed"):
        for split in (1, 2, 4):
            bat = BatchedDispersion([num, num], [pos, pos2], np.array([lat, lat]), np.ones((2, 3), dtype=bool))
            bat.set_realspace_cutoff(*cut)
            bat.set_precision(precision)
            bat.set_tuning(0.0, split)
            library.set_batch_counting(bat._batch, True)
            res = bat.get_dispersion(_param_obj(PAR), grad=True)
            counts.append(tuple(int(x) for x in library.get_batch_counts(bat._batch)))
            for k in range(2):
                e, er = float(res["energy"][k]), refs[k]["energy"]
                tol = RTOL64 if precision == "fp64" else ETOL_MIXED
                assert abs(e - er) <= tol * abs(er), (precision, split, k, (e - er) / er)
    assert counts[0][0] > 0 and counts[0][2] > 0
    assert all(c == counts[0] for c in counts), counts
