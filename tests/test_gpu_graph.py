"""GPU tests of the captured launch sequence (CUDA graph replay), the launch
shape settings and the autotuner: every shape and every replay must give the
FP64 oracle's results to 1e-12."""
import numpy as np
import pytest

import oracle_ref as O
from test_gpu_twobody import GTOL64, RTOL64

pytestmark = pytest.mark.gpu


def _molecules(nmol, seed):
    from dftd3 import synthetic as S
    return S.batch4096(nmol=nmol, seed=seed)


def _param(s9=1.0):
    from dftd3 import synthetic as S
    from dftd3.interface import RationalDampingParam
    par = dict(S.PBE_BJ, damping="rational", s9=s9)
    return par, RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp", "s9")})


def _check(res, d, par, systems):
    for k in systems:
        ref = O.dispersion(d["numbers"][k], d["positions"][k], par)
        assert abs(res["energy"][k] - ref["energy"]) <= RTOL64 * abs(ref["energy"]), k
        assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max(), k
        assert np.abs(res["virial"][k] - ref["virial"]).max() <= GTOL64 * max(np.abs(ref["virial"]).max(), 1e-30), k


@pytest.mark.parametrize("s9", [0.0, 1.0])
def test_graph_replays_match_oracle(s9):
    from dftd3.interface import BatchedDispersion
    d = _molecules(24, seed=11)
    par, param = _param(s9)
    bat = BatchedDispersion(d["numbers"], d["positions"])
    bat.set_graph(True)
    first = bat.get_dispersion(param, grad=True)      # ordinary sequence, then capture
    for _ in range(3):                                 # replays
        res = bat.get_dispersion(param, grad=True)
        assert np.allclose(res["energy"], first["energy"], rtol=1e-13, atol=0)
    _check(res, d, par, range(0, 24, 5))
    # new positions: the same graph reads the new input buffer
    rng = np.random.default_rng(2)
    moved = [p + rng.normal(scale=0.05, size=p.shape) for p in d["positions"]]
    bat.update(moved)
    res = bat.get_dispersion(param, grad=True)
    _check(res, dict(d, positions=moved), par, range(1, 24, 6))


def test_graph_list_overflow_falls_back():
    """Replay with denser geometries than at capture: the neighbour lists of
    the root kernel (systems above the molecule kernel's size) outgrow the
    captured buffers, and the replay is redone without the graph."""
    from dftd3 import synthetic as S
    from dftd3.interface import BatchedDispersion
    clusters = [S.cluster5000(seed=s, natoms=300) for s in (1, 2)]
    nums = [c["numbers"] for c in clusters]
    pos = [c["positions"] for c in clusters]
    par, param = _param(1.0)
    bat = BatchedDispersion(nums, pos)
    bat.set_graph(True)
    bat.set_realspace_cutoff(60.0, 12.0, 40.0)
    par_cut = (60.0, 12.0, 40.0, 0.0, 0.0)
    bat.get_dispersion(param, grad=True)
    bat.get_dispersion(param, grad=True)
    squeezed = [0.8 * p for p in pos]   # min distance 1.44 Bohr: more triples within 12 Bohr
    bat.update(squeezed)
    for _ in range(2):   # fallback evaluation, then a fresh capture and its replay
        res = bat.get_dispersion(param, grad=True)
        for k in range(2):
            ref = O.dispersion(nums[k], squeezed[k], par, cutoff=par_cut)
            assert abs(res["energy"][k] - ref["energy"]) <= RTOL64 * abs(ref["energy"])
            assert np.abs(res["gradient"][k] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max()


@pytest.mark.parametrize("shape", [(3.0, 4, 1, 1), (2.0, 1, 2, 2), (6.0, 2, 0, 1), (4.5, 4, 0, 0), (0.0, 2, 1, 1), (0.0, 1, 0, 2)])
def test_launch_shapes(shape):
    from dftd3.interface import BatchedDispersion
    d = _molecules(12, seed=13)
    par, param = _param(1.0)
    bat = BatchedDispersion(d["numbers"], d["positions"])
    bat.set_tuning(*shape)
    _check(bat.get_dispersion(param, grad=True), d, par, range(0, 12, 3))


def test_autotune_keeps_results():
    from dftd3.interface import BatchedDispersion
    from dftd3 import library
    d = _molecules(16, seed=14)
    par, param = _param(1.0)
    bat = BatchedDispersion(d["numbers"], d["positions"])
    tuned = bat.autotune(param, grad=True)
    assert tuned["ms"] > 0
    assert tuned["pair_split"] in (0, 1, 2, 4)
    assert tuned["atm_mol"] in (0, 1, 2)
    assert tuned["morton_cell"] in (0.0, 2.0, 3.0, 4.5, 6.0)
    bat.set_graph(True)
    for _ in range(2):
        res = bat.get_dispersion(param, grad=True)
    _check(res, d, par, range(0, 16, 4))
    with pytest.raises(RuntimeError, match="1, 2 or 4"):
        library.set_batch_tuning(bat._batch, 3.0, 6, 0)
    with pytest.raises(RuntimeError, match="0, 1 or 2"):
        library.set_batch_tuning(bat._batch, 3.0, 4, 0, 5)


def test_device_api_graph_with_parameter_derivatives():
    import torch
    from dftd3 import library
    from dftd3 import synthetic as S
    d = _molecules(10, seed=15)
    natoms = np.array([len(n) for n in d["numbers"]], dtype=np.int32)
    nums = np.concatenate(d["numbers"]).astype(np.int32)
    pos = torch.tensor(np.concatenate(d["positions"]), device="cuda")
    param = library.new_rational_damping(1.0, S.PBE_BJ["s8"], 1.0, S.PBE_BJ["a1"], S.PBE_BJ["a2"], 14.0)
    out = {}
    for graph in (False, True):
        batch = library.new_batch(natoms, nums, None, None)
        library.set_batch_graph(batch, graph)
        for _ in range(3 if graph else 1):
            e = torch.zeros(len(natoms), dtype=torch.float64, device="cuda")
            g = torch.zeros_like(pos)
            sg = torch.zeros((len(natoms), 9), dtype=torch.float64, device="cuda")
            pg = torch.zeros((len(natoms), 5), dtype=torch.float64, device="cuda")
            library.get_dispersion_device(batch, param, pos.data_ptr(), None, e.data_ptr(), g.data_ptr(),
                                          sg.data_ptr(), pg.data_ptr(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
        out[graph] = [t.cpu().numpy() for t in (e, g, sg, pg)]
    for a, b in zip(out[False], out[True]):
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(a).max(), 1e-30)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_model_graph_replay(precision):
    """dftd3_get_dispersion of a model with dftd3_b200_set_model_graph: the
    first call captures, later calls with new positions and a new lattice
    replay, each matching the oracle."""
    from dftd3 import synthetic as S
    from dftd3.interface import DispersionModel, RationalDampingParam
    import oracle_ref as O
    rng = np.random.default_rng(41)
    lat = S.triclinic(14.0, 14.5, 15.0, 89.0, 91.0, 92.0)
    num = rng.choice([1, 6, 8], size=48).astype(np.int32)
    pos = S.pack_cell(rng, 48, lat, 2.0)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    # cutoffs away from the cell edges: a self-image exactly on a cutoff
    # sphere is in or out by the last bit of r^2
    cut = (31.1, 16.3, 21.7, 0.0, 0.0)
    model = DispersionModel(num, pos, lat, np.array([True] * 3))
    model.set_realspace_cutoff(*cut)
    model.set_precision(precision)
    model.set_graph(True)
    param = RationalDampingParam(**{k: par[k] for k in ("s6", "s8", "a1", "a2", "alp", "s9")})
    for step in range(4):
        p = pos + rng.normal(scale=0.05, size=pos.shape)
        la = lat * (1.0 + 0.01 * step)
        model.update(p @ np.linalg.inv(lat) @ la, la)
        res = model.get_dispersion(param, grad=True)
        ref = O.dispersion(num, p @ np.linalg.inv(lat) @ la, par, lattice=la, periodic=[True] * 3, cutoff=cut)
        if precision == "fp64":
            assert abs(float(res["energy"]) - ref["energy"]) <= RTOL64 * abs(ref["energy"])
            assert np.abs(res["gradient"] - ref["gradient"]).max() <= GTOL64 * np.abs(ref["gradient"]).max()
        else:
            assert abs(float(res["energy"]) - ref["energy"]) <= 1e-7 * abs(ref["energy"])
            assert np.abs(res["gradient"] - ref["gradient"]).max() <= 1e-7
