"""GPU test of the allocation-free entry point, dftd3_b200_get_dispersion_noalloc.

Some callers cannot allocate device memory while they run (code under another
framework's stream capture, integrators that hand out all device memory from
their own pool, loops where cudaMalloc/cudaFree would synchronise the device).
For them the library evaluates the two-body dispersion of one system with all
work arrays taken from a fixed array inside the library.  This test calls that
entry point through the C ABI, twice in a row, and checks its energy, gradient
and virial against the regular entry point (dftd3_get_dispersion) at the FP64
parity tolerance.  The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1.0e-12


def _regular(numbers, positions, par, lattice=None, periodic=None):
    from dftd3.interface import DispersionModel, RationalDampingParam
    model = DispersionModel(numbers, positions, lattice, periodic)
    return model.get_dispersion(RationalDampingParam(**par), grad=True)


def _noalloc(numbers, positions, par, lattice=None, periodic=None):
    import torch
    from dftd3 import library as L
    param = L.new_rational_damping(par["s6"], par["s8"], par["s9"], par["a1"], par["a2"], par["alp"])
    nat = len(numbers)
    num = np.ascontiguousarray(numbers, dtype=np.int32)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=float)
    per = None if periodic is None else np.ascontiguousarray(periodic, dtype=bool)
    pos = torch.tensor(np.asarray(positions, dtype=float), device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros((nat, 3), dtype=torch.float64, device="cuda")
    s = torch.zeros(9, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    L.error_check(L.lib.dftd3_b200_get_dispersion_noalloc)(
        param.handle, nat, L._cast("int*", num), L.ffi.cast("double*", pos.data_ptr()),
        L._cast("double*", lat), L._cast("bool*", per), L.ffi.NULL, L.PRECISION_FP64,
        L.ffi.cast("double*", e.data_ptr()), L.ffi.cast("double*", g.data_ptr()),
        L.ffi.cast("double*", s.data_ptr()), L.ffi.cast("void*", stream.cuda_stream))
    torch.cuda.synchronize()
    return {"energy": e.item(), "gradient": g.cpu().numpy(), "virial": s.cpu().numpy().reshape(3, 3)}


def _check(res, ref):
    assert abs(res["energy"] - float(ref["energy"])) <= RTOL * abs(float(ref["energy"]))
    assert np.abs(res["gradient"] - ref["gradient"]).max() <= RTOL * np.abs(ref["gradient"]).max()
    assert np.abs(res["virial"] - ref["virial"]).max() <= RTOL * np.abs(ref["virial"]).max()


def test_noalloc_matches_regular_entry_point():
    from dftd3 import synthetic
    par = {k: synthetic.PBE_BJ[k] for k in ("s6", "s8", "a1", "a2", "alp")}
    par["s9"] = 0.0
    mol = synthetic.molecule100(seed=11)
    ref = _regular(mol["numbers"], mol["positions"], par)
    # two calls in a row share the scratch array; both must agree
    for _ in range(2):
        _check(_noalloc(mol["numbers"], mol["positions"], par), ref)
    # a periodic cell (wrapped positions, as the regular entry point uses them)
    rng = np.random.default_rng(12)
    lat = synthetic.triclinic(16.0, 17.0, 15.5, 89.0, 91.0, 93.0)
    num = rng.choice([1, 6, 8, 14], size=120).astype(np.int32)
    pos = synthetic.pack_cell(rng, 120, lat, 2.0)
    ref = _regular(num, pos, par, lat, np.array([True, True, True]))
    for _ in range(2):
        _check(_noalloc(num, pos, par, lat, np.array([True, True, True])), ref)


def test_noalloc_rejects_oversized_input():
    from dftd3 import synthetic
    par = {k: synthetic.PBE_BJ[k] for k in ("s6", "s8", "a1", "a2", "alp")}
    par["s9"] = 0.0
    rng = np.random.default_rng(1)
    num = np.ones(5000, dtype=np.int32)
    pos = rng.uniform(0, 100, size=(5000, 3))
    with pytest.raises(RuntimeError, match="supports 1 to 4096 atoms"):
        _noalloc(num, pos, par)
