"""GPU tests of the allocation-free entry point, dftd3_b200_get_dispersion_noalloc.

Some callers cannot allocate device memory while they run: integrators and MD
engines that hand out all device memory from their own pool, and time-step
loops in which cudaMalloc/cudaFree are not allowed because they can
synchronise the whole device.  For them the library evaluates the two-body
dispersion of one system with all work arrays taken from a fixed array inside
the library.  These tests call that entry point through the C ABI, twice in a
row (the calls share the array), and check its energy, gradient and virial
against the regular entry point (dftd3_get_dispersion) at the parity
tolerances of the other tests: 1e-12 for FP64; for the mixed form 1e-7
relative energy, 1e-7 Hartree/Bohr gradient and 1e-6 of the largest virial
component.  The
largest input it accepts (4096 atoms, periodic) is also checked against the
FP64 oracle, and inputs beyond the limits must be rejected with a message.
The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# FP64: energy 1e-12 relative, gradient and virial 1e-12 of their largest
# component.  Mixed: energy 1e-7 relative, gradient 1e-7 Hartree/Bohr, virial
# 1e-6 of its largest component (the tolerances of the other parity tests).
RTOL = {"fp64": 1.0e-12, "mixed": 1.0e-7}
GRAD_ABS_MIXED = 1.0e-7
VIRIAL_RTOL = {"fp64": 1.0e-12, "mixed": 1.0e-6}
RATIONAL = dict(s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, alp=14.0, s9=0.0)   # PBE-D3(BJ)
ZERO = dict(s6=1.0, s8=0.722, rs6=1.217, rs8=1.0, alp=14.0, s9=0.0)           # PBE-D3(0)


def _param(damping, par):
    from dftd3 import library as L
    if damping == "rational":
        return L.new_rational_damping(par["s6"], par["s8"], par["s9"], par["a1"], par["a2"], par["alp"])
    return L.new_zero_damping(par["s6"], par["s8"], par["s9"], par["rs6"], par["rs8"], par["alp"])


def _regular(numbers, positions, damping, par, precision, grad, lattice=None, periodic=None):
    from dftd3.interface import DispersionModel, RationalDampingParam, ZeroDampingParam
    model = DispersionModel(numbers, positions, lattice, periodic)
    model.set_precision(precision)
    p = RationalDampingParam(**par) if damping == "rational" else ZeroDampingParam(**par)
    return model.get_dispersion(p, grad=grad)


def _noalloc(numbers, positions, damping, par, precision="fp64", outputs=("gradient", "virial"), lattice=None,
             periodic=None):
    import torch
    from dftd3 import library as L
    param = _param(damping, par)
    nat = len(numbers)
    num = np.ascontiguousarray(numbers, dtype=np.int32)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=float)
    per = None if periodic is None else np.ascontiguousarray(periodic, dtype=bool)
    pos = torch.tensor(np.asarray(positions, dtype=float), device="cuda")
    # outputs start as NaN so that an element the call fails to write shows up
    e = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    g = torch.full((nat, 3), float("nan"), dtype=torch.float64, device="cuda")
    s = torch.full((9,), float("nan"), dtype=torch.float64, device="cuda")
    prec = L.PRECISION_FP64 if precision == "fp64" else L.PRECISION_MIXED
    stream = torch.cuda.current_stream()
    L.error_check(L.lib.dftd3_b200_get_dispersion_noalloc)(
        param.handle, nat, L._cast("int*", num), L.ffi.cast("double*", pos.data_ptr()),
        L._cast("double*", lat), L._cast("bool*", per), L.ffi.NULL, prec,
        L.ffi.cast("double*", e.data_ptr()),
        L.ffi.cast("double*", g.data_ptr()) if "gradient" in outputs else L.ffi.NULL,
        L.ffi.cast("double*", s.data_ptr()) if "virial" in outputs else L.ffi.NULL,
        L.ffi.cast("void*", stream.cuda_stream))
    torch.cuda.synchronize()
    out = {"energy": e.item()}
    if "gradient" in outputs:
        out["gradient"] = g.cpu().numpy()
    if "virial" in outputs:
        out["virial"] = s.cpu().numpy().reshape(3, 3)
    return out


def _close(a, b, rtol):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    assert np.all(np.isfinite(a))
    return float(np.abs(a - b).max()) <= rtol * max(float(np.abs(b).max()), 1e-300)


def _check(res, ref, precision):
    rtol = RTOL[precision]
    assert np.isfinite(res["energy"])
    assert abs(res["energy"] - float(ref["energy"])) <= rtol * abs(float(ref["energy"])), (res["energy"], ref["energy"])
    if "gradient" in res:
        if precision == "fp64":
            assert _close(res["gradient"], ref["gradient"], rtol)
        else:
            assert np.all(np.isfinite(res["gradient"]))
            assert float(np.abs(res["gradient"] - ref["gradient"]).max()) <= GRAD_ABS_MIXED
    if "virial" in res:
        assert _close(res["virial"], ref["virial"], VIRIAL_RTOL[precision])


def _periodic_cell(seed, natoms, edge):
    from dftd3 import synthetic
    rng = np.random.default_rng(seed)
    lat = synthetic.triclinic(edge, edge * 1.04, edge * 0.97, 89.0, 91.0, 93.0)
    num = rng.choice([1, 6, 7, 8, 14], size=natoms, p=[0.3, 0.3, 0.1, 0.2, 0.1]).astype(np.int32)
    pos = synthetic.pack_cell(rng, natoms, lat, 2.0)
    return num, pos, lat


@pytest.mark.parametrize("damping", ["rational", "zero"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_regular_entry_point(damping, precision):
    from dftd3 import synthetic
    par = RATIONAL if damping == "rational" else ZERO
    mol = synthetic.molecule100(seed=11)
    ref = _regular(mol["numbers"], mol["positions"], damping, par, precision, True)
    # two calls in a row share the scratch array; both must agree
    for _ in range(2):
        _check(_noalloc(mol["numbers"], mol["positions"], damping, par, precision), ref, precision)
    # a periodic cell (positions inside the cell, as the regular entry point wraps them)
    num, pos, lat = _periodic_cell(12, 120, 16.0)
    per = np.array([True, True, True])
    ref = _regular(num, pos, damping, par, precision, True, lat, per)
    for _ in range(2):
        _check(_noalloc(num, pos, damping, par, precision, lattice=lat, periodic=per), ref, precision)


@pytest.mark.parametrize("outputs", [(), ("gradient",), ("virial",)])
def test_noalloc_optional_outputs(outputs):
    from dftd3 import synthetic
    mol = synthetic.molecule100(seed=5)
    ref = _regular(mol["numbers"], mol["positions"], "rational", RATIONAL, "fp64", True)
    for _ in range(2):
        _check(_noalloc(mol["numbers"], mol["positions"], "rational", RATIONAL, "fp64", outputs=outputs), ref, "fp64")


def test_noalloc_vanishing_two_body_term():
    # s6 = s8 = 0: nothing is launched for the pair sum, the outputs must be zero
    # even though the previous call left its sums in the shared array
    from dftd3 import synthetic
    mol = synthetic.molecule100(seed=3)
    _noalloc(mol["numbers"], mol["positions"], "rational", RATIONAL)
    par = dict(RATIONAL, s6=0.0, s8=0.0)
    res = _noalloc(mol["numbers"], mol["positions"], "rational", par)
    assert res["energy"] == 0.0
    assert not np.any(res["gradient"]) and not np.any(res["virial"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_largest_periodic_cell_against_oracle(precision):
    # 4096 atoms (the limit), triclinic cell at the density of the 2000-atom
    # benchmark cell, 125 images within 60 Bohr
    import oracle_ref
    num, pos, lat = _periodic_cell(21, 4096, 53.0)
    per = np.array([True, True, True])
    ref = oracle_ref.dispersion(num, pos, dict(RATIONAL, damping="rational"), lattice=lat, periodic=per)
    for _ in range(2):
        _check(_noalloc(num, ref["positions"], "rational", RATIONAL, precision, lattice=lat, periodic=per), ref, precision)


def test_noalloc_rejects_inputs_beyond_limits():
    rng = np.random.default_rng(1)
    num = np.ones(4097, dtype=np.int32)
    pos = rng.uniform(0, 100, size=(4097, 3))
    with pytest.raises(RuntimeError, match="supports 1 to 4096 atoms"):
        _noalloc(num, pos, "rational", RATIONAL)
    # 17 distinct elements
    num = np.arange(1, 18, dtype=np.int32)
    pos = np.array([[3.0 * k, 0.0, 0.0] for k in range(17)])
    with pytest.raises(RuntimeError, match="at most 16 elements"):
        _noalloc(num, pos, "rational", RATIONAL)
    # periodic directions without a lattice, and a degenerate lattice
    num = np.array([6, 8], dtype=np.int32)
    pos = np.array([[0.0, 0.0, 0.0], [2.2, 0.0, 0.0]])
    with pytest.raises(RuntimeError, match="need a lattice"):
        _noalloc(num, pos, "rational", RATIONAL, periodic=np.array([True, True, True]))
    flat = np.array([[10.0, 0.0, 0.0], [0.0, 10.0, 0.0], [0.0, 0.0, 0.0]])
    with pytest.raises(RuntimeError, match="non-degenerate lattice"):
        _noalloc(num, pos, "rational", RATIONAL, lattice=flat, periodic=np.array([True, True, True]))
    # the three-body term is not covered
    with pytest.raises(RuntimeError, match="two-body term only"):
        _noalloc(num, pos, "rational", dict(RATIONAL, s9=1.0))
    # a rejected call leaves the entry point usable
    from dftd3 import synthetic
    mol = synthetic.molecule100(seed=11)
    ref = _regular(mol["numbers"], mol["positions"], "rational", RATIONAL, "fp64", True)
    _check(_noalloc(mol["numbers"], mol["positions"], "rational", RATIONAL), ref, "fp64")
