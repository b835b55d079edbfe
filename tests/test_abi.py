"""The C-ABI library loads, exports every entry point the public headers
declare, and its host-side logic (argument checks, structure handling, error
convention) behaves like the reference API -- all without a GPU."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "simple-dftd3_b200" / "lib" / "libsdftd3_b200.so"


def _declared(header):
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / header).read_text(), flags=re.S)
    # drop preprocessor definitions (the _Generic dftd3_delete macro)
    text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
    return sorted(set(re.findall(r"\b(dftd3_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def clib():
    if not LIB.exists():
        import subprocess, sys
        subprocess.run([sys.executable, str(ROOT / "simple-dftd3_b200" / "build.py")], check=True)
    return ctypes.CDLL(str(LIB))


@pytest.mark.parametrize("header", ["s-dftd3.h", "dftd3_b200.h"])
def test_exports_every_declared_symbol(clib, header):
    names = _declared(header)
    assert names
    missing = [n for n in names if not hasattr(clib, n)]
    assert not missing, missing


def test_reference_entry_points_complete():
    """Every dftd3_* entry point of the reference API is declared."""
    names = set(_declared("s-dftd3.h"))
    required = {
        "dftd3_get_version", "dftd3_new_error", "dftd3_check_error", "dftd3_get_error",
        "dftd3_delete_error", "dftd3_new_structure", "dftd3_delete_structure",
        "dftd3_update_structure", "dftd3_new_d3_model", "dftd3_set_model_realspace_cutoff",
        "dftd3_set_model_realspace_cutoff_smooth", "dftd3_set_model_ghost_index",
        "dftd3_delete_model", "dftd3_new_rational_damping", "dftd3_new_zero_damping",
        "dftd3_delete_param", "dftd3_get_dispersion", "dftd3_set_model_work_partition",
    }
    assert required <= names


def test_version_and_features():
    from dftd3 import library
    assert library.get_api_version() == "1.6.0"
    assert not library.lib.dftd3_has_feature(library.ffi.new("char[]", b"mpi"))


def test_structure_checks():
    """Validation of python/dftd3/test_interface.py:197-229, host side only."""
    from dftd3.interface import Structure, DispersionModel
    numbers = np.array([6, 7, 6, 1])
    positions = np.array([[0.0, 0.0, 0.0], [2.5, 0.0, 0.0], [0.0, 2.6, 0.0], [0.0, 0.0, 2.0]])
    with pytest.raises(RuntimeError, match="Too close interatomic distances found"):
        Structure(numbers, np.zeros((4, 3)))
    with pytest.raises(ValueError, match="Dimension missmatch"):
        Structure(np.array([1, 1, 1]), positions)
    with pytest.raises(ValueError, match="Expected tripels"):
        Structure(numbers, np.arange(7.0))
    inst = DispersionModel(numbers, positions)
    with pytest.raises(ValueError, match="Dimension missmatch for positions"):
        inst.update(np.arange(7.0))
    with pytest.raises(ValueError, match="Invalid lattice provided"):
        inst.update(positions, np.arange(7.0))
    with pytest.raises(RuntimeError, match="Too close interatomic distances found"):
        inst.update(np.zeros((4, 3)))


def test_model_setup_errors():
    from dftd3.interface import DispersionModel, RationalDampingParam, ModifiedZeroDampingParam
    numbers = np.array([6, 8])
    positions = np.array([[0.0, 0.0, 0.0], [2.1, 0.0, 0.0]])
    model = DispersionModel(numbers, positions)
    with pytest.raises(RuntimeError, match="Invalid dispersion work partition"):
        model.set_work_partition(3, 3)
    with pytest.raises(RuntimeError, match="Index out of bounds"):
        model.set_ghost_atoms([5])
    ModifiedZeroDampingParam(s8=1.0, rs6=1.2, bet=1.0)
    with pytest.raises(TypeError, match="s8"):
        RationalDampingParam(a1=0.4, a2=5.0)
    with pytest.raises(TypeError, match="a1"):
        RationalDampingParam(s8=1.0, a2=5.0)
    with pytest.raises(ValueError, match="Unknown precision"):
        model.set_precision("fp16")


def test_null_handles():
    """A NULL handle sets the reference's messages (api.f90:1056-1081)."""
    from dftd3 import library as L
    err = L.new_error()
    e = np.zeros(1)
    L.lib.dftd3_get_dispersion(err, L.ffi.NULL, L.ffi.NULL, L.ffi.NULL, L.ffi.cast("double*", e.ctypes.data),
                               L.ffi.NULL, L.ffi.NULL)
    assert L.lib.dftd3_check_error(err) == 1
    buf = L.ffi.new("char[]", 512)
    L.lib.dftd3_get_error(err, buf, L.ffi.NULL)
    assert L.ffi.string(buf).decode() == "Molecular structure data is missing"
    # a NULL error handle returns silently
    L.lib.dftd3_get_dispersion(L.ffi.NULL, L.ffi.NULL, L.ffi.NULL, L.ffi.NULL, L.ffi.NULL, L.ffi.NULL, L.ffi.NULL)
    assert L.lib.dftd3_check_error(L.ffi.NULL) == 2


def test_error_buffer_truncation():
    from dftd3 import library as L
    err = L.new_error()
    L.lib.dftd3_set_model_work_partition(err, L.ffi.NULL, 0, 1)
    buf = L.ffi.new("char[]", 8)
    size = L.ffi.new("int*", 8)
    L.lib.dftd3_get_error(err, buf, size)
    assert L.ffi.string(buf).decode() == "D3 disp"


def test_family_constructor_arguments():
    """Insufficient arguments of the other families' constructors raise
    TypeError naming the missing parameter (test_interface.py:147-200)."""
    from dftd3.interface import ModifiedZeroDampingParam, OptimizedPowerDampingParam, ZDampingParam
    with pytest.raises(TypeError):
        ModifiedZeroDampingParam()
    with pytest.raises(TypeError, match="s8"):
        ModifiedZeroDampingParam(rs6=1.2, bet=1.0)
    with pytest.raises(TypeError, match="rs6"):
        ModifiedZeroDampingParam(s8=1.0, bet=1.0)
    with pytest.raises(TypeError, match="bet"):
        ModifiedZeroDampingParam(s8=1.0, rs6=1.2)
    with pytest.raises(TypeError):
        ModifiedZeroDampingParam(s8=1.0, rs6=1.2, bet=1.0, method="abc")
    with pytest.raises(TypeError):
        OptimizedPowerDampingParam()
    with pytest.raises(TypeError, match="s8"):
        OptimizedPowerDampingParam(a1=0.3, a2=4.2, bet=1.0)
    with pytest.raises(TypeError, match="a1"):
        OptimizedPowerDampingParam(s8=1.0, a2=4.2, bet=1.0)
    with pytest.raises(TypeError, match="a2"):
        OptimizedPowerDampingParam(s8=1.0, a1=0.3, bet=1.0)
    with pytest.raises(TypeError, match="bet"):
        OptimizedPowerDampingParam(s8=1.0, a1=0.3, a2=4.2)
    with pytest.raises(TypeError):
        OptimizedPowerDampingParam(s8=1.0, a1=0.3, a2=4.2, bet=1.0, method="abc")
    with pytest.raises(TypeError):
        ZDampingParam()
    with pytest.raises(TypeError, match="a1"):
        ZDampingParam(s8=1.0)
    with pytest.raises(TypeError):
        ZDampingParam(a1=200770.0, method="abc")


def test_pairwise_and_hessian_argument_errors():
    """dftd3_get_pairwise_dispersion and dftd3_get_dispersion_hessian check
    their handles before any device work (api.f90:1115-1236)."""
    from dftd3 import library as L
    from dftd3.interface import RationalDampingParam

    def message(call, *args):
        err = L.new_error()
        call(err, *args)
        assert L.lib.dftd3_check_error(err) == 1
        buf = L.ffi.new("char[]", 512)
        L.lib.dftd3_get_error(err, buf, L.ffi.NULL)
        return L.ffi.string(buf).decode()

    n = L.ffi.NULL
    e = np.zeros(4)
    p = L.ffi.cast("double*", e.ctypes.data)
    assert message(L.lib.dftd3_get_pairwise_dispersion, n, n, n, p, p) == "Molecular structure data is missing"
    assert message(L.lib.dftd3_get_dispersion_hessian, n, n, n, p, p) == "Molecular structure data is missing"
    numbers = np.array([8, 1, 1], dtype=np.int32)
    xyz = np.array([[0.0, 0.0, 0.0], [1.8, 0.0, 0.0], [-0.5, 1.7, 0.0]])
    mol = L.new_structure(3, numbers, xyz, None, None)
    disp = L.new_d3_model(mol)
    assert message(L.lib.dftd3_get_pairwise_dispersion, mol.handle, disp.handle, n, p, p) == \
        "Damping parameters are missing"
    param = RationalDampingParam(method="pbe0")._param
    assert message(L.lib.dftd3_get_pairwise_dispersion, mol.handle, disp.handle, param.handle, p, n) == \
        "Pairwise energy arrays are missing"
    assert message(L.lib.dftd3_get_dispersion_hessian, mol.handle, disp.handle, param.handle, p, n) == \
        "Hessian array is missing"
    assert message(L.lib.dftd3_b200_set_model_graph, n, 1) == "D3 dispersion model is missing"
