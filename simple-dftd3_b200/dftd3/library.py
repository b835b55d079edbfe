"""Thin cffi wrapper around the B200 DFT-D3 shared library.

Mirrors the reference module ``dftd3.library`` (python/dftd3/library.py): the
same handle classes, ``error_check`` convention (C errors become
``RuntimeError`` with the library's message) and one function per C entry
point.  The cffi declarations are read from ``include/s-dftd3.h`` and
``include/dftd3_b200.h`` (ABI mode, no compiled extension module); the shared
library is the in-tree build ``lib/libsdftd3_b200.so``.  Importing fails loudly
if the library is missing: there is no CPU fallback.
"""
import functools
import os
import re
from pathlib import Path
from typing import Optional

import numpy as np
from cffi import FFI

_PKG = Path(__file__).resolve().parents[1]
_INCLUDE = _PKG.parent / "include"
_LIBPATH = Path(os.environ.get("DFTD3_B200_LIBRARY", _PKG / "lib" / "libsdftd3_b200.so"))


def _cdef_from_header(text: str) -> str:
    """Strip the preprocessor parts of the public headers for cffi.cdef."""
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out, skip = [], False
    for line in text.splitlines():
        stripped = line.strip()
        if skip:
            skip = stripped.endswith("\\")
            continue
        if stripped.startswith("#"):
            skip = stripped.endswith("\\")
            continue
        out.append(line)
    text = "\n".join(out)
    text = re.sub(r"\bSDFTD3_API_(ENTRY|CALL)\b", "", text)
    text = re.sub(r"\bSDFTD3_API_SUFFIX__V_\d+_\d+\b", "", text)
    text = re.sub(r"\(\s*\)", "(void)", text)
    return text


ffi = FFI()
ffi.cdef(_cdef_from_header((_INCLUDE / "s-dftd3.h").read_text()))
ffi.cdef(_cdef_from_header((_INCLUDE / "dftd3_b200.h").read_text()))

if not _LIBPATH.exists():
    raise ImportError(
        f"DFT-D3 B200 library not found at {_LIBPATH}; build it with "
        "'python simple-dftd3_b200/build.py'"
    )
lib = ffi.dlopen(str(_LIBPATH))

PRECISION_FP64 = 0
PRECISION_MIXED = 1


def get_api_version() -> str:
    """Library version as a semantic version string."""
    api_version = lib.dftd3_get_version()
    return "{}.{}.{}".format(api_version // 10000, api_version % 10000 // 100, api_version % 100)


class Handle:
    def __init__(self, handle):
        self.handle = handle

    @classmethod
    def with_gc(cls, handle):
        return cls(ffi.gc(handle, cls._delete))

    @classmethod
    def null(cls):
        return cls(ffi.NULL)

    @staticmethod
    def _delete(handle):
        raise NotImplementedError("Delete function not implemented")


class StructureHandle(Handle):
    @staticmethod
    def _delete(handle):
        ptr = ffi.new("dftd3_structure *")
        ptr[0] = handle
        lib.dftd3_delete_structure(ptr)


class ModelHandle(Handle):
    @staticmethod
    def _delete(handle):
        ptr = ffi.new("dftd3_model *")
        ptr[0] = handle
        lib.dftd3_delete_model(ptr)


class ParamHandle(Handle):
    @staticmethod
    def _delete(handle):
        ptr = ffi.new("dftd3_param *")
        ptr[0] = handle
        lib.dftd3_delete_param(ptr)


class GCPHandle(Handle):
    @staticmethod
    def _delete(handle):
        ptr = ffi.new("dftd3_gcp *")
        ptr[0] = handle
        lib.dftd3_delete_gcp(ptr)


class BatchHandle(Handle):
    @staticmethod
    def _delete(handle):
        ptr = ffi.new("dftd3_b200_batch *")
        ptr[0] = handle
        lib.dftd3_b200_delete_batch(ptr)


def _delete_error(err):
    ptr = ffi.new("dftd3_error *")
    ptr[0] = err
    lib.dftd3_delete_error(ptr)


def new_error():
    """Create new error handle object"""
    return ffi.gc(lib.dftd3_new_error(), _delete_error)


def error_check(func):
    """Run a library function with a fresh error handle, raise on error."""

    @functools.wraps(func)
    def handle_error(*args, **kwargs):
        _err = new_error()
        value = func(_err, *args, **kwargs)
        if lib.dftd3_check_error(_err):
            _message = ffi.new("char[]", 512)
            lib.dftd3_get_error(_err, _message, ffi.NULL)
            raise RuntimeError(ffi.string(_message).decode())
        return value

    return handle_error


def new_structure(natoms: int, numbers: np.ndarray, positions: np.ndarray,
                  lattice: Optional[np.ndarray], periodic: Optional[np.ndarray]) -> StructureHandle:
    return StructureHandle.with_gc(
        error_check(lib.dftd3_new_structure)(
            natoms, _cast("int*", numbers), _cast("double*", positions),
            _cast("double*", lattice), _cast("bool*", periodic)))


def new_d3_model(mol: StructureHandle) -> ModelHandle:
    return ModelHandle.with_gc(error_check(lib.dftd3_new_d3_model)(mol.handle))


def set_model_realspace_cutoff(disp: ModelHandle, disp2: float, disp3: float, cn: float,
                               width2: float = 0.0, width3: float = 0.0) -> None:
    error_check(lib.dftd3_set_model_realspace_cutoff_smooth)(disp.handle, disp2, disp3, cn, width2, width3)


def set_model_ewald(disp: ModelHandle, rank: int, tolerance: float, kcut: float, mesh: int) -> None:
    error_check(lib.dftd3_set_model_ewald)(disp.handle, rank, tolerance, kcut, mesh)


def set_model_ghost_index(disp: ModelHandle, ghost: np.ndarray) -> None:
    if ghost.size == 0:
        return
    error_check(lib.dftd3_set_model_ghost_index)(disp.handle, _cast("int*", ghost), ghost.size)


def set_model_work_partition(disp: ModelHandle, part: int, nparts: int) -> None:
    error_check(lib.dftd3_set_model_work_partition)(disp.handle, part, nparts)


def set_model_precision(disp: ModelHandle, precision: int) -> None:
    error_check(lib.dftd3_b200_set_model_precision)(disp.handle, precision)


def set_model_graph(disp: ModelHandle, enable: bool) -> None:
    error_check(lib.dftd3_b200_set_model_graph)(disp.handle, 1 if enable else 0)


def new_zero_damping(s6: float, s8: float, s9: float, rs6: float, rs8: float, alp: float) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_new_zero_damping)(s6, s8, s9, rs6, rs8, alp))


def load_zero_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_zero_damping)(_char(method), atm))


def new_rational_damping(s6: float, s8: float, s9: float, a1: float, a2: float, alp: float) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_new_rational_damping)(s6, s8, s9, a1, a2, alp))


def load_rational_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_rational_damping)(_char(method), atm))


def new_mzero_damping(s6, s8, s9, rs6, rs8, alp, bet) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_new_mzero_damping)(s6, s8, s9, rs6, rs8, alp, bet))


def load_mzero_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_mzero_damping)(_char(method), atm))


def new_mrational_damping(s6, s8, s9, a1, a2, alp) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_new_mrational_damping)(s6, s8, s9, a1, a2, alp))


def load_mrational_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_mrational_damping)(_char(method), atm))


def new_optimizedpower_damping(s6, s8, s9, a1, a2, alp, bet) -> ParamHandle:
    return ParamHandle.with_gc(
        error_check(lib.dftd3_new_optimizedpower_damping)(s6, s8, s9, a1, a2, alp, bet))


def load_optimizedpower_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_optimizedpower_damping)(_char(method), atm))


def new_cso_damping(s6, s9, a1, a2, a3, a4, alp) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_new_cso_damping)(s6, s9, a1, a2, a3, a4, alp))


def load_cso_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_cso_damping)(_char(method), atm))


def new_z_damping(s6, s8, s9, a1, alp) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_new_z_damping)(s6, s8, s9, a1, alp))


def load_z_damping(method: str, atm: bool) -> ParamHandle:
    return ParamHandle.with_gc(error_check(lib.dftd3_load_z_damping)(_char(method), atm))


def update_structure(mol: StructureHandle, positions: np.ndarray, lattice: Optional[np.ndarray]) -> None:
    return error_check(lib.dftd3_update_structure)(
        mol.handle, _cast("double*", positions), _cast("double*", lattice))


def get_dispersion(mol: StructureHandle, disp: ModelHandle, param: ParamHandle, energy: np.ndarray,
                   gradient: Optional[np.ndarray], sigma: Optional[np.ndarray]) -> None:
    return error_check(lib.dftd3_get_dispersion)(
        mol.handle, disp.handle, param.handle, _cast("double*", energy),
        _cast("double*", gradient), _cast("double*", sigma))


def get_pairwise_dispersion(mol, disp, param, pair_energy2, pair_energy3) -> None:
    return error_check(lib.dftd3_get_pairwise_dispersion)(
        mol.handle, disp.handle, param.handle, _cast("double*", pair_energy2), _cast("double*", pair_energy3))


def get_dispersion_hessian(mol, disp, param, energy, hessian) -> None:
    return error_check(lib.dftd3_get_dispersion_hessian)(
        mol.handle, disp.handle, param.handle, _cast("double*", energy), _cast("double*", hessian))


def load_gcp_param(mol: StructureHandle, method: Optional[str], basis: Optional[str]) -> GCPHandle:
    return GCPHandle.with_gc(error_check(lib.dftd3_load_gcp_param)(mol.handle, _char(method), _char(basis)))


def set_gcp_realspace_cutoff(gcp: GCPHandle, bas: float, srb: float) -> None:
    error_check(lib.dftd3_set_gcp_realspace_cutoff)(gcp.handle, bas, srb)


def set_gcp_work_partition(gcp: GCPHandle, part: int, nparts: int) -> None:
    error_check(lib.dftd3_set_gcp_work_partition)(gcp.handle, part, nparts)


def get_counterpoise(mol, gcp, energy, gradient, sigma) -> None:
    return error_check(lib.dftd3_get_counterpoise)(
        mol.handle, gcp.handle, _cast("double*", energy), _cast("double*", gradient), _cast("double*", sigma))


def get_counterpoise_hessian(mol, gcp, energy, hessian) -> None:
    return error_check(lib.dftd3_get_counterpoise_hessian)(
        mol.handle, gcp.handle, _cast("double*", energy), _cast("double*", hessian))


# ------------------------------------------------------------- extensions --

def new_batch(natoms: np.ndarray, numbers: np.ndarray, lattices: Optional[np.ndarray],
              periodic: Optional[np.ndarray]) -> BatchHandle:
    return BatchHandle.with_gc(
        error_check(lib.dftd3_b200_new_batch)(
            natoms.size, _cast("int*", natoms), _cast("int*", numbers),
            _cast("double*", lattices), _cast("bool*", periodic)))


def set_batch_realspace_cutoff(batch: BatchHandle, disp2, disp3, cn, width2=0.0, width3=0.0) -> None:
    error_check(lib.dftd3_b200_set_batch_realspace_cutoff)(batch.handle, disp2, disp3, cn, width2, width3)


def set_batch_precision(batch: BatchHandle, precision: int) -> None:
    error_check(lib.dftd3_b200_set_batch_precision)(batch.handle, precision)


def set_batch_counting(batch: BatchHandle, enable: bool) -> None:
    error_check(lib.dftd3_b200_set_batch_counting)(batch.handle, 1 if enable else 0)


def get_batch_counts(batch: BatchHandle) -> np.ndarray:
    counts = np.zeros(3, dtype=np.int64)
    error_check(lib.dftd3_b200_get_batch_counts)(batch.handle, _cast("long long*", counts))
    return counts


def set_batch_profiling(batch: BatchHandle, enable: bool) -> None:
    error_check(lib.dftd3_b200_set_batch_profiling)(batch.handle, 1 if enable else 0)


STAGES = ("split", "cn", "weights", "two_body", "three_body", "cn_chain", "reduce", "two_body_kernel",
          "three_body_kernel")


def get_batch_graph_kernels(batch: BatchHandle) -> int:
    """Kernel launches of one replay of the batch's captured CUDA graph (0 if none)."""
    n = np.zeros(1, dtype=np.int64)
    error_check(lib.dftd3_b200_get_batch_graph_kernels)(batch.handle, _cast("long long*", n))
    return int(n[0])


def get_batch_stage_times(batch: BatchHandle) -> dict:
    ms = np.zeros(len(STAGES))
    error_check(lib.dftd3_b200_get_batch_stage_times)(batch.handle, _cast("double*", ms))
    return dict(zip(STAGES, ms))


def set_batch_graph(batch: BatchHandle, enable: bool) -> None:
    error_check(lib.dftd3_b200_set_batch_graph)(batch.handle, 1 if enable else 0)


TUNING = ("morton_cell", "pair_split", "atm_blocks_per_sm", "atm_mol")


def set_batch_tuning(batch: BatchHandle, morton_cell: float, pair_split: int, atm_blocks_per_sm: int,
                     atm_mol: int = 0) -> None:
    t = np.array([morton_cell, pair_split, atm_blocks_per_sm, atm_mol], dtype=float)
    error_check(lib.dftd3_b200_set_batch_tuning)(batch.handle, _cast("double*", t))


def set_model_tuning(disp: ModelHandle, morton_cell: float, pair_split: int, atm_blocks_per_sm: int,
                     atm_mol: int = 0) -> None:
    t = np.array([morton_cell, pair_split, atm_blocks_per_sm, atm_mol], dtype=float)
    error_check(lib.dftd3_b200_set_model_tuning)(disp.handle, _cast("double*", t))


def get_batch_tuning(batch: BatchHandle) -> dict:
    t = np.zeros(4)
    error_check(lib.dftd3_b200_get_batch_tuning)(batch.handle, _cast("double*", t))
    return dict(zip(TUNING, (float(t[0]), int(t[1]), int(t[2]), int(t[3]))))


def autotune_batch(batch: BatchHandle, param: ParamHandle, positions: np.ndarray, grad: bool) -> float:
    """Pick the fastest launch shape on these positions; returns its time in ms."""
    return float(error_check(lib.dftd3_b200_autotune_batch)(
        batch.handle, param.handle, _cast("double*", positions), 1 if grad else 0))


def set_batch_reducer(batch: BatchHandle, reducer, part: int, nparts: int) -> None:
    """reducer: a cffi callback of type dftd3_b200_reducer (keep it alive), or None."""
    error_check(lib.dftd3_b200_set_batch_reducer)(batch.handle, reducer if reducer is not None else ffi.NULL,
                                                  ffi.NULL, part, nparts)


PARAM_FIELDS = ("s6", "s8", "s9", "a1", "a2", "rs6", "rs8", "alp", "bet")
# DFTD3_B200_DAMPING_* in kind order; the modified rational form is "rational"
DAMPING_KINDS = ("rational", "zero", "mzero", "optimizedpower", "cso", "z")


def get_param_values(param: ParamHandle) -> dict:
    """Damping kind and values of a parameter handle (CSO: a3 and a4 in the
    rs6 and rs8 places)."""
    kind = ffi.new("int*")
    v = np.zeros(len(PARAM_FIELDS))
    error_check(lib.dftd3_b200_get_param_values)(param.handle, kind, _cast("double*", v))
    return dict(zip(PARAM_FIELDS, v.tolist()), damping=DAMPING_KINDS[kind[0]])


def fma_peak(precision: int) -> float:
    """Measured FMA throughput (TFLOP/s) of the FP64 or FP32 pipe."""
    return float(error_check(lib.dftd3_b200_fma_peak)(precision))


def get_dispersion_batched(batch: BatchHandle, param: ParamHandle, positions: np.ndarray,
                           lattices: Optional[np.ndarray], energies: np.ndarray,
                           gradient: Optional[np.ndarray], sigma: Optional[np.ndarray]) -> None:
    error_check(lib.dftd3_b200_get_dispersion_batched)(
        batch.handle, param.handle, _cast("double*", positions), _cast("double*", lattices),
        _cast("double*", energies), _cast("double*", gradient), _cast("double*", sigma))


def get_dispersion_device(batch: BatchHandle, param: ParamHandle, d_positions: int,
                          lattices: Optional[np.ndarray], d_energies: int, d_gradient: int,
                          d_sigma: int, d_param_grad: int, stream: int) -> None:
    """Device-pointer evaluation; pointers are integers (0 for NULL)."""
    error_check(lib.dftd3_b200_get_dispersion_device)(
        batch.handle, param.handle, ffi.cast("double*", d_positions), _cast("double*", lattices),
        ffi.cast("double*", d_energies), ffi.cast("double*", d_gradient), ffi.cast("double*", d_sigma),
        ffi.cast("double*", d_param_grad), ffi.cast("void*", stream))


def _char(value: Optional[str]):
    return ffi.new("char[]", value.encode()) if value is not None else ffi.NULL


def _cast(ctype: str, array: Optional[np.ndarray]):
    return ffi.cast(ctype, array.ctypes.data) if array is not None else ffi.NULL
