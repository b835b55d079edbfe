"""Pythonic classes over the B200 DFT-D3 C API.

Drop-in for the reference module ``dftd3.interface`` (python/dftd3/interface.py):
``Structure``, the damping parameter classes, ``DispersionModel`` and
``GeometricCounterpoise`` keep the reference's constructor arguments, keyword
aliases, validation messages and result dictionaries.  The evaluation itself
runs on the GPU through ``dftd3.library``.

Extensions: ``DispersionModel.set_precision`` selects the mixed FP32/FP64 form
and ``BatchedDispersion`` evaluates many independent systems in one call.
"""
from typing import Optional, Sequence

import numpy as np

from . import library


def _rename_kwargs(kwargs: dict, old: str, new: str) -> None:
    if old in kwargs:
        if new in kwargs:
            raise TypeError(f"Keyword '{old}' is an alias of '{new}', pass only one of them")
        kwargs[new] = kwargs.pop(old)


class Structure:
    """Molecular structure data: atomic numbers, Cartesian positions (Bohr) and
    an optional lattice with its periodicity.  The number of atoms, the atomic
    numbers and the periodicity are fixed after construction."""

    _mol = library.StructureHandle.null()

    def __init__(self, numbers: np.ndarray, positions: np.ndarray,
                 lattice: Optional[np.ndarray] = None, periodic: Optional[np.ndarray] = None):
        if positions.size % 3 != 0:
            raise ValueError("Expected tripels of cartesian coordinates")
        if 3 * numbers.size != positions.size:
            raise ValueError("Dimension missmatch between numbers and positions")
        self._natoms = len(numbers)
        _numbers = np.ascontiguousarray(numbers, dtype="i4")
        _positions = np.ascontiguousarray(positions, dtype=float)
        _lattice = None
        if lattice is not None:
            if lattice.size != 9:
                raise ValueError("Invalid lattice provided")
            _lattice = np.ascontiguousarray(lattice, dtype=float)
        _periodic = None
        if periodic is not None:
            if periodic.size != 3:
                raise ValueError("Invalid periodicity provided")
            _periodic = np.ascontiguousarray(periodic, dtype="bool")
        self._mol = library.new_structure(self._natoms, _numbers, _positions, _lattice, _periodic)

    def __len__(self):
        return self._natoms

    def update(self, positions: np.ndarray, lattice: Optional[np.ndarray] = None) -> None:
        """Update the Cartesian coordinates and optionally the lattice (Bohr)."""
        if 3 * len(self) != positions.size:
            raise ValueError("Dimension missmatch for positions")
        _positions = np.ascontiguousarray(positions, dtype=float)
        _lattice = None
        if lattice is not None:
            if lattice.size != 9:
                raise ValueError("Invalid lattice provided")
            _lattice = np.ascontiguousarray(lattice, dtype=float)
        library.update_structure(self._mol, _positions, _lattice)


class DampingParam:
    """Damping parameters of a DFT-D3 method, created either from a method name
    (``method=...``) or from explicit values, never from a mix of both."""

    _param = library.ParamHandle.null()

    def __init__(self, **kwargs):
        if "method" in kwargs and kwargs["method"] is None:
            del kwargs["method"]
        if "method" in kwargs:
            self._param = self.load_param(**kwargs)
        else:
            self._param = self.new_param(**kwargs)

    @staticmethod
    def load_param(method, **kwargs) -> library.ParamHandle:
        raise NotImplementedError("Child class has to define parameter loading")

    @staticmethod
    def new_param(**kwargs) -> library.ParamHandle:
        raise NotImplementedError("Child class has to define parameter construction")


class RationalDampingParam(DampingParam):
    """Rational (Becke-Johnson) damping; the three-body term uses zero damping."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "alpha6", "alp")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_rational_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s8: float, s9: float = 1.0, a1: float, a2: float,
                  alp: float = 14.0) -> library.ParamHandle:
        return library.new_rational_damping(s6, s8, s9, a1, a2, alp)


class ZeroDampingParam(DampingParam):
    """Original (Chai-Head-Gordon type) zero damping of DFT-D3."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "sr6", "rs6")
        _rename_kwargs(kwargs, "sr8", "rs8")
        _rename_kwargs(kwargs, "alpha6", "alp")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_zero_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s8: float, s9: float = 1.0, rs6: float, rs8: float = 1.0,
                  alp: float = 14.0) -> library.ParamHandle:
        return library.new_zero_damping(s6, s8, s9, rs6, rs8, alp)


class ModifiedRationalDampingParam(DampingParam):
    """Modified rational damping: the rational form with re-fitted parameters."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "alpha6", "alp")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_mrational_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s8: float, s9: float = 1.0, a1: float, a2: float,
                  alp: float = 14.0) -> library.ParamHandle:
        return library.new_mrational_damping(s6, s8, s9, a1, a2, alp)


class ModifiedZeroDampingParam(DampingParam):
    """Modified zero damping (mzero.f90)."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "sr6", "rs6")
        _rename_kwargs(kwargs, "sr8", "rs8")
        _rename_kwargs(kwargs, "alpha6", "alp")
        _rename_kwargs(kwargs, "beta", "bet")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_mzero_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s8: float, s9: float = 1.0, rs6: float, rs8: float = 1.0,
                  alp: float = 14.0, bet: float) -> library.ParamHandle:
        return library.new_mzero_damping(s6, s8, s9, rs6, rs8, alp, bet)


class OptimizedPowerDampingParam(DampingParam):
    """Optimized power damping (optimizedpower.f90)."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "alpha6", "alp")
        _rename_kwargs(kwargs, "beta", "bet")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_optimizedpower_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s8: float, s9: float = 1.0, a1: float, a2: float,
                  alp: float = 14.0, bet) -> library.ParamHandle:
        return library.new_optimizedpower_damping(s6, s8, s9, a1, a2, alp, bet)


class CSODampingParam(DampingParam):
    """C6-scaled-only damping (cso.f90)."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "alpha6", "alp")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_cso_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s9: float = 1.0, a1: float, a2: float = 2.5, a3: float = 0.0,
                  a4: float = 6.25, alp: float = 14.0) -> library.ParamHandle:
        return library.new_cso_damping(s6, s9, a1, a2, a3, a4, alp)


class ZDampingParam(DampingParam):
    """Z damping (z.f90): R0 = a1 / (sum of the species indices of the pair)."""

    def __init__(self, **kwargs):
        _rename_kwargs(kwargs, "alpha6", "alp")
        DampingParam.__init__(self, **kwargs)

    @staticmethod
    def load_param(method: str, atm: bool = False) -> library.ParamHandle:
        return library.load_z_damping(method, atm)

    @staticmethod
    def new_param(*, s6: float = 1.0, s8: float = 1.0, s9: float = 1.0, a1: float,
                  alp: float = 14.0) -> library.ParamHandle:
        return library.new_z_damping(s6, s8, s9, a1, alp)


class DispersionModel(Structure):
    """D3 dispersion model bound to its structure; evaluates energy, gradient
    and virial on the GPU."""

    _disp = library.ModelHandle.null()

    def __init__(self, numbers: np.ndarray, positions: np.ndarray,
                 lattice: Optional[np.ndarray] = None, periodic: Optional[np.ndarray] = None):
        Structure.__init__(self, numbers, positions, lattice, periodic)
        self._disp = library.new_d3_model(self._mol)

    def set_realspace_cutoff(self, disp2: float, disp3: float, cn: float, width2: float = 0.0,
                             width3: float = 0.0):
        """Set the real space cutoffs (Bohr) and smoothing widths."""
        library.set_model_realspace_cutoff(self._disp, disp2, disp3, cn, width2, width3)

    def set_ewald_summation(self, rank: int = 0, tolerance: float = 0.0, kcut: float = 0.0,
                            mesh: int = 0) -> None:
        """Reciprocal space summation (reported as not supported)."""
        library.set_model_ewald(self._disp, rank, tolerance, kcut, mesh)

    def set_ghost_atoms(self, ghost_atoms) -> None:
        """Exclude the listed (zero-based) atoms from the dispersion energy."""
        library.set_model_ghost_index(self._disp, np.asarray(ghost_atoms, dtype="i4"))

    def set_work_partition(self, part: int, nparts: int) -> None:
        """Evaluate only part ``part`` of ``nparts`` of the pair and triple loops;
        the parts sum to the complete result."""
        library.set_model_work_partition(self._disp, part, nparts)

    def set_tuning(self, morton_cell: float, pair_split: int, atm_blocks_per_sm: int = 0, atm_mol: int = 0) -> None:
        """Launch shapes (extension, see dftd3_b200_set_model_tuning)."""
        library.set_model_tuning(self._disp, morton_cell, pair_split, atm_blocks_per_sm, atm_mol)

    def set_graph(self, enable: bool = True) -> None:
        """Replay the evaluation as one captured CUDA graph (extension, see
        dftd3_b200_set_model_graph): worth it for many evaluations of one
        structure with new positions."""
        library.set_model_graph(self._disp, enable)

    def set_precision(self, precision: str) -> None:
        """'fp64' (default) or 'mixed' (FP32 pair arithmetic, FP64 accumulation)."""
        modes = {"fp64": library.PRECISION_FP64, "mixed": library.PRECISION_MIXED}
        if precision not in modes:
            raise ValueError(f"Unknown precision '{precision}', expected one of {sorted(modes)}")
        library.set_model_precision(self._disp, modes[precision])

    def get_dispersion(self, param: DampingParam, grad: bool) -> dict:
        """Dispersion energy, and with ``grad`` the gradient and virial."""
        _energy = np.array(0.0)
        _gradient = np.zeros((len(self), 3)) if grad else None
        _sigma = np.zeros((3, 3)) if grad else None
        library.get_dispersion(self._mol, self._disp, param._param, _energy, _gradient, _sigma)
        results = dict(energy=_energy)
        if _gradient is not None:
            results.update(gradient=_gradient)
        if _sigma is not None:
            results.update(virial=_sigma)
        return results

    def get_pairwise_dispersion(self, param: DampingParam) -> dict:
        """Pairwise representation of the dispersion energy: the additive (two-body)
        and non-additive (three-body) energy of every atom pair, FP64."""
        _pair_disp2 = np.zeros((len(self), len(self)))
        _pair_disp3 = np.zeros((len(self), len(self)))
        library.get_pairwise_dispersion(self._mol, self._disp, param._param, _pair_disp2, _pair_disp3)
        return {"additive pairwise energy": _pair_disp2, "non-additive pairwise energy": _pair_disp3}

    def get_hessian(self, param: DampingParam) -> dict:
        """Analytic Hessian of the dispersion energy, (3n, 3n) in Hartree/Bohr^2 (FP64),
        and the energy."""
        _energy = np.array(0.0)
        _hessian = np.zeros((3 * len(self), 3 * len(self)))
        library.get_dispersion_hessian(self._mol, self._disp, param._param, _energy, _hessian)
        return {"energy": _energy, "hessian": _hessian}


class GeometricCounterpoise(Structure):
    """Geometric counter-poise correction (reported as not supported)."""

    _gcp = library.GCPHandle.null()

    def __init__(self, numbers: np.ndarray, positions: np.ndarray, lattice: Optional[np.ndarray] = None,
                 periodic: Optional[np.ndarray] = None, method: Optional[str] = None,
                 basis: Optional[str] = None):
        Structure.__init__(self, numbers, positions, lattice, periodic)
        self._gcp = library.load_gcp_param(self._mol, method, basis)

    def set_realspace_cutoff(self, bas: float, srb: float):
        library.set_gcp_realspace_cutoff(self._gcp, bas, srb)

    def set_work_partition(self, part: int, nparts: int) -> None:
        library.set_gcp_work_partition(self._gcp, part, nparts)

    def get_counterpoise(self, grad: bool) -> dict:
        _energy = np.array(0.0)
        _gradient = np.zeros((len(self), 3)) if grad else None
        _sigma = np.zeros((3, 3)) if grad else None
        library.get_counterpoise(self._mol, self._gcp, _energy, _gradient, _sigma)
        results = dict(energy=_energy)
        if _gradient is not None:
            results.update(gradient=_gradient)
        if _sigma is not None:
            results.update(virial=_sigma)
        return results

    def get_hessian(self) -> dict:
        _energy = np.array(0.0)
        _hessian = np.zeros((3 * len(self), 3 * len(self)))
        library.get_counterpoise_hessian(self._mol, self._gcp, _energy, _hessian)
        return {"energy": _energy, "hessian": _hessian}


class BatchedDispersion:
    """Many independent systems evaluated in one GPU pass (extension).

    ``numbers`` and ``positions`` are sequences with one array per system;
    ``lattices`` (nsys x 3 x 3) and ``periodic`` (nsys x 3) are optional."""

    def __init__(self, numbers: Sequence[np.ndarray], positions: Sequence[np.ndarray],
                 lattices: Optional[np.ndarray] = None, periodic: Optional[np.ndarray] = None):
        self._natoms = np.ascontiguousarray([len(n) for n in numbers], dtype="i4")
        self._offsets = np.concatenate([[0], np.cumsum(self._natoms)])
        _numbers = np.ascontiguousarray(np.concatenate([np.asarray(n) for n in numbers]), dtype="i4")
        self._lattices = None if lattices is None else np.ascontiguousarray(lattices, dtype=float)
        _periodic = None if periodic is None else np.ascontiguousarray(periodic, dtype="bool")
        self._positions = self._flatten(positions)
        self._batch = library.new_batch(self._natoms, _numbers, self._lattices, _periodic)

    def _flatten(self, positions) -> np.ndarray:
        pos = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=float).reshape(-1, 3) for p in positions]))
        if pos.shape[0] != self._offsets[-1]:
            raise ValueError("Dimension missmatch for positions")
        return pos

    def __len__(self):
        return len(self._natoms)

    def set_realspace_cutoff(self, disp2: float, disp3: float, cn: float, width2: float = 0.0,
                             width3: float = 0.0):
        library.set_batch_realspace_cutoff(self._batch, disp2, disp3, cn, width2, width3)

    def set_precision(self, precision: str) -> None:
        modes = {"fp64": library.PRECISION_FP64, "mixed": library.PRECISION_MIXED}
        if precision not in modes:
            raise ValueError(f"Unknown precision '{precision}', expected one of {sorted(modes)}")
        library.set_batch_precision(self._batch, modes[precision])

    def set_graph(self, enable: bool = True) -> None:
        """Replay the pipeline as one captured CUDA graph after the first evaluation."""
        library.set_batch_graph(self._batch, enable)

    def autotune(self, param: DampingParam, grad: bool = True) -> dict:
        """Time the candidate launch shapes on the current positions and keep the fastest."""
        ms = library.autotune_batch(self._batch, param._param, self._positions, grad)
        return dict(library.get_batch_tuning(self._batch), ms=ms)

    def set_tuning(self, morton_cell: float, pair_split: int, atm_blocks_per_sm: int = 0, atm_mol: int = 0) -> None:
        library.set_batch_tuning(self._batch, morton_cell, pair_split, atm_blocks_per_sm, atm_mol)

    def update(self, positions, lattices: Optional[np.ndarray] = None) -> None:
        self._positions = self._flatten(positions)
        if lattices is not None:
            self._lattices = np.ascontiguousarray(lattices, dtype=float)

    def get_dispersion(self, param: DampingParam, grad: bool) -> dict:
        """Per-system energies, and with ``grad`` per-system gradients and virials."""
        nsys = len(self)
        energies = np.zeros(nsys)
        gradient = np.zeros_like(self._positions) if grad else None
        sigma = np.zeros((nsys, 3, 3)) if grad else None
        library.get_dispersion_batched(self._batch, param._param, self._positions, self._lattices,
                                       energies, gradient, sigma)
        out = {"energy": energies}
        if grad:
            out["gradient"] = [gradient[a:b] for a, b in zip(self._offsets[:-1], self._offsets[1:])]
            out["virial"] = sigma
        return out
