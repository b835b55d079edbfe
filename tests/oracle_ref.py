"""ctypes binding of the FP64 CPU oracle (oracle/liboracle_d3.so).

Test infrastructure: the tests use it as the parity checker; the product
library never imports it.  Builds the oracle on first use if it is missing.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
AUTOAA = 0.52917721090380
AATOAU = 1.0 / AUTOAA


class OracleParam(C.Structure):
    _fields_ = [("damping", C.c_int), ("s6", C.c_double), ("s8", C.c_double), ("s9", C.c_double),
                ("a1", C.c_double), ("a2", C.c_double), ("rs6", C.c_double), ("rs8", C.c_double),
                ("alp", C.c_double), ("bet", C.c_double)]


class OracleCutoff(C.Structure):
    _fields_ = [("disp2", C.c_double), ("disp3", C.c_double), ("cn", C.c_double),
                ("width2", C.c_double), ("width3", C.c_double)]


_lib = None
# in-place sum of count doubles over all parts; 0 on success
REDUCER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p)


def lib():
    global _lib
    if _lib is None:
        so = ORACLE_DIR / "liboracle_d3.so"
        if not so.exists():
            subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)
        _lib = C.CDLL(str(so))
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        _lib.oracle_get_dispersion.restype = C.c_int
        _lib.oracle_get_dispersion.argtypes = [
            C.c_int, ip, dp, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(OracleParam),
            C.POINTER(OracleCutoff), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
            C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_get_dispersion_reduced.restype = C.c_int
        _lib.oracle_get_dispersion_reduced.argtypes = [
            C.c_int, ip, dp, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(OracleParam),
            C.POINTER(OracleCutoff), C.c_int, C.c_int, REDUCER, C.c_void_p, C.c_void_p, C.c_void_p,
            C.c_void_p, C.c_void_p]
        _lib.oracle_get_pairwise_dispersion.restype = C.c_int
        _lib.oracle_get_pairwise_dispersion.argtypes = [
            C.c_int, ip, dp, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(OracleParam),
            C.POINTER(OracleCutoff), dp, dp]
        _lib.oracle_get_dispersion_hessian.restype = C.c_int
        _lib.oracle_get_dispersion_hessian.argtypes = [
            C.c_int, ip, dp, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(OracleParam),
            C.POINTER(OracleCutoff), C.c_int, C.c_int, dp]
        _lib.oracle_coordination_number.argtypes = [C.c_int, ip, dp, C.c_void_p, C.c_void_p,
                                                    C.c_double, dp]
        _lib.oracle_weight_references.argtypes = [C.c_int, ip, dp, C.POINTER(C.c_int),
                                                  C.c_void_p, C.c_void_p]
        _lib.oracle_lattice_points.restype = C.c_int
        _lib.oracle_lattice_points.argtypes = [dp, C.c_void_p, C.c_double, C.c_void_p, C.c_int]
        _lib.oracle_wrap_to_central_cell.argtypes = [C.c_int, dp, dp, C.c_void_p]
        _lib.oracle_covalent_radius.restype = C.c_double
        _lib.oracle_covalent_radius.argtypes = [C.c_int]
        _lib.oracle_r4r2.restype = C.c_double
        _lib.oracle_r4r2.argtypes = [C.c_int]
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


DAMPING = {"rational": 0, "mrational": 0, "zero": 1, "mzero": 2, "optimizedpower": 3, "cso": 4, "z": 5}


def make_param(p):
    """Oracle parameter record from a fixture/param dict.  CSO's a3 and a4
    travel in rs6 and rs8, as new_cso_damping stores them (cso.f90:74-90)."""
    kind = p.get("damping", "rational")
    rs6, rs8 = p.get("rs6", 1.0), p.get("rs8", 1.0)
    if kind == "cso":
        rs6, rs8 = p.get("a3", 0.0), p.get("a4", 6.25)
    return OracleParam(DAMPING[kind], p.get("s6", 1.0), p.get("s8", 1.0), p.get("s9", 0.0),
                       p.get("a1", 0.4), p.get("a2", 5.0), rs6, rs8, p.get("alp", 14.0), p.get("bet", 0.0))


def dispersion(numbers, positions, param, lattice=None, periodic=None, grad=True,
               cutoff=(60.0, 40.0, 40.0, 0.0, 0.0), ghost=None, part=0, nparts=1, wrap=True):
    """Evaluate the oracle; positions in Bohr.  Returns a dict like the API's
    get_dispersion plus 'cn', 'dEdcn' and 'energies'."""
    numbers = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.array(positions, dtype=np.float64).reshape(-1, 3).copy()
    nat = len(numbers)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=np.float64).reshape(3, 3)
    per = None
    if periodic is not None:
        per = np.ascontiguousarray([1 if p else 0 for p in np.ravel(periodic)], dtype=np.int32)
    elif lat is not None:
        per = np.ones(3, dtype=np.int32)
    if wrap and per is not None and per.any():
        lib().oracle_wrap_to_central_cell(nat, xyz, lat, _ptr(per))
    ghost_arr = None
    if ghost is not None:
        ghost_arr = np.zeros(nat, dtype=np.int32)
        ghost_arr[np.asarray(ghost, dtype=int)] = 1
    e = np.zeros(1)
    energies = np.zeros(max(nat, 1))
    g = np.zeros((max(nat, 1), 3)) if grad else None
    s = np.zeros((3, 3)) if grad else None
    cn = np.zeros(max(nat, 1))
    dedcn = np.zeros(max(nat, 1))
    prm = make_param(param)
    cut = OracleCutoff(*cutoff)
    rc = lib().oracle_get_dispersion(nat, numbers, xyz, _ptr(lat), _ptr(per), _ptr(ghost_arr),
                                     C.byref(prm), C.byref(cut), part, nparts, _ptr(e),
                                     _ptr(energies), _ptr(g), _ptr(s), _ptr(cn), _ptr(dedcn))
    if rc != 0:
        raise ValueError("oracle: unsupported element")
    out = {"energy": float(e[0]), "energies": energies[:nat], "cn": cn[:nat], "positions": xyz}
    if grad:
        out.update(gradient=g[:nat], virial=s, dEdcn=dedcn[:nat])
    return out


def pairwise_dispersion(numbers, positions, param, lattice=None, periodic=None,
                        cutoff=(60.0, 40.0, 40.0, 0.0, 0.0), ghost=None, wrap=True):
    """Pairwise decomposition of the oracle (positions in Bohr): the
    reference's 'additive pairwise energy' and 'non-additive pairwise energy'
    as (nat, nat) arrays."""
    numbers = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.array(positions, dtype=np.float64).reshape(-1, 3).copy()
    nat = len(numbers)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=np.float64).reshape(3, 3)
    per = None
    if periodic is not None:
        per = np.ascontiguousarray([1 if p else 0 for p in np.ravel(periodic)], dtype=np.int32)
    elif lat is not None:
        per = np.ones(3, dtype=np.int32)
    if wrap and per is not None and per.any():
        lib().oracle_wrap_to_central_cell(nat, xyz, lat, _ptr(per))
    ghost_arr = None
    if ghost is not None:
        ghost_arr = np.zeros(nat, dtype=np.int32)
        ghost_arr[np.asarray(ghost, dtype=int)] = 1
    e2 = np.zeros((max(nat, 1), max(nat, 1)))
    e3 = np.zeros((max(nat, 1), max(nat, 1)))
    prm = make_param(param)
    cut = OracleCutoff(*cutoff)
    rc = lib().oracle_get_pairwise_dispersion(nat, numbers, xyz, _ptr(lat), _ptr(per), _ptr(ghost_arr),
                                              C.byref(prm), C.byref(cut), e2, e3)
    if rc != 0:
        raise ValueError("oracle: unsupported element or damping")
    return {"additive pairwise energy": e2[:nat, :nat], "non-additive pairwise energy": e3[:nat, :nat]}


def hessian(numbers, positions, param, lattice=None, periodic=None, cutoff=(60.0, 40.0, 40.0, 0.0, 0.0),
            ghost=None, part=0, nparts=1, wrap=True):
    """Analytic Hessian of the oracle, (3 nat, 3 nat) in Hartree/Bohr^2."""
    numbers = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.array(positions, dtype=np.float64).reshape(-1, 3).copy()
    nat = len(numbers)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=np.float64).reshape(3, 3)
    per = None
    if periodic is not None:
        per = np.ascontiguousarray([1 if p else 0 for p in np.ravel(periodic)], dtype=np.int32)
    elif lat is not None:
        per = np.ones(3, dtype=np.int32)
    if wrap and per is not None and per.any():
        lib().oracle_wrap_to_central_cell(nat, xyz, lat, _ptr(per))
    ghost_arr = None
    if ghost is not None:
        ghost_arr = np.zeros(nat, dtype=np.int32)
        ghost_arr[np.asarray(ghost, dtype=int)] = 1
    h = np.zeros((3 * max(nat, 1), 3 * max(nat, 1)))
    prm = make_param(param)
    cut = OracleCutoff(*cutoff)
    rc = lib().oracle_get_dispersion_hessian(nat, numbers, xyz, _ptr(lat), _ptr(per), _ptr(ghost_arr),
                                             C.byref(prm), C.byref(cut), part, nparts, h)
    if rc != 0:
        raise ValueError("oracle: unsupported element or damping")
    return h[:3 * nat, :3 * nat]


def coordination_number(numbers, positions, cutoff, lattice=None, periodic=None):
    numbers = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    cn = np.zeros(len(numbers))
    per = None if periodic is None else np.ascontiguousarray(periodic, dtype=np.int32)
    if per is None:
        per = np.zeros(3, dtype=np.int32)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=np.float64)
    lib().oracle_coordination_number(len(numbers), numbers, xyz, _ptr(lat), _ptr(per), cutoff, cn)
    return cn


def weight_references(numbers, cn):
    numbers = np.ascontiguousarray(numbers, dtype=np.int32)
    cn = np.ascontiguousarray(cn, dtype=np.float64)
    mref = C.c_int(0)
    lib().oracle_weight_references(len(numbers), numbers, cn, C.byref(mref), None, None)
    gw = np.zeros((len(numbers), mref.value))
    dgw = np.zeros((len(numbers), mref.value))
    lib().oracle_weight_references(len(numbers), numbers, cn, C.byref(mref), _ptr(gw), _ptr(dgw))
    return gw, dgw


def lattice_points(lattice, periodic, cutoff):
    lat = np.ascontiguousarray(lattice, dtype=np.float64).reshape(3, 3)
    per = np.ascontiguousarray([1 if p else 0 for p in periodic], dtype=np.int32)
    n = lib().oracle_lattice_points(lat, _ptr(per), cutoff, None, 0)
    t = np.zeros((n, 3))
    lib().oracle_lattice_points(lat, _ptr(per), cutoff, _ptr(t), n)
    return t


def dispersion_reduced(numbers, positions, param, reduce, part, nparts, lattice=None, periodic=None, grad=True,
                       cutoff=(60.0, 40.0, 40.0, 0.0, 0.0)):
    """Partitioned oracle evaluation with a reducer (the reference's MPI path):
    `reduce(address, count)` sums count doubles at address over all parts in
    place.  Returns the complete energy, gradient and virial on every part."""
    numbers = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.array(positions, dtype=np.float64).reshape(-1, 3).copy()
    nat = len(numbers)
    lat = None if lattice is None else np.ascontiguousarray(lattice, dtype=np.float64).reshape(3, 3)
    per = None
    if periodic is not None:
        per = np.ascontiguousarray([1 if p else 0 for p in np.ravel(periodic)], dtype=np.int32)
    elif lat is not None:
        per = np.ones(3, dtype=np.int32)
    if per is not None and per.any():
        lib().oracle_wrap_to_central_cell(nat, xyz, lat, _ptr(per))

    def cb(address, count, user):
        try:
            reduce(address, count)
        except Exception:
            return 1
        return 0

    cfun = REDUCER(cb)
    e = np.zeros(1)
    energies = np.zeros(max(nat, 1))
    g = np.zeros((max(nat, 1), 3)) if grad else None
    s = np.zeros((3, 3)) if grad else None
    prm = make_param(param)
    cut = OracleCutoff(*cutoff)
    rc = lib().oracle_get_dispersion_reduced(nat, numbers, xyz, _ptr(lat), _ptr(per), None, C.byref(prm),
                                             C.byref(cut), part, nparts, cfun, None, _ptr(e), _ptr(energies),
                                             _ptr(g), _ptr(s))
    if rc != 0:
        raise RuntimeError(f"oracle: reduced evaluation failed ({rc})")
    out = {"energy": float(e[0]), "energies": energies[:nat]}
    if grad:
        out.update(gradient=g[:nat], virial=s)
    return out
