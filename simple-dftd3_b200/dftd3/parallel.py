"""Distribution of one evaluation over the processes of a torch.distributed
group: the counterpart of the reference's MPI path (dftd3_set_model_mpi_comm,
api.f90:483-506; get_dispersion_mpi_atomic, mpi.f90), with NCCL (GPU
buffers) or gloo (host buffers) in place of MPI.

Every process evaluates its share of the pair and triple loops (pair
ownership of partition.f90:127-147); the coordination numbers and dE/dCN are
summed over the group before they are used (disp.f90:120-126,166-171) and the
results once at the end, so every process receives the complete energies,
gradient and virial.  The library calls the reducer defined here between its
kernel launches (``dftd3_b200_set_batch_reducer``).
"""
from typing import Optional, Sequence

import numpy as np

from . import library


class _DeviceArray:
    """A device buffer described by the CUDA array interface (no copy)."""

    def __init__(self, ptr: int, count: int, stream: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


def allreduce_device(ptr: int, count: int, stream: int, group=None) -> None:
    """Sum a device buffer of float64 in place over the group, ordered on `stream`."""
    import torch
    import torch.distributed as dist
    buf = torch.as_tensor(_DeviceArray(ptr, count, stream), device="cuda")
    ext = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
    with torch.cuda.stream(ext):
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)


def allreduce_host(ptr: int, count: int, group=None) -> None:
    """Sum a host buffer of float64 in place over the group (gloo)."""
    import ctypes
    import torch
    import torch.distributed as dist
    arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), shape=(count,))
    buf = torch.from_numpy(arr)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)


def make_device_reducer(group=None):
    """cffi callback for dftd3_b200_set_batch_reducer over a torch.distributed
    group.  Keep the returned object alive while the batch uses it."""
    ffi = library.ffi

    def reduce(buffer, count, stream, user):
        try:
            allreduce_device(int(ffi.cast("uintptr_t", buffer)), int(count), int(ffi.cast("uintptr_t", stream)),
                             group)
        except Exception:   # reported to the library, which raises in the caller
            return 1
        return 0

    return ffi.callback("dftd3_b200_reducer", reduce)


class ShardedDispersion:
    """Systems evaluated by all processes of a group, each doing 1/world of
    every loop (one GPU per process).

    numbers / positions: one array per system; lattices (nsys, 3, 3) and
    periodic (nsys, 3) optional.  All processes must pass the same inputs.
    """

    def __init__(self, numbers: Sequence[np.ndarray], lattices: Optional[np.ndarray] = None,
                 periodic: Optional[np.ndarray] = None, group=None, precision: str = "mixed",
                 tuning: Optional[tuple] = None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.natoms = np.ascontiguousarray([len(n) for n in numbers], dtype=np.int32)
        nums = np.ascontiguousarray(np.concatenate([np.asarray(n) for n in numbers]), dtype=np.int32)
        lat = None if lattices is None else np.ascontiguousarray(lattices, dtype=float).reshape(-1, 3, 3)
        per = None if periodic is None else np.ascontiguousarray(periodic, dtype=bool)
        self.lattices = lat
        self.batch = library.new_batch(self.natoms, nums, lat, per)
        library.set_batch_precision(self.batch, library.PRECISION_MIXED if precision == "mixed"
                                    else library.PRECISION_FP64)
        # the parts must order the atoms alike: fixed launch shapes on every process
        library.set_batch_tuning(self.batch, *(tuning or (0.0, 0, 0, 0)))
        self._reducer = make_device_reducer(group)
        library.set_batch_reducer(self.batch, self._reducer, self.rank, self.world)

    def set_realspace_cutoff(self, disp2, disp3, cn, width2=0.0, width3=0.0):
        library.set_batch_realspace_cutoff(self.batch, disp2, disp3, cn, width2, width3)

    def get_dispersion(self, param, d_positions, d_energies, d_gradient=0, d_sigma=0, stream=0):
        """Device-pointer evaluation (see library.get_dispersion_device)."""
        library.get_dispersion_device(self.batch, param, d_positions, None, d_energies, d_gradient, d_sigma, 0,
                                      stream)
