"""Distribution of dispersion work over the processes of a torch.distributed
group (one GPU per process), with NCCL (GPU buffers) or gloo (host buffers).

* One large system (ShardedDispersion): the counterpart of the reference's
  MPI path (dftd3_set_model_mpi_comm, api.f90:483-506;
  get_dispersion_mpi_atomic, mpi.f90).  Every process evaluates its share of
  the pair and triple loops (pair ownership of partition.f90:127-147); the
  coordination numbers and dE/dCN are summed over the group before they are
  used (disp.f90:120-126,166-171) and the results once at the end, so every
  process receives the complete energies, gradient and virial.  The library
  calls the reducer defined here between its kernel launches
  (``dftd3_b200_set_batch_reducer``).
* Many independent systems (shard_systems, gather_results): whole systems
  are dealt to the processes in bins of about equal cost, each process
  evaluates its bin as one batch with no exchange during the evaluation, and
  the per-system results are gathered once at the end if every process needs
  them.
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


def system_cost(natoms: int, periodic: bool = False) -> float:
    """Relative cost of one system: its pair work plus its triple work (the
    triple loop dominates from a few dozen atoms on).  Periodic systems
    count their lattice images through a larger effective atom count."""
    n = float(natoms) * (8.0 if periodic else 1.0)
    return n * n + n * n * n / 64.0


def shard_systems(costs: Sequence[float], nparts: int) -> list:
    """Deal systems to nparts bins of about equal total cost: the largest
    system first, each to the bin with the smallest total so far (ties to
    the lowest bin).  Returns one ascending list of system indices per bin;
    every process computing it from the same costs gets the same bins."""
    if nparts < 1:
        raise ValueError("nparts must be positive")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * nparts
    bins = [[] for _ in range(nparts)]
    for k in order:
        b = min(range(nparts), key=lambda q: (load[q], q))
        bins[b].append(k)
        load[b] += float(costs[k])
    return [sorted(b) for b in bins]


def gather_results(local: dict, indices: Sequence[int], nsys: int, group=None) -> dict:
    """Per-system results of every process's bin, in system order, on every
    process: ``local`` holds this process's "energy" (len(indices)) and
    optionally "gradient" (a list of (n_k, 3) arrays) and "virial"
    ((len(indices), 3, 3)); ``indices`` are its systems.  One all-gather of
    host objects (works with the gloo and the NCCL backend)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    payload = {"indices": list(indices), "energy": np.asarray(local["energy"], dtype=float).tolist()}
    if "gradient" in local:
        payload["gradient"] = [np.asarray(g, dtype=float).tolist() for g in local["gradient"]]
        payload["virial"] = np.asarray(local["virial"], dtype=float).tolist()
    dist.all_gather_object(parts, payload, group=group)
    energy = np.zeros(nsys)
    gradient = [None] * nsys if "gradient" in local else None
    virial = np.zeros((nsys, 3, 3)) if "gradient" in local else None
    for part in parts:
        for pos, k in enumerate(part["indices"]):
            energy[k] = part["energy"][pos]
            if gradient is not None:
                gradient[k] = np.asarray(part["gradient"][pos])
                virial[k] = np.asarray(part["virial"][pos])
    out = {"energy": energy}
    if gradient is not None:
        out.update(gradient=gradient, virial=virial)
    return out
