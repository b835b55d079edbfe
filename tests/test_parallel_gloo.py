"""Partitioned evaluation over several processes, on the CPU.

The reference's MPI path (partitioned pair/triple loops, CN and dE/dCN summed
over the parts before use, results summed at the end: disp.f90:120-171,
mpi.f90) is the protocol the GPU engine follows with its reducer.  Here the
FP64 oracle runs that protocol with (a) the product's torch.distributed
reducer over gloo in two processes and (b) a thread exchange in one process,
and every part must receive the serial result."""
import os
import socket
import threading

import numpy as np
import pytest

import oracle_ref as O

CUT = (25.0, 14.0, 20.0, 0.0, 0.0)


def _cell(seed=4, n=20):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(seed)
    lat = S.triclinic(9.5, 10.0, 10.5, 87.0, 91.0, 94.0)
    num = rng.choice([1, 6, 8], size=n).astype(np.int32)
    pos = S.pack_cell(rng, n, lat, 2.0)
    return num, pos, lat


PARAMS = {
    "rational_atm": dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, s9=1.0, alp=14.0),
    "zero": dict(damping="zero", s6=1.0, s8=1.703, rs6=1.261, rs8=1.0, s9=0.0, alp=14.0),
}


def _compare(res, ref):
    assert abs(res["energy"] - ref["energy"]) <= 1e-12 * abs(ref["energy"])
    assert np.abs(res["gradient"] - ref["gradient"]).max() <= 1e-12 * np.abs(ref["gradient"]).max()
    assert np.abs(res["virial"] - ref["virial"]).max() <= 1e-12 * np.abs(ref["virial"]).max()


@pytest.mark.parametrize("name", sorted(PARAMS))
def test_thread_parts_match_serial(name):
    """Three parts in one process; the reducer sums through a host exchange."""
    num, pos, lat = _cell()
    par = PARAMS[name]
    ref = O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=CUT)
    nparts = 3
    barrier = threading.Barrier(nparts)
    slots = [None] * nparts
    out = [None] * nparts

    def worker(part):
        import ctypes

        def reduce(address, count):
            arr = np.ctypeslib.as_array(ctypes.cast(address, ctypes.POINTER(ctypes.c_double)), shape=(count,))
            slots[part] = arr.copy()
            barrier.wait()
            total = np.sum(slots, axis=0)
            barrier.wait()
            arr[:] = total

        out[part] = O.dispersion_reduced(num, pos, par, reduce, part, nparts, lattice=lat, periodic=[True] * 3,
                                         cutoff=CUT)

    threads = [threading.Thread(target=worker, args=(p,)) for p in range(nparts)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for r in out:
        _compare(r, ref)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, name, queue):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root / "tests"), str(root / "simple-dftd3_b200")]
    import datetime
    import torch.distributed as dist
    import oracle_ref
    from dftd3 import parallel
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        num, pos, lat = _cell()
        res = oracle_ref.dispersion_reduced(num, pos, PARAMS[name], lambda a, c: parallel.allreduce_host(a, c),
                                            rank, world, lattice=lat, periodic=[True] * 3, cutoff=CUT)
        queue.put((rank, res["energy"], res["gradient"], res["virial"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", sorted(PARAMS))
def test_gloo_two_ranks_match_serial(name):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, name, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    num, pos, lat = _cell()
    ref = O.dispersion(num, pos, PARAMS[name], lattice=lat, periodic=[True] * 3, cutoff=CUT)
    for _, e, g, s in results:
        _compare({"energy": e, "gradient": g, "virial": s}, ref)


def test_partition_parts_differ_from_serial():
    """Without the final sum a part holds only its share (the partition is real)."""
    num, pos, lat = _cell()
    par = PARAMS["rational_atm"]
    ref = O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=CUT)
    parts = [O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=CUT, part=p, nparts=2)
             for p in range(2)]
    assert all(abs(p["energy"] - ref["energy"]) > 1e-6 * abs(ref["energy"]) for p in parts)
    assert abs(sum(p["energy"] for p in parts) - ref["energy"]) <= 1e-12 * abs(ref["energy"])


def test_shard_systems_balance():
    """Longest-first binning: every system in exactly one bin, bins
    deterministic and within the largest system's cost of each other."""
    from dftd3 import parallel
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(8), np.log(257), size=500)).astype(int)
    costs = [parallel.system_cost(n) for n in sizes]
    for nparts in (1, 2, 3, 8):
        bins = parallel.shard_systems(costs, nparts)
        assert sorted(k for b in bins for k in b) == list(range(len(sizes)))
        assert bins == parallel.shard_systems(costs, nparts)
        loads = [sum(costs[k] for k in b) for b in bins]
        assert max(loads) - min(loads) <= max(costs)
    assert parallel.system_cost(64, periodic=True) > parallel.system_cost(64)


def _gloo_batch_rank(rank, world, port, queue):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root / "tests"), str(root / "simple-dftd3_b200")]
    import datetime
    import torch.distributed as dist
    import oracle_ref
    from dftd3 import parallel, synthetic as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        d = S.batch4096(nmol=9, seed=17, nmin=6, nmax=20)
        par = dict(S.PBE_BJ, damping="rational", s9=1.0)
        bins = parallel.shard_systems([parallel.system_cost(len(n)) for n in d["numbers"]], world)
        mine = bins[rank]
        # this process's bin (the oracle stands in for the GPU batch here)
        res = [oracle_ref.dispersion(d["numbers"][k], d["positions"][k], par) for k in mine]
        local = {"energy": [r["energy"] for r in res], "gradient": [r["gradient"] for r in res],
                 "virial": [r["virial"] for r in res]}
        out = parallel.gather_results(local, mine, len(d["numbers"]))
        queue.put((rank, out["energy"].tolist(), [g.tolist() for g in out["gradient"]]))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_batch_shards():
    """Two processes evaluate disjoint bins of a batch and both end with
    every system's result, equal to evaluating the whole batch in one."""
    import torch.multiprocessing as mp
    from dftd3 import synthetic as S
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_batch_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    d = S.batch4096(nmol=9, seed=17, nmin=6, nmax=20)
    par = dict(S.PBE_BJ, damping="rational", s9=1.0)
    for _, energies, grads in results:
        for k in range(9):
            ref = O.dispersion(d["numbers"][k], d["positions"][k], par)
            # the oracle's threaded sums are not bit-reproducible between runs
            assert abs(energies[k] - ref["energy"]) <= 1e-12 * abs(ref["energy"])
            assert np.abs(np.asarray(grads[k]) - ref["gradient"]).max() <= 1e-12 * np.abs(ref["gradient"]).max()
