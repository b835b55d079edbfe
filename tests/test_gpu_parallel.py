"""GPU tests of the partitioned evaluation with a reducer (the engine side of
the multi-process path).  Two parts run as two host threads on one GPU, each
with its own batch and stream; the reducer synchronises its stream and sums
through host memory, so no kernel waits for another part.  A one-process NCCL
group checks the torch.distributed reducer end to end."""
import threading

import numpy as np
import pytest

import oracle_ref as O

pytestmark = pytest.mark.gpu

CUT = (25.0, 14.0, 20.0, 0.0, 0.0)


def _cell(seed=4, n=40):
    from dftd3 import synthetic as S
    rng = np.random.default_rng(seed)
    # no lattice vector length at an integer fraction of a cutoff: the mixed
    # form decides the cutoff test in FP32, so a self-image exactly on the
    # cutoff sphere may flip
    lat = S.triclinic(11.3, 11.9, 12.35, 87.0, 91.0, 94.0)
    num = rng.choice([1, 6, 7, 8], size=n).astype(np.int32)
    pos = S.pack_cell(rng, n, lat, 2.0)
    return num, pos, lat


@pytest.mark.parametrize("s9,precision", [(1.0, "fp64"), (0.0, "fp64"), (1.0, "mixed")])
def test_two_parts_on_threads(s9, precision):
    import torch
    from dftd3 import library
    num, pos, lat = _cell()
    par = dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, s9=s9, alp=14.0)
    ref = O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=CUT, wrap=False)
    nparts = 2
    barrier = threading.Barrier(nparts, timeout=60)
    slots = [None] * nparts
    out = [None] * nparts
    errors = []

    def worker(part):
        try:
            torch.cuda.set_device(0)
            stream = torch.cuda.Stream()

            def host_reduce(buffer, count, st, user):
                dev = device_view(buffer, count)
                ext = torch.cuda.ExternalStream(int(library.ffi.cast("uintptr_t", st)))
                ext.synchronize()                 # this part's kernels are done
                slots[part] = dev.cpu().numpy()
                barrier.wait()
                total = np.sum(slots, axis=0)
                barrier.wait()
                dev.copy_(torch.from_numpy(total).to("cuda"))
                torch.cuda.synchronize()
                return 0

            cb = library.ffi.callback("dftd3_b200_reducer", host_reduce)
            batch = library.new_batch(np.array([len(num)], dtype=np.int32), num, lat[None], np.ones((1, 3), bool))
            library.set_batch_realspace_cutoff(batch, *CUT)
            library.set_batch_precision(batch, library.PRECISION_MIXED if precision == "mixed"
                                        else library.PRECISION_FP64)
            library.set_batch_reducer(batch, cb, part, nparts)
            with torch.cuda.stream(stream):
                x = torch.tensor(pos, device="cuda")
                e = torch.zeros(1, dtype=torch.float64, device="cuda")
                g = torch.zeros_like(x)
                sg = torch.zeros(9, dtype=torch.float64, device="cuda")
                library.get_dispersion_device(batch, param_of(par), x.data_ptr(), None, e.data_ptr(), g.data_ptr(),
                                              sg.data_ptr(), 0, stream.cuda_stream)
                stream.synchronize()
            out[part] = (e.item(), g.cpu().numpy(), sg.cpu().numpy().reshape(3, 3))
        except Exception as exc:   # reported by the main thread
            errors.append(exc)
            barrier.abort()

    threads = [threading.Thread(target=worker, args=(p,)) for p in range(nparts)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    etol, gtol = (1e-12, 1e-12) if precision == "fp64" else (1e-7, None)
    for e, g, sg in out:
        assert abs(e - ref["energy"]) <= etol * abs(ref["energy"])
        if gtol:
            assert np.abs(g - ref["gradient"]).max() <= gtol * np.abs(ref["gradient"]).max()
            assert np.abs(sg.T - ref["virial"]).max() <= gtol * np.abs(ref["virial"]).max()
        else:
            assert np.abs(g - ref["gradient"]).max() <= 1e-7


def param_of(par):
    from dftd3 import library
    return library.new_rational_damping(par["s6"], par["s8"], par["s9"], par["a1"], par["a2"], par["alp"])


def device_view(buffer, count):
    """float64 tensor over a device pointer handed to the reducer (no copy)."""
    import torch
    from dftd3 import library
    from dftd3.parallel import _DeviceArray
    return torch.as_tensor(_DeviceArray(int(library.ffi.cast("uintptr_t", buffer)), count, 0), device="cuda")


def test_nccl_single_rank_sharded():
    """torch.distributed NCCL reducer with one rank: the complete result."""
    import datetime
    import os
    import socket
    import torch
    import torch.distributed as dist
    from dftd3 import library
    from dftd3.parallel import ShardedDispersion
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        num, pos, lat = _cell(seed=5)
        par = dict(damping="rational", s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, s9=1.0, alp=14.0)
        ref = O.dispersion(num, pos, par, lattice=lat, periodic=[True] * 3, cutoff=CUT, wrap=False)
        sh = ShardedDispersion([num], lattices=lat[None], periodic=np.ones((1, 3), bool), precision="fp64")
        sh.set_realspace_cutoff(*CUT)
        x = torch.tensor(pos, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        g = torch.zeros_like(x)
        sh.get_dispersion(param_of(par), x.data_ptr(), e.data_ptr(), g.data_ptr(), 0,
                          torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert abs(e.item() - ref["energy"]) <= 1e-12 * abs(ref["energy"])
        assert np.abs(g.cpu().numpy() - ref["gradient"]).max() <= 1e-12 * np.abs(ref["gradient"]).max()
        del sh
    finally:
        dist.destroy_process_group()
