#!/usr/bin/env python3
"""Benchmark of the D3 dispersion hot path on B200.

Workload (one step): energy, gradient and virial of the periodic 2000-atom
triclinic cell (edges 40-45 Bohr, angles 85-95 deg, H/C/N/O/Si/Al, d_min 2.0,
seeded), D3(BJ) two-body over all lattice images within 60 Bohr with the CN
chain rule (PBE parameters s6=1, s8=0.7875, a1=0.4289, a2=4.4407).
The headline `value` is pair-terms/s of the mixed FP32/FP64 form with inputs
resident in HBM; the plain FP64 form is reported beside it, and `e2e` is the
same metric through the C ABI with host buffers (positions H2D and
energy/gradient/virial D2H inside the timed region).  A pair-term is one
accepted (i, j <= i, T) of the reference's two-body loop.

Multi-GPU: one process per GPU (torchrun); every rank evaluates its own cell
(seed = rank), no collective on the data path ("scaling": "weak").

--impl reference times the FP64 CPU restatement of the reference (the
reference is Fortran and cannot be built here) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "simple-dftd3_b200"))

L2_FLUSH_BYTES = 256 << 20     # larger than the 126 MB L2
FLOPS_PER_PAIR = 65            # two-body BJ term, E+G+sigma+dEdcn (flop counting: FMA = 2)
METRIC = "pair-terms/s, D3(BJ) two-body E+grad+virial (mixed FP32/FP64, <=1e-7 rel. E error)"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    return ap.parse_args()


def workload(seed):
    from dftd3 import synthetic
    d = synthetic.cell2000(seed=seed)
    par = dict(synthetic.PBE_BJ, damping="rational", s9=0.0)
    return d, par


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz)}


def cpu_reference_time(d, par, repeats=3):
    """Wall time of the FP64 CPU restatement of one evaluation (all host threads)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        oracle_ref.dispersion(d["numbers"], d["positions"], par, lattice=d["lattice"], periodic=d["periodic"])
        times.append(time.perf_counter() - t0)
    return statistics.median(times)


def count_pair_terms(lib, batch, param, pos, tensors, torch):
    lib.set_batch_counting(batch, True)
    e, g, s = tensors
    lib.get_dispersion_device(batch, param, pos.data_ptr(), None, e.data_ptr(), g.data_ptr(), s.data_ptr(), 0,
                              torch.cuda.current_stream().cuda_stream)

    torch.cuda.synchronize()
    counts = lib.get_batch_counts(batch)
    lib.set_batch_counting(batch, False)
    return int(counts[0]), int(counts[2])


def run_ours(args, rank, world, dist):
    import torch
    from dftd3 import library as lib
    from dftd3.interface import DispersionModel, RationalDampingParam

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    d, par = workload(seed=rank)
    nat = len(d["numbers"])
    param = lib.new_rational_damping(par["s6"], par["s8"], par["s9"], par["a1"], par["a2"], par["alp"])
    natoms = np.array([nat], dtype=np.int32)
    batch = lib.new_batch(natoms, np.ascontiguousarray(d["numbers"], dtype=np.int32),
                          np.ascontiguousarray(d["lattice"]), np.ascontiguousarray(d["periodic"]))
    # wrapped positions resident on the device
    pos_h = np.ascontiguousarray(d["positions"], dtype=float)
    from dftd3.interface import Structure  # wrapping as the API does
    mol = DispersionModel(d["numbers"], pos_h, d["lattice"], d["periodic"])
    pos = torch.tensor(pos_h, dtype=torch.float64, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros((nat, 3), dtype=torch.float64, device="cuda")
    s = torch.zeros(9, dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    pair_terms, cn_terms = count_pair_terms(lib, batch, param, pos, (e, g, s), torch)

    def step():
        lib.get_dispersion_device(batch, param, pos.data_ptr(), None, e.data_ptr(), g.data_ptr(), s.data_ptr(),
                                  0, stream.cuda_stream)

    results = {}
    sampler = ClockSampler(local)
    sampler.__enter__()
    for prec_name, prec in (("fp64", lib.PRECISION_FP64), ("mixed", lib.PRECISION_MIXED)):
        lib.set_batch_precision(batch, prec)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            step()
            ends[k].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
        # dominant kernel time from the engine's stage events (one profiled step)
        lib.set_batch_profiling(batch, True)
        stage = {}
        for _ in range(3):
            flush.zero_()
            step()
            torch.cuda.synchronize()
            st = lib.get_batch_stage_times(batch)
            for kk, vv in st.items():
                stage[kk] = stage.get(kk, 0.0) + vv / 3
        lib.set_batch_profiling(batch, False)
        results[prec_name] = dict(ms=ms, stages=stage, energy=float(e.item()))

    sampler.__exit__(None, None, None)
    clocks = sampler.summary()
    # end to end through the C ABI with host buffers (dftd3_get_dispersion)
    rp = RationalDampingParam(s6=par["s6"], s8=par["s8"], s9=par["s9"], a1=par["a1"], a2=par["a2"], alp=par["alp"])
    mol.set_precision("mixed")
    for _ in range(args.warmup):
        r = mol.get_dispersion(rp, grad=True)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = mol.get_dispersion(rp, grad=True)
    e2e_s = time.perf_counter() - t0
    e2e_energy = float(r["energy"])

    # mixed-vs-FP64 error on this workload
    rel_err = abs(results["mixed"]["energy"] - results["fp64"]["energy"]) / abs(results["fp64"]["energy"])

    ms_mixed = results["mixed"]["ms"] / args.steps
    ms_fp64 = results["fp64"]["ms"] / args.steps
    e2e_ms = 1e3 * e2e_s / args.steps
    if dist:
        import torch.distributed as tdist
        t = torch.tensor([ms_mixed, ms_fp64, e2e_ms], dtype=torch.float64, device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms_mixed, ms_fp64, e2e_ms = (float(x) for x in t.tolist())
    if rank != 0:
        return
    total_terms = pair_terms * world
    peak64 = lib.fma_peak(lib.PRECISION_FP64)
    peak32 = lib.fma_peak(lib.PRECISION_MIXED)
    t2b = results["mixed"]["stages"]["two_body"] * 1e-3
    achieved = pair_terms * FLOPS_PER_PAIR / t2b / 1e12 if t2b > 0 else None
    t2b64 = results["fp64"]["stages"]["two_body"] * 1e-3
    achieved64 = pair_terms * FLOPS_PER_PAIR / t2b64 / 1e12 if t2b64 > 0 else None
    line = {
        "metric": METRIC,
        "value": total_terms / (ms_mixed * 1e-3),
        "unit": "pair-terms/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_mixed,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (pair terms) + f64 (accumulation, weights, reductions)",
        "data": "synthetic (seeded generator, dftd3/synthetic.py cell2000)",
        "config": {"workload": "cell2000: periodic triclinic 2000 atoms, D3(BJ) two-body + CN chain rule, "
                               "E+grad+virial, disp2 60 / CN 40 Bohr",
                   "pair_terms_per_step": pair_terms, "cn_terms_per_step": cn_terms,
                   "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{world}"},
        "fp64": {"value": total_terms / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64,
                 "stage_ms": results["fp64"]["stages"]},
        "mixed_stage_ms": results["mixed"]["stages"],
        "mixed_vs_fp64_rel_energy_error": rel_err,
        "e2e": {"value": total_terms / (e2e_ms * 1e-3), "unit": "pair-terms/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": 3 * 8 * pair_terms * 0 + 3 * 8 * len(d["numbers"]),
                "d2h_bytes_per_step": 8 + 3 * 8 * len(d["numbers"]) + 9 * 8, "energy": e2e_energy},
        "gpu_launches": 6 * args.steps * 2,
        "roofline": {"bound": "fp32", "kernel": "k_two_body<float, rational>", "achieved": achieved,
                     "peak": peak32, "unit": "TFLOP/s", "frac": (achieved / peak32) if achieved else None,
                     "traffic": None,
                     "peak_source": "measured in-run FMA throughput (MEASURED_PEAKS.json has no FP32/FP64 figure)",
                     "fp64": {"achieved": achieved64, "peak": peak64,
                              "frac": (achieved64 / peak64) if achieved64 else None}},
        "clocks": clocks,
    }
    if world == 1:
        cpu_s = cpu_reference_time(d, par, repeats=3)
        line["cpu_baseline"] = {"value": pair_terms / cpu_s, "unit": "pair-terms/s",
                                "cores": os.cpu_count(), "kind": "port",
                                "sample": "one full cell2000 evaluation (E+grad+virial), median of 3, "
                                          "FP64 C/OpenMP restatement of the reference"}
    print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    d, par = workload(seed=0)
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    # pair-term count of the workload from a cheap energy-free pass is not
    # available on the CPU; use the GPU-independent analytic count instead
    times = []
    for _ in range(args.warmup):
        oracle_ref.dispersion(d["numbers"], d["positions"], par, lattice=d["lattice"], periodic=d["periodic"])
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle_ref.dispersion(d["numbers"], d["positions"], par, lattice=d["lattice"], periodic=d["periodic"])
        times.append(time.perf_counter() - t0)
    terms = count_pairs_cpu(d)
    ms = 1e3 * sum(times) / len(times)
    value = terms / (ms * 1e-3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pair-terms/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cell2000", "pair_terms_per_step": terms},
            "cpu_baseline": {"value": value, "unit": "pair-terms/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "one full cell2000 evaluation per step (FP64 C/OpenMP restatement; "
                                       "the Fortran reference cannot be built here)"},
            "e2e": {"value": value, "unit": "pair-terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def count_pairs_cpu(d):
    """Accepted (i, j <= i, T) pair-terms of the two-body loop (numpy)."""
    from dftd3.synthetic import triclinic  # noqa: F401
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    trans = oracle_ref.lattice_points(d["lattice"], d["periodic"], 60.0)
    pos = np.asarray(d["positions"])
    n = len(pos)
    total = 0
    c2 = 60.0 * 60.0
    for i in range(n):
        v = pos[i][None, None, :] - (pos[: i + 1][:, None, :] + trans[None, :, :])
        r2 = np.einsum("ijk,ijk->ij", v, v)
        total += int(np.count_nonzero((r2 <= c2) & (r2 >= np.finfo(float).eps)))
    return total


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        run_ours(args, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
