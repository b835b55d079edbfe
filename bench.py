#!/usr/bin/env python3
"""Benchmark of the D3 dispersion hot path on B200.

Headline workload (one step): energy, gradient and virial of the periodic
2000-atom triclinic cell (edges 40-45 Bohr, angles 85-95 deg, H/C/N/O/Si/Al,
d_min 2.0, seeded), D3(BJ) two-body over all lattice images within 60 Bohr with
the CN chain rule (PBE parameters s6=1, s8=0.7875, a1=0.4289, a2=4.4407).
`value` is pair-terms/s of the mixed FP32/FP64 form with inputs resident in
HBM; the plain FP64 form is reported beside it, and `e2e` is the same metric
through the C ABI with host buffers (positions H2D and energy/gradient/virial
D2H inside the timed region).  A pair-term is one accepted (i, j <= i, T) of
the reference's two-body loop; a triple-term one accepted ATM triple.

The three-body workloads (ATM, s9 = 1) are measured beside the headline in
`extra_workloads`: the 5000-atom cluster (triple-terms/s), the batch of 4096
molecules (molecules/s) and a subset of the 256 periodic frames.  Any of them
can be the only workload with --workload (used for profiling small cases with
--natoms / --nsys).

Multi-GPU: one process per GPU (torchrun); every rank evaluates its own copy
of the workload (seed = rank), no collective on the data path ("scaling":
"weak").  --impl reference times the FP64 CPU restatement of the reference (the
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
# algorithmic flops per unit of work (FMA = 2); fixed between the two forms
FLOPS_PER_PAIR = 65            # two-body BJ term with gradient, virial and dE/dCN
FLOPS_PER_TRIPLE = 220         # ATM term with gradient, virial and dE/dCN
METRIC = "pair-terms/s, D3(BJ) two-body E+grad+virial (mixed FP32/FP64, <=1e-7 rel. E error)"
# DRAM bytes (read + write) of one k_two_body_tt<float, rational> launch on cell2000, from
# an ncu capture of that launch
TWO_BODY_TRAFFIC_BYTES = 1065728


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cell2000",
                    choices=["cell2000", "molecule100", "cluster5000", "batch4096", "frames256"])
    ap.add_argument("--natoms", type=int, default=None, help="atoms per system (smaller cases for profiling)")
    ap.add_argument("--nsys", type=int, default=None, help="systems of the batched workloads")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--shard", action="store_true",
                    help="with N > 1: all ranks share one copy of the workload (partitioned loops, NCCL "
                         "all-reduce of CN, dE/dCN and results; strong scaling) instead of one copy per rank")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true")
    return ap.parse_args()


def make_workload(name, seed=0, natoms=None, nsys=None):
    """(systems, parameters): systems is a list of (numbers, positions, lattice, periodic)."""
    from dftd3 import synthetic as S
    if name == "cell2000":
        d = S.cell2000(seed=seed, natoms=natoms or 2000)
        systems = [(d["numbers"], d["positions"], d["lattice"], d["periodic"])]
        s9 = 0.0
    elif name == "molecule100":
        d = S.molecule100(seed=seed)
        systems = [(d["numbers"], d["positions"], None, None)]
        s9 = 0.0
    elif name == "cluster5000":
        d = S.cluster5000(seed=seed, natoms=natoms or 5000)
        systems = [(d["numbers"], d["positions"], None, None)]
        s9 = 1.0
    elif name == "batch4096":
        d = S.batch4096(seed=seed, nmol=nsys or 4096)
        systems = [(n, p, None, None) for n, p in zip(d["numbers"], d["positions"])]
        s9 = 1.0
    else:
        d = S.frames256(seed=seed, nframes=nsys or 256, natoms=natoms or 512)
        systems = [(n, p, l, per) for n, p, l, per in zip(d["numbers"], d["positions"], d["lattices"],
                                                          d["periodic"])]
        s9 = 1.0
    par = dict(S.PBE_BJ, damping="rational", s9=s9)
    return systems, par


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the GPU work runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
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


class Runner:
    """One workload on the device: batch handle, device buffers, timed steps."""

    def __init__(self, systems, par):
        import torch
        from dftd3 import library as lib
        self.torch, self.lib = torch, lib
        self.systems = systems
        self.natoms = np.array([len(s[0]) for s in systems], dtype=np.int32)
        numbers = np.ascontiguousarray(np.concatenate([np.asarray(s[0]) for s in systems]), dtype=np.int32)
        pos = np.ascontiguousarray(np.concatenate([np.asarray(s[1], dtype=float).reshape(-1, 3) for s in systems]))
        periodic = systems[0][2] is not None
        lat = np.ascontiguousarray([s[2] for s in systems], dtype=float) if periodic else None
        per = np.ascontiguousarray([s[3] for s in systems], dtype=bool) if periodic else None
        self.batch = lib.new_batch(self.natoms, numbers, lat, per)
        self.param = lib.new_rational_damping(par["s6"], par["s8"], par["s9"], par["a1"], par["a2"], par["alp"])
        self.pos = torch.tensor(pos, dtype=torch.float64, device="cuda")
        nsys = len(systems)
        self.e = torch.zeros(nsys, dtype=torch.float64, device="cuda")
        self.g = torch.zeros_like(self.pos)
        self.s = torch.zeros(9 * nsys, dtype=torch.float64, device="cuda")
        self.stream = torch.cuda.current_stream()

    def step(self):
        self.lib.get_dispersion_device(self.batch, self.param, self.pos.data_ptr(), None, self.e.data_ptr(),
                                       self.g.data_ptr(), self.s.data_ptr(), 0, self.stream.cuda_stream)

    def counts(self):
        self.lib.set_batch_counting(self.batch, True)
        self.step()
        self.torch.cuda.synchronize()
        c = self.lib.get_batch_counts(self.batch)
        self.lib.set_batch_counting(self.batch, False)
        return {"pair_terms": int(c[0]), "triple_terms": int(c[1]), "cn_terms": int(c[2])}

    def time(self, precision, steps, warmup, flush, dist=None, stages=True, graph=False):
        """Device time of one step; with graph=True every step replays the
        batch's captured CUDA graph (dftd3_b200_set_batch_graph), positions
        copied in and results copied out inside the step.  Stage times come
        from separate ordinary steps with the engine's CUDA events."""
        torch, lib = self.torch, self.lib
        lib.set_batch_precision(self.batch, lib.PRECISION_FP64 if precision == "fp64" else lib.PRECISION_MIXED)
        lib.set_batch_graph(self.batch, graph)
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            flush.zero_()
            starts[k].record(self.stream)
            self.step()
            ends[k].record(self.stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / steps
        lib.set_batch_graph(self.batch, False)
        if not stages:
            return {"ms_per_step": ms, "energy": self.e.double().sum().item()}
        # per-stage device times of a few more steps (CUDA events inside the engine)
        lib.set_batch_profiling(self.batch, True)
        stages = {}
        for _ in range(3):
            flush.zero_()
            self.step()
            torch.cuda.synchronize()
            for kk, vv in lib.get_batch_stage_times(self.batch).items():
                stages[kk] = stages.get(kk, 0.0) + vv / 3
        lib.set_batch_profiling(self.batch, False)
        return {"ms_per_step": ms, "stage_ms": stages, "energy": self.e.double().sum().item()}


def batched_launch_modes(run, systems, par, flush, dist, sample=256):
    """Batch of molecules: the whole batch as one captured graph (autotuned
    launch shapes) against one evaluation per molecule (a sample of them)."""
    import torch
    lib = run.lib
    lib.set_batch_precision(run.batch, lib.PRECISION_MIXED)
    pos_host = run.pos.cpu().numpy()
    tuned_ms = lib.autotune_batch(run.batch, run.param, pos_host, True)
    out = {"autotune": dict(lib.get_batch_tuning(run.batch), best_ms=tuned_ms)}
    graph = {p: run.time(p, 3, 2, flush, dist, stages=False, graph=True) for p in ("fp64", "mixed")}
    out["graph"] = {p: {"ms_per_step": graph[p]["ms_per_step"],
                        "systems_per_s": len(systems) / (graph[p]["ms_per_step"] * 1e-3)} for p in graph}
    out["graph"]["mixed_speedup_vs_fp64"] = graph["fp64"]["ms_per_step"] / graph["mixed"]["ms_per_step"]
    # one batch (own engine and launch sequence) per molecule, same precision and stream
    singles = [Runner([sy], par) for sy in systems[:sample]]
    for r in singles:
        lib.set_batch_precision(r.batch, lib.PRECISION_MIXED)
        r.step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    t0.record(stream)
    for r in singles:
        r.step()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    out["per_molecule_launches"] = {"molecules": len(singles), "ms": ms,
                                    "systems_per_s": len(singles) / (ms * 1e-3), "precision": "mixed"}
    del singles
    return out


def autograd_step(systems, par, flush, steps=2):
    """Periodic frames through the torch.autograd wrapper: mixed forward (energies)
    and recomputing backward for positions, cell strain and (s6, s8, a1, a2, s9)."""
    import torch
    from dftd3.torch_api import D3Batch
    nums = [np.asarray(sy[0]) for sy in systems]
    lat = np.array([sy[2] for sy in systems], dtype=float)
    per = np.array([sy[3] for sy in systems], dtype=bool)
    model = D3Batch(nums, lattices=lat, periodic=per, damping="rational", precision="mixed")
    x = torch.tensor(np.concatenate([np.asarray(sy[1], dtype=float) for sy in systems]), device="cuda",
                     requires_grad=True)
    params = torch.tensor([par["s6"], par["s8"], par["a1"], par["a2"], par["s9"]], dtype=torch.float64,
                          device="cuda", requires_grad=True)
    strain = torch.zeros((len(systems), 3, 3), dtype=torch.float64, device="cuda", requires_grad=True)

    def one():
        e = model(x, params, strain)
        e.sum().backward()
        return e

    one()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(steps):
        flush.zero_()
        x.grad = None; params.grad = None; strain.grad = None
        t0.record(stream)
        one()
        t1.record(stream)
        torch.cuda.synchronize()
        ms.append(t0.elapsed_time(t1))
    best = min(ms)
    return {"frames": len(systems), "ms_forward_backward": best, "frames_per_s": len(systems) / (best * 1e-3),
            "precision": "mixed", "derivatives": "positions, strain, s6, s8, a1, a2, s9"}


def roofline(units, flops_per_unit, stage_ms, peak, kernel, bound):
    t = stage_ms * 1e-3
    achieved = units * flops_per_unit / t / 1e12 if t > 0 else None
    return {"bound": bound, "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None}


def cpu_reference_seconds(systems, par, repeats=3):
    """Wall time of the FP64 CPU restatement for the given systems (all host threads)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        for num, pos, lat, per in systems:
            oracle_ref.dispersion(num, pos, par, lattice=lat, periodic=per)
        times.append(time.perf_counter() - t0)
    return statistics.median(times)


def run_ours(args, rank, world, dist):
    import torch
    from dftd3 import library as lib
    from dftd3.interface import DispersionModel, RationalDampingParam

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    shard = args.shard and world > 1
    systems, par = make_workload(args.workload, seed=0 if shard else rank, natoms=args.natoms, nsys=args.nsys)
    run = Runner(systems, par)
    if shard:
        from dftd3 import parallel
        lib.set_batch_tuning(run.batch, 0.0, 0, 0, 0)
        run.reducer = parallel.make_device_reducer()
        lib.set_batch_reducer(run.batch, run.reducer, rank, world)
    counts = run.counts()
    if shard:
        # each rank counted its share of the loops
        ct = torch.tensor([counts[k] for k in sorted(counts)], dtype=torch.float64, device="cuda")
        dist.all_reduce(ct)
        counts = {k: int(v) for k, v in zip(sorted(counts), ct.tolist())}
    precs = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    sampler = ClockSampler(local)
    sampler.start()
    res = {p: run.time(p, args.steps, args.warmup, flush, dist, graph=not shard) for p in precs}
    extra = {}
    # the three-body workloads are reported at N = 1 (with N > 1 every rank would
    # repeat minutes of single-GPU work that the scaling run does not need)
    if not args.no_extra and args.workload == "cell2000" and not shard and world == 1:
        for name, steps in (("cluster5000", 3), ("batch4096", 3), ("frames256", 1)):
            nsys = 16 if name == "frames256" else None
            sy, pr = make_workload(name, seed=rank, nsys=nsys)
            rx = Runner(sy, pr)
            cx = rx.counts()
            tx = {p: rx.time(p, steps, 1, flush, dist) for p in ("fp64", "mixed")}
            units = cx["triple_terms"]
            entry = {"systems": len(sy), "atoms": int(rx.natoms.sum()), **cx}
            for p in tx:
                entry[p] = {"ms_per_step": tx[p]["ms_per_step"], "stage_ms": tx[p]["stage_ms"],
                            "triple_terms_per_s": units / (tx[p]["ms_per_step"] * 1e-3),
                            "systems_per_s": len(sy) / (tx[p]["ms_per_step"] * 1e-3)}
            entry["mixed_speedup_vs_fp64"] = tx["fp64"]["ms_per_step"] / tx["mixed"]["ms_per_step"]
            entry["mixed_vs_fp64_rel_energy_error"] = (abs(tx["mixed"]["energy"] - tx["fp64"]["energy"])
                                                       / abs(tx["fp64"]["energy"]))
            if name == "frames256":
                entry["note"] = "16 of the 256 frames per step"
                entry["autograd"] = autograd_step(sy, pr, flush)
            if name == "batch4096":
                entry.update(batched_launch_modes(rx, sy, pr, flush, dist))
            extra[name] = entry
            del rx
    sampler.stop()
    clocks = sampler.summary()

    e2e_ms = None
    if not args.no_e2e and len(systems) == 1 and not shard:
        num, pos, lat, per = systems[0]
        mol = DispersionModel(np.asarray(num), np.asarray(pos, dtype=float), lat, per)
        mol.set_precision("mixed" if "mixed" in precs else "fp64")
        # the evaluation replays one captured CUDA graph (dftd3_b200_set_model_graph)
        mol.set_graph(True)
        rp = RationalDampingParam(s6=par["s6"], s8=par["s8"], s9=par["s9"], a1=par["a1"], a2=par["a2"], alp=par["alp"])
        for _ in range(args.warmup):
            mol.get_dispersion(rp, grad=True)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            mol.get_dispersion(rp, grad=True)
        e2e_ms = 1e3 * (time.perf_counter() - t0) / args.steps

    head = "mixed" if "mixed" in res else "fp64"
    ms = res[head]["ms_per_step"]
    if dist:
        import torch.distributed as tdist
        t = torch.tensor([res[p]["ms_per_step"] for p in precs] + [e2e_ms or 0.0], dtype=torch.float64,
                         device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        vals = t.tolist()
        for k, p in enumerate(precs):
            res[p]["ms_per_step"] = vals[k]
        e2e_ms = vals[-1] if e2e_ms else None
        ms = res[head]["ms_per_step"]
    if rank != 0:
        return

    atm = par["s9"] != 0.0
    unit_key = "triple_terms" if atm else "pair_terms"
    unit = "triple-terms/s" if atm else "pair-terms/s"
    units = counts[unit_key]
    peak64 = lib.fma_peak(lib.PRECISION_FP64)
    peak32 = lib.fma_peak(lib.PRECISION_MIXED)
    # the dominant kernel alone, timed with CUDA events around its launch
    stage = "three_body_kernel" if atm else "two_body_kernel"
    flops = FLOPS_PER_TRIPLE if atm else FLOPS_PER_PAIR
    kern = "k_triples" if atm else "k_two_body_tt"
    line = {
        "metric": METRIC if args.workload == "cell2000" else f"{unit} ({args.workload})",
        "value": (1 if shard else world) * units / (ms * 1e-3),
        "unit": unit,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "strong" if shard else "weak",
        "vs_baseline": None,
        "dtype": "f32 pair/triple terms, f64 accumulation, weights and reductions" if head == "mixed" else "f64",
        "data": f"synthetic (seeded generator dftd3/synthetic.py, {args.workload})",
        "config": {"workload": {"cell2000": "cell2000: periodic triclinic 2000 atoms, D3(BJ) two-body + CN chain "
                                            "rule, E+grad+virial, disp2 60 / CN 40 Bohr"}.get(args.workload, args.workload),
                   "systems": len(systems), "atoms": int(run.natoms.sum()), **counts,
                   "l2": "flushed between timed steps (256 MB write)",
                   "launch": "ordinary launches" if shard else "captured CUDA graph replayed per step",
                   "parallelism": f"pair partition x{world} (NCCL)" if shard else f"replicas x{world}"},
        "precision_results": {p: {"value": (1 if shard else world) * units / (res[p]["ms_per_step"] * 1e-3), **res[p]}
                              for p in precs},
        "gpu_launches": None,
        "roofline": None,
        "clocks": clocks,
    }
    if "mixed" in res and "fp64" in res:
        line["mixed_speedup_vs_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
        line["mixed_vs_fp64_rel_energy_error"] = abs(res["mixed"]["energy"] - res["fp64"]["energy"]) / abs(
            res["fp64"]["energy"])
    # kernels launched per step (counted in the ncu launch list of the headline): the
    # column order (system shape and three rank passes; systems above 16384 atoms take
    # Morton keys, a radix sort of about nine kernels and a gather instead), tile
    # bounds, CN tile pairs + gather with weights and species vectors, two-body tile
    # pairs + gather, chain rule + gather, reduction; ATM adds the C6 table, neighbour
    # count, scan (2), capacity guard, fill and the triple kernel
    order_kernels = 4 if int(run.natoms.max()) <= 16384 else 11
    per_step = order_kernels + 8 + (7 if atm else 0)
    line["gpu_launches"] = per_step * args.steps * len(precs)
    rl = roofline(units, flops, res[head]["stage_ms"][stage], peak32 if head == "mixed" else peak64,
                  kern + ("<float>" if head == "mixed" else "<double>"), "fp32" if head == "mixed" else "fp64")
    rl["traffic"] = TWO_BODY_TRAFFIC_BYTES if (args.workload == "cell2000" and head == "mixed") else None
    if rl["traffic"] is not None:
        rl["traffic_source"] = "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch"
    rl["peak_source"] = "measured in-run FMA throughput (MEASURED_PEAKS.json has no FP32/FP64 pipe figure)"
    if "fp64" in res:
        rl["fp64"] = roofline(units, flops, res["fp64"]["stage_ms"][stage], peak64, kern + "<double>", "fp64")
    line["roofline"] = rl
    if e2e_ms:
        line["e2e"] = {"value": world * units / (e2e_ms * 1e-3), "unit": unit, "ms_per_step": e2e_ms,
                       "h2d_bytes_per_step": 24 * int(run.natoms.sum()),
                       "d2h_bytes_per_step": 8 + 24 * int(run.natoms.sum()) + 72}
    if extra:
        line["extra_workloads"] = extra
        for name, entry in extra.items():
            entry["roofline_mixed"] = roofline(entry["triple_terms"], FLOPS_PER_TRIPLE,
                                               entry["mixed"]["stage_ms"]["three_body_kernel"], peak32,
                                               "k_triples_mol<float>" if name == "batch4096" else "k_triples<float>",
                                               "fp32")
    if world == 1 and not args.no_cpu:
        sample = systems if len(systems) == 1 else systems[:64]
        cpu_s = cpu_reference_seconds(sample, par, repeats=3)
        sample_units = units if len(sample) == len(systems) else None
        line["cpu_baseline"] = {
            "value": (sample_units / cpu_s) if sample_units else len(sample) / cpu_s,
            "unit": unit if sample_units else "systems/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{len(sample)} system(s) of {args.workload} (E+grad+virial), median of 3 runs, "
                      "FP64 C/OpenMP restatement of the reference"}
    print(json.dumps(line), flush=True)


def count_pairs_cpu(systems, cutoff=60.0):
    """Accepted (i, j <= i, T) two-body terms (numpy, for the reference arm)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    total = 0
    for num, pos, lat, per in systems:
        trans = oracle_ref.lattice_points(lat, per, cutoff) if lat is not None else np.zeros((1, 3))
        pos = np.asarray(pos)
        for i in range(len(pos)):
            v = pos[i][None, None, :] - (pos[: i + 1][:, None, :] + trans[None, :, :])
            r2 = np.einsum("ijk,ijk->ij", v, v)
            total += int(np.count_nonzero((r2 <= cutoff * cutoff) & (r2 >= np.finfo(float).eps)))
    return total


def run_reference(args, rank, world):
    if rank != 0:
        return
    systems, par = make_workload(args.workload, seed=0, natoms=args.natoms, nsys=args.nsys)
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    sample = systems if len(systems) == 1 else systems[:64]

    def one():
        for num, pos, lat, per in sample:
            oracle_ref.dispersion(num, pos, par, lattice=lat, periodic=per)

    for _ in range(args.warmup):
        one()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    if par["s9"] == 0.0 and len(sample) == len(systems):
        units = count_pairs_cpu(sample)
        unit = "pair-terms/s"
        value = units / (ms * 1e-3)
    else:
        unit = "systems/s"
        value = len(sample) / (ms * 1e-3)
    line = {"impl": "reference", "metric": METRIC if args.workload == "cell2000" else f"{unit} ({args.workload})",
            "value": value, "unit": unit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (seeded generator dftd3/synthetic.py, {args.workload})",
            "config": {"workload": args.workload, "systems_per_step": len(sample)},
            "cpu_baseline": {"value": value, "unit": unit, "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{len(sample)} system(s) of {args.workload} per step (FP64 C/OpenMP "
                                       "restatement; the Fortran reference cannot be built here)"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    dist = None
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
