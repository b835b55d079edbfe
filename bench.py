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

The other workloads are measured beside the headline in `extra_workloads`:
the 100-atom molecule (microseconds per call through the C API), and the
three-body workloads (ATM, s9 = 1): the 5000-atom cluster (triple-terms/s),
the batch of 4096 molecules (molecules/s) and the 256 periodic frames of 512
atoms (triple-terms/s, and the autograd forward + backward).  Each carries the
FP64 oracle's CPU time on a bounded sample (`cpu_baseline`, all host threads),
the GPU/CPU ratio, and the error of both GPU forms against the FP64 oracle
(relative energy, largest gradient error in Hartree/Bohr, relative virial).
Any workload can be the only one with --workload (used for profiling small
cases with --natoms / --nsys).

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
        self.out = {}

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

    def time(self, precision, steps, warmup, flush, dist=None, stages=3, graph=False):
        """Device time of one step.  First `stages` ordinary steps with the
        engine's CUDA events per stage (they also warm up), then `warmup`
        untimed and `steps` timed steps; with graph=True every step replays the
        batch's captured CUDA graph (dftd3_b200_set_batch_graph), positions
        copied in and results copied out inside the step."""
        torch, lib = self.torch, self.lib
        lib.set_batch_precision(self.batch, lib.PRECISION_FP64 if precision == "fp64" else lib.PRECISION_MIXED)
        lib.set_batch_graph(self.batch, False)
        st = {}
        if stages:
            # one untimed step first: the first evaluation in a form allocates its buffers
            self.step()
            torch.cuda.synchronize()
            lib.set_batch_profiling(self.batch, True)
            for _ in range(stages):
                flush.zero_()
                self.step()
                torch.cuda.synchronize()
                for kk, vv in lib.get_batch_stage_times(self.batch).items():
                    st[kk] = st.get(kk, 0.0) + vv / stages
            lib.set_batch_profiling(self.batch, False)
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
        kernels = lib.get_batch_graph_kernels(self.batch) if graph else None
        lib.set_batch_graph(self.batch, False)
        # results of the last timed step (the positions are the same every step)
        self.out[precision] = (self.e.cpu().numpy().copy(), self.g.cpu().numpy().copy(),
                               self.s.cpu().numpy().reshape(-1, 3, 3).copy())
        res = {"ms_per_step": ms, "energy": self.e.double().sum().item()}
        if kernels is not None:
            res["graph_kernels"] = kernels
        if stages:
            res["stage_ms"] = st
        return res


def batched_launch_modes(run, systems, par, flush, dist, sample=256):
    """Batch of molecules: the whole batch as one captured graph (autotuned
    launch shapes) against one evaluation per molecule (a sample of them)."""
    import torch
    lib = run.lib
    lib.set_batch_precision(run.batch, lib.PRECISION_MIXED)
    pos_host = run.pos.cpu().numpy()
    tuned_ms = lib.autotune_batch(run.batch, run.param, pos_host, True)
    out = {"autotune": dict(lib.get_batch_tuning(run.batch), best_ms=tuned_ms)}
    graph = {p: run.time(p, 3, 2, flush, dist, stages=0, graph=True) for p in ("fp64", "mixed")}
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
    """Periodic frames through the torch.autograd wrapper: mixed forward (energies
    with the analytic derivatives of the same pass) and backward for positions,
    cell strain and (s6, s8, a1, a2, s9)."""
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


WORKLOAD_TEXT = {
    "cell2000": "cell2000: periodic triclinic 2000 atoms, D3(BJ) two-body + CN chain rule, E+grad+virial, "
                "disp2 60 / CN 40 Bohr",
    "molecule100": "molecule100: 100-atom molecule, D3(BJ) two-body, E+grad, FP64",
    "cluster5000": "cluster5000: 5000-atom ball, D3(BJ) + ATM (s9 1, 40 Bohr), E+grad+virial",
    "batch4096": "batch4096: 4096 molecules of 8-256 atoms, D3(BJ) + ATM, E+grad+virial",
    "frames256": "frames256: 256 periodic cubic frames of 512 atoms, D3(BJ) + ATM, E+grad+virial",
}
# the covalent radii of the CN come from mctc-lib, which is not part of the reference
# tree; they are restated from the published D3 radius set, and Si (10% of cell2000)
# occurs in none of the reference's own known-answer vectors
UNPINNED = "covalent radius of Si (Z=14) pinned by no reference vector (radii restated from the literature)"


def workload_config(name, systems, world, shard=False):
    """The `config` both arms print for one workload (identical dicts)."""
    cfg = {"workload": WORKLOAD_TEXT.get(name, name), "systems": len(systems),
           "atoms": int(sum(len(s[0]) for s in systems)),
           "l2": "flushed between timed GPU steps (256 MB write)",
           "parallelism": f"pair partition x{world} (NCCL)" if shard else f"replicas x{world}"}
    if name == "cell2000":
        cfg["note"] = UNPINNED
    return cfg


# ------------------------------------------------------------------ CPU side --

def oracle():
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ref
    return oracle_ref


def cpu_info():
    """Host cores and the OpenMP settings the oracle runs with."""
    import ctypes
    oracle().lib()   # loads the oracle and with it the OpenMP runtime
    info = {"logical_cpus": os.cpu_count()}
    try:
        txt = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
        kv = {}
        for ln in txt.splitlines():
            if ":" in ln:
                k, v = ln.split(":", 1)
                kv[k.strip()] = v.strip()
        info["model"] = kv.get("Model name")
        info["physical_cores"] = int(kv.get("Core(s) per socket", 0)) * int(kv.get("Socket(s)", 0)) or None
        info["threads_per_core"] = int(kv.get("Thread(s) per core", 0)) or None
    except (OSError, ValueError, subprocess.TimeoutExpired):
        pass
    try:
        info["threads"] = int(ctypes.CDLL("libgomp.so.1").omp_get_max_threads())
    except OSError:
        info["threads"] = os.cpu_count()
    info["OMP_NUM_THREADS"] = os.environ.get("OMP_NUM_THREADS", "unset (one thread per logical CPU)")
    info["OMP_SCHEDULE"] = ("dynamic,1 in the oracle's pair and triple loops (set in its source; "
                            "the reference's loops read schedule(runtime))")
    return info


def cpu_seconds(systems, par, part=0, nparts=1):
    O = oracle()
    t0 = time.perf_counter()
    for num, pos, lat, per in systems:
        O.dispersion(num, pos, par, lattice=lat, periodic=per, part=part, nparts=nparts)
    return time.perf_counter() - t0


def cpu_baseline(name, systems, par, work, info, repeats=3):
    """Time of the FP64 oracle (C/OpenMP restatement of the reference, all host
    threads) on a bounded sample of the workload, scaled to the workload's unit."""
    base = {"kind": "port", "cores": info.get("threads"), "cpu": info}
    if name == "cell2000":
        t = statistics.median(cpu_seconds(systems, par) for _ in range(repeats))
        return dict(base, value=work["pair_terms"] / t, unit="pair-terms/s", seconds=t,
                    sample=f"the whole cell (E+grad+virial), median of {repeats} runs")
    if name == "molecule100":
        cpu_seconds(systems, par)
        t = statistics.median(cpu_seconds(systems, par) for _ in range(20))
        return dict(base, value=t * 1e6, unit="us/call", higher_is_better=False, seconds=t,
                    sample="the whole molecule (E+grad), median of 20 calls")
    if name == "batch4096":
        sample = systems[::8]
        t = cpu_seconds(sample, par)
        return dict(base, value=len(sample) / t, unit="molecules/s", seconds=t,
                    sample=f"every 8th molecule of the batch ({len(sample)} molecules, "
                           f"{sum(len(s[0]) for s in sample)} atoms), E+grad+virial, one run")
    nparts = 16
    if name == "cluster5000":
        t = nparts * cpu_seconds(systems, par, part=0, nparts=nparts)
        return dict(base, value=work["triple_terms"] / t, unit="triple-terms/s", seconds=t,
                    sample=f"part 0 of {nparts} of the cluster's pair and triple loops (the reference's "
                           f"own work partition, pairs dealt cyclically) timed once and scaled by {nparts}; "
                           "the coordination number, computed whole in each part, makes this a slight "
                           "overestimate of the CPU time")
    if name == "frames256":
        t = nparts * cpu_seconds(systems[:1], par, part=0, nparts=nparts)
        return dict(base, value=work["frame0_triple_terms"] / t, unit="triple-terms/s", seconds=t,
                    frames_per_s=1.0 / t,
                    sample=f"frame 0: part 0 of {nparts} of its pair and triple loops (the reference's own "
                           f"work partition) timed once and scaled by {nparts}; triple-terms of frame 0")
    raise ValueError(name)


def errors_vs_oracle(name, run, systems, par, natoms_sys):
    """Error of each GPU form against the FP64 oracle on the workload (or a
    fixed sample of it): largest relative energy error, largest gradient error
    (Hartree/Bohr) and largest virial error relative to the system's largest
    virial component."""
    O = oracle()
    off = np.concatenate([[0], np.cumsum(natoms_sys)])
    refs = {}
    if name in ("cluster5000", "frames256"):
        fx = np.load(ROOT / "tests" / "golden" / "atm_configs.npz")
        keys = ["cluster5000"] if name == "cluster5000" else ["frame0", "frame1"]
        for k, key in enumerate(keys):
            pos = np.asarray(systems[k][1], dtype=float)
            if float(np.sum(pos * np.arange(1, 4))) != float(fx[f"{key}_checksum"]):
                return {"error": f"generated {key} positions differ from the stored oracle results"}
            refs[k] = {"energy": float(fx[f"{key}_energy"]), "gradient": fx[f"{key}_gradient"],
                       "virial": fx[f"{key}_virial"]}
        source = ("stored FP64 oracle results (tests/golden/atm_configs.npz, made by "
                  "tests/golden/make_atm_fixtures.py): " + ("the whole cluster" if name == "cluster5000"
                                                             else "frames 0 and 1"))
    else:
        if name == "batch4096":
            from dftd3 import synthetic as S
            pick = S.batch4096_sample(natoms_sys)
            source = (f"FP64 oracle on {len(pick)} molecules of the batch (its 8 largest, 256 atoms, "
                      "and 56 spread over the rest)")
        else:
            pick = list(range(len(systems)))
            source = "FP64 oracle on the whole workload"
        for k in pick:
            num, pos, lat, per = systems[k]
            refs[k] = O.dispersion(num, pos, par, lattice=lat, periodic=per)
    out = {"source": source, "systems_checked": len(refs)}
    for prec, (e, g, s) in run.out.items():
        re_, ge, ve = 0.0, 0.0, 0.0
        for k, ref in refs.items():
            re_ = max(re_, abs(e[k] - ref["energy"]) / abs(ref["energy"]))
            ge = max(ge, float(np.abs(g[off[k]:off[k + 1]] - ref["gradient"]).max()))
            ve = max(ve, float(np.abs(s[k] - ref["virial"]).max() / np.abs(ref["virial"]).max()))
        out[prec] = {"rel_energy": re_, "max_grad_abs": ge, "rel_virial": ve}
    return out


def molecule100_latency(flush, calls=200, warmup=20):
    """The 100-atom molecule through DispersionModel.get_dispersion (FP64,
    dftd3_get_dispersion on host buffers): microseconds per call with ordinary
    launches and with the model's captured graph replayed."""
    from dftd3.interface import DispersionModel, RationalDampingParam
    systems, par = make_workload("molecule100")
    num, pos, _, _ = systems[0]
    model = DispersionModel(np.asarray(num), np.asarray(pos, dtype=float))
    rp = RationalDampingParam(s6=par["s6"], s8=par["s8"], s9=par["s9"], a1=par["a1"], a2=par["a2"], alp=par["alp"])
    out = {"atoms": len(num), "precision": "fp64", "outputs": "energy, gradient, virial"}
    for graph in (False, True):
        model.set_graph(graph)
        for _ in range(warmup):
            res = model.get_dispersion(rp, grad=True)
        t0 = time.perf_counter()
        for _ in range(calls):
            res = model.get_dispersion(rp, grad=True)
        us = 1e6 * (time.perf_counter() - t0) / calls
        out["graph_replay" if graph else "ordinary_launches"] = {"us_per_call": us, "calls_per_s": 1e6 / us}
    ref = oracle().dispersion(num, pos, par)
    out["error_vs_oracle"] = {"fp64": {
        "rel_energy": abs(float(res["energy"]) - ref["energy"]) / abs(ref["energy"]),
        "max_grad_abs": float(np.abs(res["gradient"] - ref["gradient"]).max()),
        "rel_virial": float(np.abs(res["virial"] - ref["virial"]).max() / np.abs(ref["virial"]).max())},
        "source": "FP64 oracle on the whole molecule", "systems_checked": 1}
    return out, systems, par


def three_body_workload(name, rank, flush, dist, info, want_cpu):
    """One three-body workload: FP64 and mixed device times (stage times from
    ordinary steps), oracle errors, CPU baseline and GPU/CPU ratio."""
    nsys = None
    steps, stages = (3, 3) if name != "frames256" else (1, 1)
    sy, pr = make_workload(name, seed=rank, nsys=nsys)
    rx = Runner(sy, pr)
    cx = rx.counts()
    # frames256: the stage-timed step is the only warm-up
    tx = {p: rx.time(p, steps, 1 if name != "frames256" else 0, flush, dist, stages=stages)
          for p in ("fp64", "mixed")}
    units = cx["triple_terms"]
    entry = {"config": workload_config(name, sy, 1), "work": cx}
    for p in tx:
        entry[p] = {"ms_per_step": tx[p]["ms_per_step"], "stage_ms": tx[p]["stage_ms"],
                    "triple_terms_per_s": units / (tx[p]["ms_per_step"] * 1e-3),
                    "systems_per_s": len(sy) / (tx[p]["ms_per_step"] * 1e-3)}
    entry["mixed_speedup_vs_fp64"] = tx["fp64"]["ms_per_step"] / tx["mixed"]["ms_per_step"]
    entry["error_vs_oracle"] = errors_vs_oracle(name, rx, sy, pr, rx.natoms)
    if name == "frames256":
        entry["note"] = "all 256 frames per step; one warm-up (the stage-timed step) and one timed step per form"
        entry["autograd"] = autograd_step(sy, pr, flush, steps=1)
        one = Runner(sy[:1], pr)
        cx["frame0_triple_terms"] = one.counts()["triple_terms"]
        del one
    if name == "batch4096":
        entry.update(batched_launch_modes(rx, sy, pr, flush, dist))
    if want_cpu:
        cb = cpu_baseline(name, sy, pr, cx, info)
        entry["cpu_baseline"] = cb
        if name == "batch4096":
            gpu = entry["graph"]["mixed"]["systems_per_s"]
            entry["vs_cpu"] = {"mixed": gpu / cb["value"], "fp64": entry["graph"]["fp64"]["systems_per_s"] / cb["value"],
                               "unit": "molecules/s", "gpu": "one captured graph per batch"}
        else:
            entry["vs_cpu"] = {p: entry[p]["triple_terms_per_s"] / cb["value"] for p in ("fp64", "mixed")}
            entry["vs_cpu"]["unit"] = "triple-terms/s"
    del rx
    return entry


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
    want_cpu = world == 1 and not args.no_cpu
    info = cpu_info() if want_cpu else None
    sampler = ClockSampler(local)
    sampler.start()
    graph = not shard
    res = {p: run.time(p, args.steps, args.warmup, flush, dist, graph=graph) for p in precs}
    extra = {}
    # the other workloads are reported at N = 1 (with N > 1 every rank would
    # repeat minutes of single-GPU work that the scaling run does not need)
    if not args.no_extra and args.workload == "cell2000" and not shard and world == 1:
        m100, m_sys, m_par = molecule100_latency(flush)
        if want_cpu:
            m100["cpu_baseline"] = cpu_baseline("molecule100", m_sys, m_par, None, info)
            m100["vs_cpu"] = {"graph_replay": m100["cpu_baseline"]["value"] / m100["graph_replay"]["us_per_call"],
                              "ordinary_launches": (m100["cpu_baseline"]["value"]
                                                    / m100["ordinary_launches"]["us_per_call"]),
                              "unit": "CPU us per call / GPU us per call"}
        m100["config"] = workload_config("molecule100", m_sys, 1)
        extra["molecule100"] = m100
        for name in ("cluster5000", "batch4096", "frames256"):
            extra[name] = three_body_workload(name, rank, flush, dist, info, want_cpu)
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
        "config": workload_config(args.workload, systems, world, shard),
        "work": counts,
        "launch": "ordinary launches" if shard else "captured CUDA graph replayed per step",
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
    if graph and all("graph_kernels" in res[p] for p in precs):
        # kernel nodes of the captured graph of each form, one replay per timed step
        line["gpu_launches"] = sum(res[p]["graph_kernels"] * args.steps for p in precs)
        line["gpu_launches_source"] = "kernel nodes of the captured graph (cudaGraphGetNodes) x timed steps"
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
    if world == 1 and not shard:
        line["error_vs_oracle"] = errors_vs_oracle(args.workload, run, systems, par, run.natoms)
    if extra:
        line["extra_workloads"] = extra
        for name, entry in extra.items():
            if "mixed" not in entry:
                continue
            entry["roofline_mixed"] = roofline(entry["work"]["triple_terms"], FLOPS_PER_TRIPLE,
                                               entry["mixed"]["stage_ms"]["three_body_kernel"], peak32,
                                               "k_triples_mol<float>" if name == "batch4096" else "k_triples<float>",
                                               "fp32")
            entry["roofline_fp64"] = roofline(entry["work"]["triple_terms"], FLOPS_PER_TRIPLE,
                                              entry["fp64"]["stage_ms"]["three_body_kernel"], peak64,
                                              "k_triples_mol<double>" if name == "batch4096" else "k_triples<double>",
                                              "fp64")
    if want_cpu:
        if args.workload in ("cell2000", "cluster5000", "batch4096", "frames256"):
            if args.workload == "frames256":
                one = Runner(systems[:1], par)
                counts["frame0_triple_terms"] = one.counts()["triple_terms"]
                del one
            cb = cpu_baseline(args.workload, systems, par, counts, info)
            line["cpu_baseline"] = cb
            if cb["unit"] == unit:
                line["vs_cpu"] = {"value": line["value"] / cb["value"]}
                if "e2e" in line:
                    line["vs_cpu"]["e2e"] = line["e2e"]["value"] / cb["value"]
    print(json.dumps(line), flush=True)


def count_pairs_cpu(systems, cutoff=60.0):
    """Accepted (i, j <= i, T) two-body terms (numpy, for the reference arm)."""
    O = oracle()
    total = 0
    for num, pos, lat, per in systems:
        trans = O.lattice_points(lat, per, cutoff) if lat is not None else np.zeros((1, 3))
        pos = np.asarray(pos)
        for i in range(len(pos)):
            v = pos[i][None, None, :] - (pos[: i + 1][:, None, :] + trans[None, :, :])
            r2 = np.einsum("ijk,ijk->ij", v, v)
            total += int(np.count_nonzero((r2 <= cutoff * cutoff) & (r2 >= np.finfo(float).eps)))
    return total


def run_reference(args, rank, world):
    """The reference arm: the FP64 CPU restatement of the reference (the
    Fortran reference cannot be built here) on all host threads, timed on the
    same workload and printed with the same metric, unit and config."""
    if rank != 0:
        return
    systems, par = make_workload(args.workload, seed=0, natoms=args.natoms, nsys=args.nsys)
    info = cpu_info()
    sample = systems if len(systems) == 1 else systems[:64]
    for _ in range(args.warmup):
        cpu_seconds(sample, par)
    times = [cpu_seconds(sample, par) for _ in range(args.steps)]
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
            "config": workload_config(args.workload, systems, world),
            "cpu_baseline": {"value": value, "unit": unit, "cores": info.get("threads"), "kind": "port", "cpu": info,
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
