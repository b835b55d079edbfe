"""The JSON line of bench.py's reference arm (the oracle port on the host
cores): one line, the contract's keys, the metric and unit of the GPU arm
on a small cell (CPU only)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--natoms", "200"], cwd=ROOT, capture_output=True, text=True,
                         timeout=300, check=True)
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    for k in KEYS:
        assert k in line, k
    assert line["unit"] == "pair-terms/s" and line["value"] > 0
    assert line["metric"].startswith("pair-terms/s")
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    # the CPU record names the threads used, the physical cores and the OpenMP settings
    cpu = line["cpu_baseline"]["cpu"]
    for k in ("threads", "physical_cores", "logical_cpus", "model", "OMP_NUM_THREADS", "OMP_SCHEDULE"):
        assert k in cpu, k
    assert cpu["threads"] == line["cpu_baseline"]["cores"]
    # both arms print the same config for the same workload
    sys.path.insert(0, str(ROOT))
    import bench
    systems, _ = bench.make_workload("cell2000", natoms=200)
    assert line["config"] == bench.workload_config("cell2000", systems, 1)
