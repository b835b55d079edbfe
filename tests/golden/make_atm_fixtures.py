#!/usr/bin/env python3
"""FP64 oracle results for the three-body workloads at their full sizes.

The CPU oracle needs minutes for these (about 3e10 triple checks for the
5000-atom cluster, 1e9 accepted triples per periodic frame), too long for a
test run, so its results are stored here once and the GPU parity tests and the
bench compare against them:

  cluster5000   the whole 5000-atom cluster of seed 0 (D3(BJ) + ATM, s9 = 1)
  frames        frames 0 and 1 of the 256-frame set of seed 0 (512 atoms each,
                cubic cells 28-32 Bohr, all images within 60 / 40 / 40 Bohr)

Energy, gradient and virial, PBE-D3(BJ) parameters (s6 = 1, s8 = 0.7875,
a1 = 0.4289, a2 = 4.4407, alp = 14), default cutoffs.  The geometries are
not stored: the seeded generator (dftd3/synthetic.py) rebuilds them, and the
file records a checksum of the positions so that a changed generator is caught.

    python tests/golden/make_atm_fixtures.py     # writes atm_configs.npz
"""
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "simple-dftd3_b200"))
sys.path.insert(0, str(ROOT / "tests"))

from dftd3 import synthetic  # noqa: E402
import oracle_ref  # noqa: E402

OUT = HERE / "atm_configs.npz"
PARAM = dict(synthetic.PBE_BJ, damping="rational", s9=1.0)


def checksum(pos):
    return float(np.sum(np.asarray(pos, dtype=float) * np.arange(1, 4)))


def main():
    data = {}
    t0 = time.perf_counter()
    c = synthetic.cluster5000(seed=0)
    r = oracle_ref.dispersion(c["numbers"], c["positions"], PARAM)
    data.update(cluster5000_energy=r["energy"], cluster5000_gradient=r["gradient"],
                cluster5000_virial=r["virial"], cluster5000_checksum=checksum(c["positions"]))
    print(f"cluster5000: E = {r['energy']:.15e} ({time.perf_counter() - t0:.0f} s)", flush=True)
    f = synthetic.frames256(seed=0, nframes=2)
    for k in range(2):
        t0 = time.perf_counter()
        r = oracle_ref.dispersion(f["numbers"][k], f["positions"][k], PARAM, lattice=f["lattices"][k],
                                  periodic=f["periodic"][k])
        data.update({f"frame{k}_energy": r["energy"], f"frame{k}_gradient": r["gradient"],
                     f"frame{k}_virial": r["virial"], f"frame{k}_checksum": checksum(f["positions"][k])})
        print(f"frame {k}: E = {r['energy']:.15e} ({time.perf_counter() - t0:.0f} s)", flush=True)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
