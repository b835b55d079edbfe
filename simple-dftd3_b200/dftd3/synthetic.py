"""Seeded synthetic geometries for the benchmark and parity workloads.

Each generator draws elements with the stated probabilities and places atoms
by random sequential packing with a minimum interatomic distance (minimum
image distance for periodic cells).  All lengths are in Bohr.

Workloads (the five benchmark configurations):
  molecule100   100-atom molecule, H/C/N/O, 20 Bohr cube, d_min 1.8
  cell2000      2000-atom triclinic cell, edges 40-45 Bohr, angles 85-95 deg,
                H/C/N/O/Si/Al, d_min 2.0
  cluster5000   5000-atom ball at 0.012 atoms/Bohr^3, H/C/N/O/S, d_min 1.8
  batch4096     4096 molecules, n log-uniform in [8, 256], 0.01 atoms/Bohr^3,
                H/C/N/O/F/S/Cl, d_min 1.8
  frames256     256 cubic frames of 512 atoms, L in [28, 32] Bohr, H/C/N/O,
                d_min 1.9
"""
import numpy as np


def _draw_elements(rng, n, elements, probs):
    return rng.choice(np.asarray(elements), size=n, p=np.asarray(probs) / np.sum(probs)).astype(np.int32)


def pack_box(rng, n, lo, hi, dmin, shape="cube", max_tries=200000):
    """Random sequential packing in a cube [lo, hi)^3 or a ball of radius hi."""
    pos = np.empty((n, 3))
    d2 = dmin * dmin
    k = 0
    tries = 0
    while k < n:
        tries += 1
        if tries > max_tries * max(n, 1):
            raise RuntimeError("packing failed: density too high for d_min")
        if shape == "cube":
            c = rng.uniform(lo, hi, size=3)
        else:
            v = rng.normal(size=3)
            c = v / np.linalg.norm(v) * hi * rng.uniform() ** (1.0 / 3.0)
        if k and np.min(np.sum((pos[:k] - c) ** 2, axis=1)) < d2:
            continue
        pos[k] = c
        k += 1
    return pos


def pack_cell(rng, n, lattice, dmin, max_tries=200000):
    """Random sequential packing in a periodic cell (rows of `lattice` are the
    lattice vectors) with the minimum image distance."""
    frac = np.empty((n, 3))
    d2 = dmin * dmin
    k = 0
    tries = 0
    while k < n:
        tries += 1
        if tries > max_tries * max(n, 1):
            raise RuntimeError("packing failed: density too high for d_min")
        f = rng.uniform(size=3)
        if k:
            df = frac[:k] - f
            df -= np.rint(df)
            dx = df @ lattice
            if np.min(np.sum(dx * dx, axis=1)) < d2:
                continue
        frac[k] = f
        k += 1
    return frac @ lattice


def triclinic(a, b, c, alpha, beta, gamma):
    """Lattice vectors (rows) from edge lengths and angles in degrees."""
    al, be, ga = np.radians([alpha, beta, gamma])
    va = np.array([a, 0.0, 0.0])
    vb = np.array([b * np.cos(ga), b * np.sin(ga), 0.0])
    cx = c * np.cos(be)
    cy = c * (np.cos(al) - np.cos(be) * np.cos(ga)) / np.sin(ga)
    cz = np.sqrt(max(c * c - cx * cx - cy * cy, 0.0))
    return np.array([va, vb, [cx, cy, cz]])


PBE_BJ = dict(s6=1.0, s8=0.7875, a1=0.4289, a2=4.4407, alp=14.0)


def molecule100(seed=0):
    rng = np.random.default_rng(seed)
    num = _draw_elements(rng, 100, [1, 6, 7, 8], [0.5, 0.3, 0.1, 0.1])
    pos = pack_box(rng, 100, 0.0, 20.0, 1.8)
    return dict(numbers=num, positions=pos, lattice=None, periodic=None, s9=0.0)


def cell2000(seed=0, natoms=2000):
    rng = np.random.default_rng(seed)
    a, b, c = rng.uniform(40.0, 45.0, size=3)
    al, be, ga = rng.uniform(85.0, 95.0, size=3)
    lat = triclinic(a, b, c, al, be, ga)
    num = _draw_elements(rng, natoms, [1, 6, 7, 8, 14, 13], [0.3, 0.25, 0.1, 0.15, 0.1, 0.1])
    pos = pack_cell(rng, natoms, lat, 2.0)
    return dict(numbers=num, positions=pos, lattice=lat, periodic=np.array([True, True, True]), s9=0.0)


def cluster5000(seed=0, natoms=5000, density=0.012):
    rng = np.random.default_rng(seed)
    radius = (3.0 * natoms / (4.0 * np.pi * density)) ** (1.0 / 3.0)
    num = _draw_elements(rng, natoms, [1, 6, 7, 8, 16], [0.45, 0.3, 0.1, 0.1, 0.05])
    pos = pack_box(rng, natoms, 0.0, radius, 1.8, shape="ball")
    return dict(numbers=num, positions=pos, lattice=None, periodic=None, s9=1.0)


def batch4096(seed=0, nmol=4096, nmin=8, nmax=256, density=0.01):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax + 1), size=nmol)).astype(int)
    sizes = np.clip(sizes, nmin, nmax)
    numbers, positions = [], []
    for n in sizes:
        side = (n / density) ** (1.0 / 3.0)
        numbers.append(_draw_elements(rng, n, [1, 6, 7, 8, 9, 16, 17], [0.45, 0.28, 0.1, 0.1, 0.03, 0.02, 0.02]))
        positions.append(pack_box(rng, n, 0.0, side, 1.8))
    return dict(numbers=numbers, positions=positions, lattices=None, periodic=None, s9=1.0)


def frames256(seed=0, nframes=256, natoms=512):
    rng = np.random.default_rng(seed)
    numbers, positions, lattices = [], [], []
    for _ in range(nframes):
        box = rng.uniform(28.0, 32.0)
        lat = np.eye(3) * box
        numbers.append(_draw_elements(rng, natoms, [1, 6, 7, 8], [0.4, 0.3, 0.15, 0.15]))
        positions.append(pack_cell(rng, natoms, lat, 1.9))
        lattices.append(lat)
    return dict(numbers=numbers, positions=positions, lattices=np.array(lattices),
                periodic=np.ones((nframes, 3), dtype=bool), s9=1.0)


def batch4096_sample(sizes, n=64, largest=8):
    """Indices of a fixed sample of a molecule batch for parity checks against
    the FP64 oracle: the `largest` biggest molecules and n - largest more
    spread evenly over the rest of the batch (in batch order)."""
    sizes = np.asarray(sizes)
    order = np.argsort(-sizes, kind="stable")
    big = set(int(k) for k in order[:largest])
    rest = [k for k in range(len(sizes)) if k not in big]
    step = max(len(rest) // max(n - largest, 1), 1)
    pick = sorted(big) + rest[::step][: n - largest]
    return sorted(pick)
