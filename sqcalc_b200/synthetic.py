"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference's own generator (test/gen_dump.py) writes LAMMPS dumps of ideal
gases, triclinic gases and lattices from fixed seeds; these builders produce the
same kinds of systems directly as arrays (rows of `cell` are the lattice vectors
a, b, c in LAMMPS' restricted triclinic form: a = (lx, 0, 0), b = (xy, ly, 0),
c = (xz, yz, lz)).
"""
from __future__ import annotations

import numpy as np

FCC_BASIS = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])


def fcc_solid(cells: int, a: float = 4.0, tilt=(5.0, 3.0, 0.0), types_on_basis=(1, 2, 1, 2)):
    """Perfect FCC crystal of cells^3 conventional cells of edge a in a
    triclinic box with tilts (xy, xz, yz); type of each of the four basis
    sublattices from `types_on_basis`.  Returns (positions (N, 3), types (N,),
    cell (3, 3))."""
    L = cells * a
    xy, xz, yz = (float(t) for t in tilt)
    cell = np.array([[L, 0.0, 0.0], [xy, L, 0.0], [xz, yz, L]])
    idx = np.stack(np.meshgrid(np.arange(cells), np.arange(cells), np.arange(cells),
                               indexing="ij"), axis=-1).reshape(-1, 1, 3)
    frac = ((idx + FCC_BASIS[None]) / cells).reshape(-1, 3)
    pos = frac @ cell
    types = np.tile(np.asarray(types_on_basis, dtype=np.int32), cells ** 3)
    return pos, types, cell


def thermal_frames(pos0, sigma, nframes, seed):
    """Frames of pos0 displaced by independent N(0, sigma^2) per coordinate."""
    rng = np.random.default_rng(seed)
    return [pos0 + rng.normal(0.0, sigma, pos0.shape) for _ in range(nframes)]


def uniform_two_types(natoms: int, box: float, seed: int, ratio=(1, 2)):
    """Uniform positions in a cubic box, two types in the given ratio, shuffled."""
    rng = np.random.default_rng(seed)
    n1 = natoms * ratio[0] // (ratio[0] + ratio[1])
    types = np.repeat(np.array([1, 2], dtype=np.int32), [n1, natoms - n1])
    rng.shuffle(types)
    return rng.random((natoms, 3)) * box, types


def batched_systems(nsystems: int, seed: int, nmin=5_000, nmax=200_000, density=0.08):
    """Independent cubic systems with N ~ U[nmin, nmax] atoms at the given
    number density (L = (N / density)^(1/3)), two types 1:2 shuffled.
    Returns a list of (natoms, box, types)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nsystems):
        n = int(rng.integers(nmin, nmax + 1))
        box = (n / density) ** (1.0 / 3.0)
        n1 = n // 3
        types = np.repeat(np.array([1, 2], dtype=np.int32), [n1, n - n1])
        rng.shuffle(types)
        out.append((n, box, types))
    return out
