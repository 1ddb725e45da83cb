"""Seeded synthetic geometries for the benchmark workloads.

No public dataset is involved: every structure is generated from a seed.

* ``water()``: O at the origin, H at (+-0.7570, 0.5859, 0) Angstrom
  (O-H 0.9572 Angstrom, angle 104.52 degrees).
* ``water_cluster(nx, ny, nz, count, seed)``: ``count`` of the nx*ny*nz sites of a
  cubic lattice with 3.0 Angstrom spacing, each water given a uniform random
  rotation (about its O atom) and a +-0.2 Angstrom uniform translation jitter.
  (H2O)16 uses a 3x3x2 lattice, (H2O)32 a 4x4x2 lattice.
* ``alkane(n, seed)``: all-trans CnH2n+2, C-C 1.54, C-H 1.09 Angstrom, tetrahedral
  angles, +-0.02 Angstrom uniform jitter per atom.
* ``water_dimer(seed)``: the cluster generator on a 2x1x1 lattice.
* ``displacements(mol, step)``: the +-step bohr displaced copies along every
  Cartesian coordinate (finite-difference frequency inputs, the pattern of
  chem/scf/Frequency.cpp:40-65).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .basis import A_TO_BOHR, Molecule

WATER_ANGSTROM = [(8, (0.0, 0.0, 0.0)), (1, (0.7570, 0.5859, 0.0)), (1, (-0.7570, 0.5859, 0.0))]


def water() -> Molecule:
    return Molecule([z for z, _ in WATER_ANGSTROM],
                    [tuple(c * A_TO_BOHR for c in p) for _, p in WATER_ANGSTROM])


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    # Uniform rotation from a uniform unit quaternion (Shoemake 1992).
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2),
                  math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3),
                  math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(nx: int, ny: int, nz: int, count: int, seed: int = 0,
                  spacing: float = 3.0, jitter: float = 0.2) -> Molecule:
    rng = np.random.default_rng(seed)
    sites = [(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)]
    if count > len(sites):
        raise ValueError("more molecules than lattice sites")
    chosen = sorted(rng.permutation(len(sites))[:count].tolist())
    base = np.array([p for _, p in WATER_ANGSTROM])
    Z: List[int] = []
    xyz: List[Tuple[float, float, float]] = []
    for s in chosen:
        R = _random_rotation(rng)
        shift = np.array(sites[s], dtype=float) * spacing + rng.uniform(-jitter, jitter, 3)
        pos = base @ R.T + shift
        for (z, _), p in zip(WATER_ANGSTROM, pos):
            Z.append(z)
            xyz.append(tuple(float(c) * A_TO_BOHR for c in p))
    return Molecule(Z, xyz)


def water_dimer(seed: int = 0) -> Molecule:
    return water_cluster(2, 1, 1, 2, seed)


def alkane(n: int, seed: int = 0, jitter: float = 0.02) -> Molecule:
    """All-trans CnH2n+2 in the xy plane zig-zag, hydrogens tetrahedral."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.54, 1.09
    half = math.radians(109.4712206) / 2.0
    dx = cc * math.sin(half)
    dy = cc * math.cos(half)
    carbons = [np.array([i * dx, (dy if i % 2 else 0.0), 0.0]) for i in range(n)]
    atoms: List[Tuple[int, np.ndarray]] = [(6, c) for c in carbons]
    for i, c in enumerate(carbons):
        up = 1.0 if i % 2 == 0 else -1.0  # away from the zig-zag neighbours
        # Two hydrogens out of plane, pointing away from the chain's bend.
        bis = np.array([0.0, -up, 0.0])
        tz = math.cos(math.radians(109.4712206) / 2.0)
        tp = math.sin(math.radians(109.4712206) / 2.0)
        for sgn in (1.0, -1.0):
            d = bis * tz + np.array([0.0, 0.0, sgn * tp])
            atoms.append((1, c + ch * d / np.linalg.norm(d)))
        if i == 0 or i == n - 1:
            # Terminal carbon: third hydrogen along the missing chain direction.
            if n == 1:
                # Methane: tetrahedron.
                atoms = [(6, c)]
                for v in ([1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]):
                    v = np.array(v, dtype=float)
                    atoms.append((1, c + ch * v / np.linalg.norm(v)))
                break
            nb = carbons[1] if i == 0 else carbons[n - 2]
            d = c - nb
            d = d / np.linalg.norm(d)
            # Reflect the C-C direction to keep the tetrahedral angle with the plane pair.
            other = np.array([d[0], -d[1], 0.0]) if i == 0 else np.array([d[0], -d[1], 0.0])
            atoms.append((1, c + ch * other / np.linalg.norm(other)))
    Z = [z for z, _ in atoms]
    xyz = [tuple(float(v) * A_TO_BOHR for v in (p + rng.uniform(-jitter, jitter, 3))) for _, p in atoms]
    return Molecule(Z, xyz)


def displacements(mol: Molecule, step: float = 0.005) -> List[Molecule]:
    out = []
    for a in range(mol.natom):
        for k in range(3):
            for sgn in (1.0, -1.0):
                xyz = [list(p) for p in mol.xyz]
                xyz[a][k] += sgn * step
                out.append(Molecule(list(mol.Z), [tuple(p) for p in xyz]))
    return out
