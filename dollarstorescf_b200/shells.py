"""Flattening a molecule and basis into the shell arrays the C ABI takes.

Function order follows ``scf::constructBasis`` (chem/scf/SCFBasis.cpp:120-139):
atoms in input order, shells in basis-file order (SP already split S then P),
and within a spherical shell m = -l..l.  Within a Cartesian (6D) shell the
monomials are x-major: x^a y^b z^c with a descending, then b descending.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from .basis import BasisSet, Molecule


@dataclass
class ShellArrays:
    natom: int
    Z: np.ndarray            # int32 [natom]
    atom_xyz: np.ndarray     # float64 [natom, 3] bohr
    shell_atom: np.ndarray   # int32 [nshell]
    shell_l: np.ndarray      # int32 [nshell]
    shell_nprim: np.ndarray  # int32 [nshell]
    exps: np.ndarray         # float64 [sum nprim]
    coefs: np.ndarray        # float64 [sum nprim], file (unnormalised) coefficients
    centers: np.ndarray      # float64 [nshell, 3] bohr
    pure: bool

    @property
    def nshell(self) -> int:
        return int(self.shell_l.shape[0])

    def nbf(self) -> int:
        if self.pure:
            return int(np.sum(2 * self.shell_l + 1))
        return int(np.sum((self.shell_l + 1) * (self.shell_l + 2) // 2))

    def n_electrons(self, charge: int = 0) -> int:
        return int(np.sum(self.Z)) - charge


def build_shells(mol: Molecule, basis: BasisSet, pure: bool = True) -> ShellArrays:
    sa: List[int] = []
    sl: List[int] = []
    sn: List[int] = []
    ex: List[float] = []
    co: List[float] = []
    ce: List[List[float]] = []
    for a, z in enumerate(mol.Z):
        for sh in basis.shells_for(z):
            sa.append(a)
            sl.append(sh.l)
            sn.append(len(sh.exps))
            ex.extend(sh.exps)
            co.extend(sh.coefs)
            ce.append(list(mol.xyz[a]))
    return ShellArrays(
        natom=mol.natom,
        Z=np.asarray(mol.Z, dtype=np.int32),
        atom_xyz=np.asarray(mol.xyz, dtype=np.float64).reshape(-1, 3),
        shell_atom=np.asarray(sa, dtype=np.int32),
        shell_l=np.asarray(sl, dtype=np.int32),
        shell_nprim=np.asarray(sn, dtype=np.int32),
        exps=np.asarray(ex, dtype=np.float64),
        coefs=np.asarray(co, dtype=np.float64),
        centers=np.asarray(ce, dtype=np.float64).reshape(-1, 3),
        pure=pure,
    )


def packed_index(y: int, x: int) -> int:
    """LAPACK 'U' packed index of element (y <= x) (lalib/Matrix.ipp:332-356)."""
    if y > x:
        y, x = x, y
    return x * (x + 1) // 2 + y


def unpack(p: np.ndarray, n: int) -> np.ndarray:
    """Packed-upper column-major vector -> dense symmetric matrix."""
    m = np.zeros((n, n))
    iu = np.triu_indices(n)
    # column-major upper: element (y, x), y<=x at x(x+1)/2 + y
    cols = iu[1]
    rows = iu[0]
    idx = cols * (cols + 1) // 2 + rows
    m[rows, cols] = p[idx]
    m[cols, rows] = p[idx]
    return m


def pack(m: np.ndarray) -> np.ndarray:
    n = m.shape[0]
    out = np.empty(n * (n + 1) // 2)
    iu = np.triu_indices(n)
    rows, cols = iu
    out[cols * (cols + 1) // 2 + rows] = m[rows, cols]
    return out
