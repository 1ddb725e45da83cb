"""Basis-set and geometry input, mirroring the reference's loaders.

* ``read_basis(path)`` reads a Gaussian-format basis file (Basis Set Exchange
  export) the way ``flo::Gaussian::readBasis`` does (chem/BasisReader.cpp:98-114,
  ``readAtomicBasis`` :9-96): element blocks start with ``<Sym> 0``; shells are
  ``<type> <nprim> <scale>`` followed by ``nprim`` lines; ``SP`` shells are split
  into an S shell followed by a P shell with the same exponents (:84-93);
  ``****`` ends an element; ECP blocks are skipped (:13); exponents must be
  positive and a shell holds 1..100 primitives (:62-75).  ``D`` exponents such
  as ``0.18D+02`` are accepted (util/TextReader.cpp:57-86).
* ``read_xyz(path)`` follows ``flo::readXYZFile`` (chem/XYZReader.cpp:6-34):
  count line, comment line, then ``Sym x y z`` in Angstrom, converted to bohr
  with ``A_to_a0 = 1.889726126`` (chem/Constants.hpp:15).

Errors raise ``BasisError`` / ``GeometryError`` instead of printing and
continuing as the reference does; the error text names the same condition.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

A_TO_BOHR = 1.889726126  # chem/Constants.hpp:15

ELEMENT_SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
    "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr Rf "
    "Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og"
).split()

_L_LETTERS = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6, "J": 7}


class BasisError(ValueError):
    pass


class GeometryError(ValueError):
    pass


def element_number(symbol: str) -> int:
    """Atomic number for an exact (case-sensitive) symbol, 0 if unknown
    (chem/Element.cpp:178-186)."""
    if 0 < len(symbol) < 3 and symbol in ELEMENT_SYMBOLS:
        return ELEMENT_SYMBOLS.index(symbol) + 1
    return 0


@dataclass
class Shell:
    """One contracted shell: angular momentum, exponents and the file's
    (unnormalised) contraction coefficients (chem/GTO.hpp:44-51)."""

    l: int
    exps: List[float]
    coefs: List[float]


@dataclass
class BasisSet:
    """Shells per atomic number (chem/GTO.hpp:55-57)."""

    name: str = ""
    elements: Dict[int, List[Shell]] = field(default_factory=dict)

    def shells_for(self, z: int) -> List[Shell]:
        if z not in self.elements or not self.elements[z]:
            raise BasisError(f"No basis assigned to element {ELEMENT_SYMBOLS[z - 1]} (Z={z})")
        return self.elements[z]


def _parse_float(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "E"))


def parse_basis_text(text: str, name: str = "") -> BasisSet:
    lines = text.splitlines()
    out = BasisSet(name=name)
    i = 0
    n = len(lines)
    while i < n:
        toks = lines[i].split()
        if len(toks) >= 2 and element_number(toks[0]) and toks[1] == "0":
            z = element_number(toks[0])
            i += 1
            # ECP blocks (first token ending in "ECP") are skipped.
            if i < n and lines[i].split() and lines[i].split()[0].endswith("ECP"):
                continue
            shells: List[Shell] = []
            while i < n:
                st = lines[i].split()
                if not st:
                    i += 1
                    continue
                if st[0].startswith("*"):
                    break
                typ = st[0]
                if typ != "SP" and (len(typ) != 1 or typ not in _L_LETTERS):
                    raise BasisError(
                        f"{typ[0]} is not a recognized angular momentum abbreviation. "
                        "Accepted values are S, P, D etc. as well as SP.")
                nprim = int(st[1])
                if nprim < 1 or nprim > 100:
                    raise BasisError(
                        f"Specified number of primitives ({nprim}) is outside of the accepted range of 1-100.")
                exps: List[float] = []
                c0: List[float] = []
                c1: List[float] = []
                for k in range(nprim):
                    i += 1
                    if i >= n:
                        raise BasisError("basis file ends inside a shell")
                    pt = lines[i].split()
                    zeta = _parse_float(pt[0])
                    if not zeta > 0.0:
                        raise BasisError("Primitive GTOs must have positive exponents!")
                    exps.append(zeta)
                    c0.append(_parse_float(pt[1]))
                    if typ == "SP":
                        c1.append(_parse_float(pt[2]))
                i += 1
                if typ == "SP":
                    shells.append(Shell(0, exps, c0))
                    shells.append(Shell(1, list(exps), c1))
                else:
                    shells.append(Shell(_L_LETTERS[typ], exps, c0))
            out.elements[z] = shells
        i += 1
    return out


def read_basis(path: str) -> BasisSet:
    if not os.path.isfile(path):
        raise BasisError(f"File '{path}' is empty or could not be found!")
    with open(path, "r") as f:
        return parse_basis_text(f.read(), os.path.basename(path))


_DATA = os.path.join(os.path.dirname(__file__), "data", "bases.json")
_BUILTIN_CACHE: Dict[str, BasisSet] = {}


def builtin_basis(name: str) -> BasisSet:
    """STO-3G, 6-31G and 6-31G* (file name 6-31GP) for H..Ne, extracted from the
    reference's basis/ directory by data/make_bases.py."""
    key = {"6-31G*": "6-31GP"}.get(name, name)
    if key not in _BUILTIN_CACHE:
        with open(_DATA) as f:
            data = json.load(f)
        if key not in data:
            raise BasisError(f"unknown builtin basis {name!r}; have {sorted(data)}")
        bs = BasisSet(name=key)
        for z, shells in data[key].items():
            bs.elements[int(z)] = [Shell(s["l"], s["exps"], s["coefs"]) for s in shells]
        _BUILTIN_CACHE[key] = bs
    return _BUILTIN_CACHE[key]


@dataclass
class Molecule:
    """Atomic numbers and positions in bohr (chem/Molecule.hpp:9-66).  The
    nuclear charge equals Z (chem/Molecule.cpp:12-18)."""

    Z: List[int]
    xyz: List[Tuple[float, float, float]]  # bohr

    @property
    def natom(self) -> int:
        return len(self.Z)

    def electron_count(self, charge: int = 0) -> int:
        return sum(self.Z) - charge

    def nuclear_repulsion(self) -> float:
        """Sum Z_A Z_B / R_AB (chem/scf/Energy.cpp:44-49)."""
        e = 0.0
        for i in range(self.natom):
            for j in range(i + 1, self.natom):
                d = sum((self.xyz[i][k] - self.xyz[j][k]) ** 2 for k in range(3)) ** 0.5
                e += self.Z[i] * self.Z[j] / d
        return e


def molecule_from_angstrom(symbols: Sequence[str], xyz_angstrom) -> Molecule:
    zs = []
    for s in symbols:
        z = element_number(s)
        if not z:
            raise GeometryError(
                f"'{s}' is not a valid element symbol. Check capitalization (e.g. Rn instead of RN)!")
        zs.append(z)
    pos = [tuple(float(c) * A_TO_BOHR for c in p) for p in xyz_angstrom]
    return Molecule(zs, pos)


def read_xyz(path: str) -> Molecule:
    if not os.path.isfile(path):
        raise GeometryError(f"File '{path}' is empty or could not be found!")
    with open(path) as f:
        lines = f.read().splitlines()
    if not lines or not lines[0].split():
        raise GeometryError("XYZ file has no atom count")
    count = int(lines[0].split()[0])
    syms, pos = [], []
    for line in lines[2:2 + count]:
        t = line.split()
        if not t:
            continue
        syms.append(t[0])
        pos.append([_parse_float(v) for v in t[1:4]])
    if len(syms) < count:
        raise GeometryError(
            f"{count} atoms expected in XYZ file, but only {len(syms)} were specified. "
            "Check for misplaced line breaks!")
    return molecule_from_angstrom(syms, pos)
