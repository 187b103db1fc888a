"""Basis sets and the structure-of-arrays shell table the device kernels consume.

The layout is the reference's ``ShellTable`` (hafnium/integrals/shell_table.py:14-82):
one entry per shell with all its contractions (a general contraction stays one
entry), ``primitive_offsets[shell + 1]``, bare-primitive coefficients stored shell
by shell as ``[contraction][primitive]``, and functions ordered contraction-major,
then ``m`` (p shells x, y, z). Coefficients are made unit-norm exactly as
``Shell.primitive_coefficients`` does (hafnium/basis/shell.py:22-31, 87-104).

Basis data ships in ``basis_data/`` (Basis Set Exchange JSON, BSD-3-Clause) for
H, He, C, N and O in sto-3g, cc-pvdz, def2-svp and def2-universal-jkfit.
"""

from __future__ import annotations

import functools
import json
import math
import pathlib
from dataclasses import dataclass

import numpy as np

from hafnium_b200.errors import InputError

DATA = pathlib.Path(__file__).resolve().parent / "basis_data"


def primitive_norm(exponent: float, l: int) -> float:
    """Norm of ``r^l exp(-a r^2)`` times a unit-norm real solid harmonic (shell.py:22-25)."""
    power = l + 1.5
    return math.sqrt(2.0 * (2.0 * exponent) ** power / math.gamma(power))


def primitive_overlap(a: float, b: float, l: int) -> float:
    """Overlap of two normalised same-harmonic primitives on one centre (shell.py:28-31)."""
    return (2.0 * math.sqrt(a * b) / (a + b)) ** (l + 1.5)


@dataclass(frozen=True, slots=True)
class Shell:
    """A contracted shell: ``l``, exponents, and one coefficient row per contraction."""

    l: int
    exponents: tuple[float, ...]
    coefficients: tuple[tuple[float, ...], ...]

    @property
    def n_functions(self) -> int:
        return len(self.coefficients) * (2 * self.l + 1)

    def primitive_coefficients(self) -> tuple[tuple[float, ...], ...]:
        """Bare-primitive coefficients that give every contraction unit norm."""
        norms = [primitive_norm(a, self.l) for a in self.exponents]
        rows = []
        for row in self.coefficients:
            square = sum(
                ci * cj * primitive_overlap(ai, aj, self.l)
                for ci, ai in zip(row, self.exponents)
                for cj, aj in zip(row, self.exponents)
            )
            if square <= 0.0:
                raise InputError("a contraction has zero norm")
            scale = 1.0 / math.sqrt(square)
            rows.append(tuple(c * n * scale for c, n in zip(row, norms)))
        return tuple(rows)


@functools.lru_cache(maxsize=None)
def _element_block(name: str, z: int):
    """One atom's part of a ShellTable for element z in basis ``name``: angular
    momenta, primitives per shell, exponents, normalised coefficients (each
    shell's contractions one after another) and contractions per shell; None
    when the basis has no functions for z. Computed once per basis and element."""
    shells = element_shells(name).get(z)
    if not shells:
        return None
    ls, nprim, exps, coefs, ks = [], [], [], [], []
    for shell in shells:
        rows = shell.primitive_coefficients()
        ls.append(shell.l)
        nprim.append(len(shell.exponents))
        exps.extend(shell.exponents)
        for row in rows:
            coefs.extend(row)
        ks.append(len(rows))
    return (np.asarray(ls, dtype=np.int64), np.asarray(nprim, dtype=np.int64), np.asarray(exps, dtype=np.float64),
            np.asarray(coefs, dtype=np.float64), np.asarray(ks, dtype=np.int64))


@functools.lru_cache(maxsize=None)
def element_shells(name: str) -> dict[int, tuple[Shell, ...]]:
    """Shells per atomic number of a shipped basis set (library.py:47-72 splitting)."""
    path = DATA / f"{name.lower()}.json"
    if not path.exists():
        raise InputError(f"basis set {name!r} is not shipped; available: "
                         + ", ".join(sorted(p.stem for p in DATA.glob('*.json'))))
    data = json.loads(path.read_text(encoding="utf-8"))
    out: dict[int, tuple[Shell, ...]] = {}
    for z, element in data["elements"].items():
        shells: list[Shell] = []
        for entry in element["electron_shells"]:
            momenta = list(entry["angular_momentum"])
            exps = tuple(float(a) for a in entry["exponents"])
            rows = [tuple(float(c) for c in row) for row in entry["coefficients"]]
            if len(momenta) == 1:
                shells.append(Shell(momenta[0], exps, tuple(rows)))
            else:
                shells.extend(Shell(l, exps, (row,)) for l, row in zip(momenta, rows))
        out[int(z)] = tuple(shells)
    return out


@dataclass(frozen=True, slots=True, eq=False)
class ShellTable:
    """Shells laid out on atoms in structure-of-arrays form (host arrays)."""

    angular_momenta: np.ndarray  # int64 [shell]
    centers: np.ndarray  # float64 [shell, 3], Bohr
    primitive_offsets: np.ndarray  # int64 [shell + 1]
    exponents: np.ndarray  # float64 [primitive]
    coefficients: np.ndarray  # float64 [sum_s k_s * p_s]
    n_contractions: np.ndarray  # int64 [shell]
    shell_atoms: np.ndarray  # int64 [shell]

    @property
    def n_shells(self) -> int:
        return int(self.angular_momenta.shape[0])

    @property
    def n_functions(self) -> int:
        return int(np.sum(self.n_contractions * (2 * self.angular_momenta + 1)))

    @property
    def max_l(self) -> int:
        return int(self.angular_momenta.max()) if self.n_shells else 0

    def function_offsets(self) -> np.ndarray:
        sizes = self.n_contractions * (2 * self.angular_momenta + 1)
        return np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)

    @classmethod
    def build(cls, name: str, symbols, positions) -> "ShellTable":
        """Lay out basis ``name`` on atoms ``symbols`` at ``positions`` (Bohr): each
        atom's shells, exponents and normalised coefficients in the order of the
        element's shells, atoms in order."""
        from hafnium_b200.molecule import atomic_number

        positions = np.asarray(positions, dtype=np.float64)
        parts = []
        for symbol in symbols:
            z = atomic_number(symbol)
            block = _element_block(name, z)
            if block is None:
                raise InputError(f"basis set {name!r} has no functions for {symbol}")
            parts.append(block)
        if not parts:
            none = np.zeros(0, dtype=np.int64)
            return cls(none, np.zeros((0, 3)), np.zeros(1, dtype=np.int64), np.zeros(0), np.zeros(0), none, none)
        nsh = np.array([len(b[0]) for b in parts])
        nprim = np.concatenate([b[1] for b in parts])
        return cls(
            np.concatenate([b[0] for b in parts]),
            np.repeat(positions[: len(parts)], nsh, axis=0).reshape(-1, 3),
            np.concatenate([[0], np.cumsum(nprim)]).astype(np.int64),
            np.concatenate([b[2] for b in parts]),
            np.concatenate([b[3] for b in parts]),
            np.concatenate([b[4] for b in parts]),
            np.repeat(np.arange(len(parts), dtype=np.int64), nsh),
        )

    @classmethod
    def from_reference(cls, basis, molecule) -> "ShellTable":
        """Lay out a reference ``BasisSet`` on a reference ``Molecule``.

        Mirrors ``ShellTable.from_basis`` (hafnium/integrals/shell_table.py:84-116)
        by duck typing, so the drop-in accepts the caller's own objects. A basis
        laid out for other elements than the molecule's is refused, as the
        reference's ``require_basis_for_atoms`` (shell_table.py:141-154) does.
        """
        basis_symbols = tuple(getattr(basis, "atom_symbols", ()))
        molecule_symbols = tuple(molecule.symbols)
        if basis_symbols != molecule_symbols:
            raise InputError(f"the basis belongs to atoms {list(basis_symbols)}, the molecule has "
                             f"{list(molecule_symbols)}; lay the basis out for this molecule's atoms")
        positions = np.asarray(molecule.positions_array(), dtype=np.float64)
        ls, centers, offsets, exps, coefs, ks, atoms = [], [], [0], [], [], [], []
        for shell, atom in zip(basis.shells, basis.shell_atoms):
            rows = shell.primitive_coefficients()
            ls.append(int(shell.angular_momentum))
            centers.append(positions[atom])
            exps.extend(shell.exponents)
            offsets.append(len(exps))
            for row in rows:
                coefs.extend(row)
            ks.append(len(rows))
            atoms.append(int(atom))
        return cls(
            np.asarray(ls, dtype=np.int64),
            np.asarray(centers, dtype=np.float64).reshape(-1, 3),
            np.asarray(offsets, dtype=np.int64),
            np.asarray(exps, dtype=np.float64),
            np.asarray(coefs, dtype=np.float64),
            np.asarray(ks, dtype=np.int64),
            np.asarray(atoms, dtype=np.int64),
        )
