"""Molecules and the seeded water clusters the workloads run on.

Positions are in Bohr inside the package; ``from_atoms`` converts from Angstrom
with the CODATA-2018 Bohr radius (hafnium/molecule/units.py:6-9). The nuclear
repulsion is the pairwise sum of hafnium/molecule/molecule.py:45-56.

A water cluster ``(H2O)n`` is built from rigid waters (O-H 0.9572 A, H-O-H
104.52 deg) with a uniformly random orientation (Haar-distributed unit
quaternion) and oxygens placed uniformly in a cube sized for a density of
1 g/cm^3, rejecting any oxygen closer than 2.7 A to one already placed.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from hafnium_b200.errors import InputError

BOHR_IN_ANGSTROM = 0.529177210903
ANGSTROM_IN_BOHR = 1.0 / BOHR_IN_ANGSTROM
AVOGADRO = 6.02214076e23
WATER_MOLAR_MASS = 18.015  # g/mol

_Z = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10}


def atomic_number(symbol: str) -> int:
    try:
        return _Z[symbol]
    except KeyError as error:
        raise InputError(f"unknown element {symbol!r}") from error


@dataclass(frozen=True, slots=True, eq=False)
class Molecule:
    """Atoms (symbols, Bohr positions), total charge; closed shells only."""

    symbols: tuple[str, ...]
    positions: np.ndarray  # [atom, 3] Bohr
    charge: int = 0

    @classmethod
    def from_atoms(cls, atoms, charge: int = 0, unit: str = "angstrom") -> "Molecule":
        scale = ANGSTROM_IN_BOHR if unit == "angstrom" else 1.0
        symbols = tuple(a[0] for a in atoms)
        positions = np.asarray([a[1] for a in atoms], dtype=np.float64) * scale
        return cls(symbols, positions, charge)

    @property
    def n_atoms(self) -> int:
        return len(self.symbols)

    @property
    def nuclear_charges(self) -> np.ndarray:
        return np.asarray([atomic_number(s) for s in self.symbols], dtype=np.float64)

    @property
    def n_electrons(self) -> int:
        return int(self.nuclear_charges.sum()) - self.charge

    @property
    def n_alpha(self) -> int:
        if self.n_electrons % 2:
            raise InputError("only closed-shell molecules are supported")
        return self.n_electrons // 2

    def nuclear_repulsion_energy(self) -> float:
        z = self.nuclear_charges
        energy = 0.0
        for i in range(self.n_atoms):
            for j in range(i + 1, self.n_atoms):
                distance = math.dist(self.positions[i], self.positions[j])
                if distance == 0.0:
                    raise InputError(f"atoms {i} and {j} coincide")
                energy += z[i] * z[j] / distance
        return energy


def water() -> Molecule:
    """Water near equilibrium, C2v in the yz plane (the reference's test molecule)."""
    return Molecule.from_atoms(
        [("O", (0.0, 0.0, 0.1173)), ("H", (0.0, 0.7572, -0.4692)), ("H", (0.0, -0.7572, -0.4692))]
    )


def _rotation(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
        ]
    )


def cube_side_angstrom(n_waters: int, density_g_cm3: float = 1.0) -> float:
    volume_cm3 = n_waters * WATER_MOLAR_MASS / (AVOGADRO * density_g_cm3)
    return volume_cm3 ** (1.0 / 3.0) * 1e8


def water_cluster(n_waters: int, seed: int, *, min_oo: float = 2.7, max_tries: int = 100000) -> Molecule:
    """Seeded ``(H2O)n``: atoms ordered O, H, H per water, positions in Bohr."""
    if n_waters < 1:
        raise InputError("a cluster holds at least one water")
    rng = np.random.default_rng(seed)
    side = cube_side_angstrom(n_waters)
    r, half = 0.9572, math.radians(104.52) / 2
    local = np.array([[0.0, 0.0, 0.0], [r * math.sin(half), 0.0, r * math.cos(half)],
                      [-r * math.sin(half), 0.0, r * math.cos(half)]])
    oxygens: list[np.ndarray] = []
    atoms = []
    tries = 0
    while len(oxygens) < n_waters:
        tries += 1
        if tries > max_tries:
            raise InputError(f"could not place {n_waters} waters at O-O >= {min_oo} A")
        candidate = rng.uniform(0.0, side, size=3)
        if any(np.linalg.norm(candidate - o) < min_oo for o in oxygens):
            continue
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        placed = candidate + local @ _rotation(q).T
        oxygens.append(candidate)
        atoms += [("O", tuple(placed[0])), ("H", tuple(placed[1])), ("H", tuple(placed[2]))]
    return Molecule.from_atoms(atoms)
