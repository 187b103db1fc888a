"""Molecules and shell tables shared by the test modules."""

from __future__ import annotations

import numpy as np

from hafnium_b200.basis import ShellTable
from hafnium_b200.molecule import Molecule, water, water_cluster

GOLDEN_CLUSTERS = {"water": (1, None), "h2o2_s0": (2, 0), "h2o4_s1": (4, 1), "h2o8_s2": (8, 2)}


def molecule(tag: str) -> Molecule:
    n, seed = GOLDEN_CLUSTERS[tag]
    return water() if seed is None else water_cluster(n, seed)


def molecule_bohr(symbols, positions) -> Molecule:
    return Molecule(tuple(symbols), np.asarray(positions, dtype=np.float64))


def tables(mol: Molecule, basis: str = "cc-pvdz", aux: str = "def2-universal-jkfit"):
    return (ShellTable.build(basis, mol.symbols, mol.positions), ShellTable.build(aux, mol.symbols, mol.positions))


def water_sto3g_pyscf_geometry(positions) -> Molecule:
    return molecule_bohr(("O", "H", "H"), positions)
