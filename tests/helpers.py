"""Molecules and shell tables shared by the test modules."""

from __future__ import annotations

import numpy as np

from hafnium_b200.basis import ShellTable
from hafnium_b200.molecule import Molecule, water, water_cluster

GOLDEN_CLUSTERS = {"water": (1, None), "h2o2_s0": (2, 0), "h2o4_s1": (4, 1), "h2o8_s2": (8, 2),
                   "h2o12_s3": (12, 3), "h2o16_s0": (16, 0), "h2o32_s0": (32, 0)}


def molecule(tag: str) -> Molecule:
    n, seed = GOLDEN_CLUSTERS[tag]
    return water() if seed is None else water_cluster(n, seed)


def molecule_bohr(symbols, positions) -> Molecule:
    return Molecule(tuple(symbols), np.asarray(positions, dtype=np.float64))


def tables(mol: Molecule, basis: str = "cc-pvdz", aux: str = "def2-universal-jkfit"):
    return (ShellTable.build(basis, mol.symbols, mol.positions), ShellTable.build(aux, mol.symbols, mol.positions))


def water_sto3g_pyscf_geometry(positions) -> Molecule:
    return molecule_bohr(("O", "H", "H"), positions)


def golden_run(tag: str) -> dict:
    """The recorded DF-RHF of cluster ``tag``: the reference's own run
    (``reference_dfrhf_*.npz``) where one exists, else the oracle's lean
    restatement (``oracle_dfrhf_*.npz``, pinned by the reference runs at 12 and
    16 waters). The density is rebuilt from its stored occupied factor where the
    file holds one (D = F F^T)."""
    from tests.conftest import GOLDEN, golden

    name = f"reference_dfrhf_{tag}.npz"
    data = golden(name if (GOLDEN / name).exists() else f"oracle_dfrhf_{tag}.npz")
    if "density" not in data:
        f = data["density_factor"]
        data["density"] = f @ f.T
    return data

