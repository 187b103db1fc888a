"""The drop-in's boundary against the reference's own objects (CPU).

``ShellTable.from_reference`` takes the caller's ``BasisSet`` and ``Molecule``
(hafnium/integrals/shell_table.py:84-116); these tests build them with the
reference's own Python package and check that the table equals both the
reference's ``ShellTable.from_basis`` and this package's ``ShellTable.build``,
and that a basis laid out for other atoms is refused
(shell_table.py:141-154). They need the reference tree (HF_REFERENCE_ROOT, or
a ``reference`` directory beside the repository) and skip without it.
"""

from __future__ import annotations

import os
import pathlib

import numpy as np
import pytest

from hafnium_b200.basis import ShellTable
from hafnium_b200.errors import InputError
from hafnium_b200.molecule import water_cluster

ROOT = pathlib.Path(__file__).resolve().parent.parent
FIELDS = ("angular_momenta", "centers", "primitive_offsets", "exponents", "coefficients", "n_contractions")


def reference_root() -> pathlib.Path | None:
    named = os.environ.get("HF_REFERENCE_ROOT")
    candidate = pathlib.Path(named) if named else ROOT.parent / "reference"
    return candidate if (candidate / "hafnium" / "integrals" / "shell_table.py").exists() else None


@pytest.fixture(scope="module")
def reference():
    root = reference_root()
    if root is None:
        pytest.skip("the reference tree is not available")
    from oracle import reference_env

    reference_env.install(root)
    import hafnium

    return hafnium


def reference_molecule(mol):
    from hafnium.molecule import Molecule

    return Molecule.from_atoms(list(zip(mol.symbols, map(tuple, mol.positions))), unit="bohr")


@pytest.mark.parametrize("name", ["cc-pvdz", "def2-universal-jkfit", "sto-3g", "def2-svp"])
def test_from_reference_equals_the_reference_table_and_build(reference, name):
    from hafnium.basis import BasisLibrary, BasisSet
    from hafnium.integrals import ShellTable as ReferenceTable

    mol = water_cluster(3, 1)
    ref_mol = reference_molecule(mol)
    basis = BasisSet.for_atoms(ref_mol, name, library=BasisLibrary(offline=True))
    ours = ShellTable.from_reference(basis, ref_mol)
    theirs = ReferenceTable.from_basis(basis, ref_mol)
    built = ShellTable.build(name, mol.symbols, mol.positions)
    for field in FIELDS:
        got = np.asarray(getattr(ours, field))
        np.testing.assert_array_equal(got, np.asarray(getattr(theirs, field)), err_msg=field)
        np.testing.assert_allclose(got, np.asarray(getattr(built, field)), rtol=1e-15, atol=0, err_msg=field)
    assert ours.n_functions == basis.n_functions


def test_from_reference_refuses_a_basis_for_other_atoms(reference):
    from hafnium.basis import BasisLibrary, BasisSet

    mol = water_cluster(2, 0)
    ref_mol = reference_molecule(mol)
    basis = BasisSet.for_atoms(ref_mol, "cc-pvdz", library=BasisLibrary(offline=True))
    other = reference_molecule(water_cluster(3, 0))
    with pytest.raises(InputError, match="lay the basis out"):
        ShellTable.from_reference(basis, other)
