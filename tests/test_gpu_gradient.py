"""The DF-RHF nuclear gradient on the device against the reference (B200).

The reference's own ``nuclear_gradient`` at its converged states
(tests/golden/reference_gradient_*.npz) is matched term by term, through the
drop-in's host NumPy entry point, to REFERENCE_GRADIENT_TOL 1e-8
(tests/tolerances.py:137 of the reference); the device SCF followed by the
device gradient matches the PySCF gradient the reference stores for
water/def2-SVP at its GRADIENT_TOL 1e-7 and the oracle on its own state.
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.gradient import gradient_from_state, nuclear_gradient, occupied_factor
from hafnium_b200.jk import B200DensityFittedCoulombExchange
from hafnium_b200.molecule import Molecule
from tests.conftest import golden

pytestmark = pytest.mark.gpu
REFERENCE_GRADIENT_TOL = 1e-8
GRADIENT_TOL = 1e-7
TERMS = ("nuclear_repulsion", "one_electron", "overlap", "coulomb", "exchange")


def _fixture(tag):
    ref = golden(f"reference_gradient_{tag}.npz")
    mol = Molecule(tuple(str(s) for s in ref["symbols"]), ref["positions_bohr"])
    return ref, mol


@pytest.mark.parametrize("tag", ["water_pyscf", "water", "h2o2_s0", "h2o4_s1"])
def test_gradient_terms_match_the_reference_run(tag):
    from hafnium_b200.basis import ShellTable
    from oracle import dfrhf

    ref, mol = _fixture(tag)
    basis = str(ref["basis"])
    orb = ShellTable.build(basis, mol.symbols, mol.positions)
    aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
    two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    occ = occupied_factor(ref["density"], dfrhf.overlap(orb), mol.n_alpha)
    grad = gradient_from_state(two_body, occ, ref["fock"], mol)
    for term in TERMS:
        err = float(np.max(np.abs(getattr(grad, term) - ref[term])))
        print(f"{tag} {term}: max |dG| = {err:.2e}")
        assert err <= REFERENCE_GRADIENT_TOL, term
    assert np.max(np.abs(grad.total - ref["total"])) <= REFERENCE_GRADIENT_TOL


def test_device_scf_gradient_matches_stored_pyscf():
    from hafnium_b200.scf import DeviceHamiltonian, ScfOptions, atomic_density_guess, solve_rhf

    ref, mol = _fixture("water_pyscf")
    ham = DeviceHamiltonian.build(mol, "def2-svp", "def2-universal-jkfit")
    result = solve_rhf(ham, guess=atomic_density_guess(mol, "def2-svp"),
                       options=ScfOptions(energy_tolerance=1e-12, gradient_tolerance=1e-9))
    grad = nuclear_gradient(ham, result, mol)
    np.testing.assert_allclose(grad.total, ref["pyscf_total"], atol=GRADIENT_TOL, rtol=0)
    np.testing.assert_allclose(grad.total.sum(axis=0), 0.0, atol=1e-8)


def test_device_gradient_matches_the_oracle_on_a_cluster():
    from hafnium_b200.basis import ShellTable
    from hafnium_b200.molecule import water_cluster
    from hafnium_b200.scf import DeviceHamiltonian, ScfOptions, atomic_density_guess, solve_rhf
    from oracle import dfrhf

    mol = water_cluster(3, 7)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    result = solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"),
                       options=ScfOptions(energy_tolerance=1e-12, gradient_tolerance=1e-9))
    grad = nuclear_gradient(ham, result, mol)
    orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
    aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
    want = dfrhf.nuclear_gradient(orb, aux, mol.nuclear_charges, mol.positions, result.density.cpu().numpy(),
                                  result.fock.cpu().numpy())
    for term in TERMS:
        np.testing.assert_allclose(getattr(grad, term), want[term], atol=REFERENCE_GRADIENT_TOL, rtol=0,
                                   err_msg=term)
    np.testing.assert_allclose(grad.total.sum(axis=0), 0.0, atol=1e-8)
