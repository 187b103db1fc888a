"""Device DF-MP2 (hf_mp2_energy) against the PySCF fixture and the oracle (B200).

Mirrors tests/reference/test_mp2_reference.py:37-80 (stored case: water/STO-3G,
def2-universal-jkfit, reference converged with TIGHT options) and adds a
cc-pVDZ water dimer against the oracle's restatement of hafnium/mp/mp2.py.
"""

from __future__ import annotations

import pytest

from oracle import dfrhf
from tests.conftest import golden
from tests.helpers import molecule, tables, water_sto3g_pyscf_geometry

pytestmark = pytest.mark.gpu
TIGHT = dict(energy_tolerance=1e-13, gradient_tolerance=1e-9)


def device_mp2(mol, basis):
    from hafnium_b200.mp2 import df_mp2
    from hafnium_b200.scf import DeviceHamiltonian, ScfOptions, atomic_density_guess, solve_rhf

    ham = DeviceHamiltonian.build(mol, basis, "def2-universal-jkfit")
    ref = solve_rhf(ham, guess=atomic_density_guess(mol, basis), options=ScfOptions(**TIGHT))
    return df_mp2(ham, ref)


def test_dfmp2_matches_the_pyscf_fixture():
    g = golden("pyscf_water.npz")
    mol = water_sto3g_pyscf_geometry(g["df_positions_bohr"])
    result = device_mp2(mol, "sto-3g")
    assert abs(result.reference_energy - float(g["dfrhf_energy_sto3g"])) < 1e-9
    assert abs(result.correlation_energy - float(g["dfmp2_correlation_sto3g"])) < 1e-9


def test_dfmp2_matches_the_oracle_on_a_dimer():
    mol = molecule("h2o2_s0")
    orb, aux = tables(mol)
    prob = dfrhf.build_problem(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                               mol.n_alpha)
    guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    ref = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, mol.n_alpha, guess=guess, **TIGHT)
    expected = dfrhf.df_mp2(prob.b, ref.mo_energies, ref.mo_coefficients, mol.n_alpha)
    result = device_mp2(mol, "cc-pvdz")
    assert abs(result.reference_energy - ref.energy) < 1e-9
    assert abs(result.correlation_energy - expected) < 1e-9
