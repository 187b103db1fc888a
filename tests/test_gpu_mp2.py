"""Device DF-MP2 (hf_mp2_energy) against the PySCF fixture and the oracle (B200).

Mirrors tests/reference/test_mp2_reference.py:37-80 (stored case: water/STO-3G,
def2-universal-jkfit, reference converged with TIGHT options) and adds a
cc-pVDZ water dimer against the oracle's restatement of hafnium/mp/mp2.py, and
the orbital-basis fitted tensor (hf_mo_fitted_tensor) the same consumers read.
"""

from __future__ import annotations

import numpy as np
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


def test_orbital_basis_tensor_contractions_match_the_oracle():
    """transform_df_tensor (orbitals/integrals.py:73-157) on the device: the
    orbital-basis four-index products sum_P B[P,p,q] B[P,r,s] against the
    oracle's tensor M^-1/2 (P|uv) (the auxiliary gauges differ by a rotation)."""
    from hafnium_b200.jk import B200DensityFittedCoulombExchange
    from oracle import dfrhf
    from tests.helpers import molecule, tables

    mol = molecule("h2o2_s0")
    orb, aux = tables(mol)
    two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    b = dfrhf.df_tensor(dfrhf.metric(aux), dfrhf.three_center(aux, orb))
    rng = np.random.default_rng(4)
    cb = rng.normal(size=(two_body.n_ao, 5)) / np.sqrt(two_body.n_ao)
    ck = rng.normal(size=(two_body.n_ao, 7)) / np.sqrt(two_body.n_ao)
    got = two_body.orbital_tensor(cb, ck)
    want = np.einsum("up,Puv,vq->Ppq", cb, b, ck)
    assert got.shape == want.shape
    g = got.reshape(got.shape[0], -1)
    w = want.reshape(want.shape[0], -1)
    np.testing.assert_allclose(g.T @ g, w.T @ w, atol=1e-10, rtol=0)
