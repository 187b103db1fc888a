"""The oracle's nuclear gradient against the reference (CPU).

Pins, in the reference's own order of evidence
(tests/unit/test_derivative_integrals.py, tests/reference/test_gradient_reference.py):

* the derivative integrals against central differences of the integrals, as
  the reference's unit tests do (step 1e-5, FINITE_DIFFERENCE_TOL 1e-7);
* the five gradient terms against the reference's own ``nuclear_gradient``
  run at its converged state (tests/golden/reference_gradient_*.npz, made by
  tests/golden/make_golden.py with the reference's Python unchanged);
* the water/def2-SVP total against the PySCF gradient the reference stores,
  at its GRADIENT_TOL 1e-7.
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.basis import ShellTable
from hafnium_b200.molecule import Molecule, water
from oracle import dfrhf, kernels
from tests.conftest import golden

STEP = 1e-5
FINITE_DIFFERENCE_TOL = 1e-7  # tests/tolerances.py:116 of the reference
GRADIENT_TOL = 1e-7  # tests/tolerances.py:186
TERMS = ("nuclear_repulsion", "one_electron", "overlap", "coulomb", "exchange")
Z3 = np.zeros((1, 3))


def _tables(mol, basis):
    orb = ShellTable.build(basis, mol.symbols, mol.positions)
    aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
    return dfrhf.kernel_table(orb), dfrhf.kernel_table(aux), orb, aux


def _moved(mol, atom, axis, h):
    pos = mol.positions.copy()
    pos[atom, axis] += h
    return Molecule(mol.symbols, pos)


def _integrals(mol, basis):
    o, a, _, _ = _tables(mol, basis)
    return (
        kernels.overlap(o, o, Z3)[0],
        kernels.kinetic(o, o, Z3)[0],
        kernels.nuclear_attraction(o, o, Z3, mol.nuclear_charges, mol.positions)[0],
        kernels.coulomb_two_center(a, a, Z3)[0],
        kernels.coulomb_three_center(a, o, o, np.zeros((1, 2, 3)))[0],
    )


@pytest.mark.parametrize("basis", ["sto-3g", "cc-pvdz"])
def test_derivative_integrals_match_finite_differences(basis):
    mol = water()
    o, a, orb, aux = _tables(mol, basis)
    s_x = kernels.overlap_derivative(o, o, Z3)[0]
    t_x = kernels.kinetic_derivative(o, o, Z3)[0]
    v_x, v_nuc = kernels.nuclear_attraction_derivative(o, o, Z3, mol.nuclear_charges, mol.positions)
    m_x = kernels.coulomb_two_center_derivative(a, a, Z3)[0]
    by_aux, by_orb = kernels.coulomb_three_center_derivative(a, o, o, np.zeros((1, 2, 3)))
    on_orb = dfrhf.functions_by_atom(orb, mol.positions) > 0
    on_aux = dfrhf.functions_by_atom(aux, mol.positions) > 0

    def symmetric(d, mask):
        out = np.zeros_like(d)
        out[mask, :] += d[mask, :]
        out[:, mask] += d[mask, :].T
        return out

    for atom in range(mol.n_atoms):
        mask, amask = on_orb[atom], on_aux[atom]
        for axis in range(3):
            plus = _integrals(_moved(mol, atom, axis, STEP), basis)
            minus = _integrals(_moved(mol, atom, axis, -STEP), basis)
            numeric = [(p - m) / (2 * STEP) for p, m in zip(plus, minus)]
            three = np.zeros_like(by_aux[0][axis])
            three[amask] += by_aux[0][axis][amask]
            three[:, mask, :] += by_orb[0][axis][:, mask, :]
            three[:, :, mask] += np.transpose(by_orb[0][axis][:, mask, :], (0, 2, 1))
            analytic = [
                symmetric(s_x[axis], mask),
                symmetric(t_x[axis], mask),
                symmetric(v_x[0][axis], mask) + v_nuc[0][atom, axis],
                symmetric(m_x[axis], amask),
                three,
            ]
            for x, y in zip(analytic, numeric):
                np.testing.assert_allclose(x, y, atol=FINITE_DIFFERENCE_TOL, rtol=0)


@pytest.mark.parametrize("tag", ["water_pyscf", "water", "h2o2_s0"])
def test_oracle_gradient_matches_the_reference_run(tag):
    ref = golden(f"reference_gradient_{tag}.npz")
    mol = Molecule(tuple(str(s) for s in ref["symbols"]), ref["positions_bohr"])
    _, _, orb, aux = _tables(mol, str(ref["basis"]))
    got = dfrhf.nuclear_gradient(orb, aux, mol.nuclear_charges, mol.positions, ref["density"], ref["fock"])
    for term in TERMS:
        np.testing.assert_allclose(got[term], ref[term], atol=1e-10, rtol=0, err_msg=term)
    np.testing.assert_allclose(sum(got[t] for t in TERMS), ref["total"], atol=1e-10, rtol=0)


def test_reference_gradient_matches_stored_pyscf():
    ref = golden("reference_gradient_water_pyscf.npz")
    np.testing.assert_allclose(ref["total"], ref["pyscf_total"], atol=GRADIENT_TOL, rtol=0)
    # translational invariance: the forces sum to zero
    np.testing.assert_allclose(ref["total"].sum(axis=0), 0.0, atol=1e-9)


def test_planted_gradient_error_is_caught():
    """A Fock matrix of the wrong sign in the energy-weighted density moves the
    overlap term far beyond the tolerance."""
    ref = golden("reference_gradient_water.npz")
    mol = Molecule(tuple(str(s) for s in ref["symbols"]), ref["positions_bohr"])
    _, _, orb, aux = _tables(mol, str(ref["basis"]))
    got = dfrhf.nuclear_gradient(orb, aux, mol.nuclear_charges, mol.positions, ref["density"], -ref["fock"])
    assert np.max(np.abs(got["overlap"] - ref["overlap"])) > 1e-3


def test_derivative_integrals_are_translationally_invariant():
    """Moving every centre together changes no integral: the bra, ket and
    auxiliary (or nuclear) derivatives sum to zero. This is the identity the
    device kernels use for the second orbital centre."""
    mol = water()
    o, a, _, _ = _tables(mol, "cc-pvdz")
    s_x = kernels.overlap_derivative(o, o, Z3)[0]
    t_x = kernels.kinetic_derivative(o, o, Z3)[0]
    v_x, v_nuc = kernels.nuclear_attraction_derivative(o, o, Z3, mol.nuclear_charges, mol.positions)
    m_x = kernels.coulomb_two_center_derivative(a, a, Z3)[0]
    by_aux, by_orb = kernels.coulomb_three_center_derivative(a, o, o, np.zeros((1, 2, 3)))
    for axis in range(3):
        np.testing.assert_allclose(s_x[axis] + s_x[axis].T, 0.0, atol=1e-12)
        np.testing.assert_allclose(t_x[axis] + t_x[axis].T, 0.0, atol=1e-11)
        np.testing.assert_allclose(v_x[0][axis] + v_x[0][axis].T + v_nuc[0][:, axis].sum(axis=0), 0.0, atol=1e-10)
        np.testing.assert_allclose(m_x[axis] + m_x[axis].T, 0.0, atol=1e-11)
        total = by_aux[0][axis] + by_orb[0][axis] + np.transpose(by_orb[0][axis], (0, 2, 1))
        np.testing.assert_allclose(total, 0.0, atol=1e-11)
