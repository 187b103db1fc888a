"""The oracle against the reference's golden vectors (CPU).

The oracle (oracle/md_oracle.cpp + oracle/dfrhf.py) restates the reference's
integrals and DF-RHF; these tests pin it to values the reference stores
(PySCF/libcint fixtures from tests/reference/data) and to the reference's own
DF-RHF runs recorded by tests/golden/make_golden.py.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import dfrhf, kernels
from tests.conftest import golden
from tests.helpers import molecule, tables, water_sto3g_pyscf_geometry

INTEGRAL_TOL = 1e-12  # tests/tolerances.py:4 of the reference
ENERGY_TOL = 1e-10  # tests/tolerances.py:3


def test_boys_matches_series_and_closed_form():
    import mpmath

    mpmath.mp.dps = 30
    for t in (0.0, 0.3, 7.0, 34.999, 35.0, 60.0, 1e4):
        values = kernels.boys_function(12, t)
        for n in (0, 3, 8, 12):
            if t == 0.0:
                expected = 1.0 / (2 * n + 1)
            else:
                half = mpmath.mpf(n) + mpmath.mpf(1) / 2
                expected = float(mpmath.gammainc(half, 0, t) / (2 * mpmath.mpf(t) ** half))
            assert values[n] == pytest.approx(expected, rel=1e-14)


def test_stored_pyscf_metric_and_three_center(pyscf_water):
    mol = water_sto3g_pyscf_geometry(pyscf_water["df_positions_bohr"])
    orb, aux = tables(mol, "sto-3g")
    np.testing.assert_allclose(dfrhf.metric(aux), pyscf_water["df_metric"], atol=INTEGRAL_TOL, rtol=0)
    np.testing.assert_allclose(dfrhf.three_center(aux, orb), pyscf_water["df_three_center"], atol=INTEGRAL_TOL, rtol=0)


def test_stored_pyscf_one_electron(pyscf_water):
    mol = water_sto3g_pyscf_geometry(pyscf_water["one_positions_bohr"])
    orb, _ = tables(mol, "cc-pvdz")
    t = dfrhf.kernel_table(orb)
    zero = np.zeros((1, 3))
    np.testing.assert_allclose(kernels.overlap(t, t, zero)[0], pyscf_water["one_overlap"], atol=INTEGRAL_TOL, rtol=0)
    np.testing.assert_allclose(kernels.kinetic(t, t, zero)[0], pyscf_water["one_kinetic"], atol=INTEGRAL_TOL, rtol=0)
    v = kernels.nuclear_attraction(t, t, zero, mol.nuclear_charges, mol.positions)[0]
    np.testing.assert_allclose(v, pyscf_water["one_nuclear"], atol=INTEGRAL_TOL, rtol=0)


def test_stored_pyscf_dfrhf_energy(pyscf_water):
    """The reference's stored PySCF DF-RHF energy of water/STO-3G (mp2_water_sto-3g.json)."""
    mol = water_sto3g_pyscf_geometry(pyscf_water["df_positions_bohr"])
    orb, aux = tables(mol, "sto-3g")
    prob = dfrhf.build_problem(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                               mol.n_alpha)
    result = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, prob.n_alpha,
                             energy_tolerance=1e-13, gradient_tolerance=1e-9)
    assert result.energy == pytest.approx(float(pyscf_water["dfrhf_energy_sto3g"]), abs=ENERGY_TOL)


@pytest.mark.parametrize("tag", ["water", "h2o2_s0"])
def test_reference_dfrhf_runs(tag):
    """The oracle's DF-RHF reproduces the reference's own run on the same cluster."""
    ref = golden(f"reference_dfrhf_{tag}.npz")
    mol = molecule(tag)
    np.testing.assert_allclose(mol.positions, ref["positions_bohr"], atol=1e-14)
    orb, aux = tables(mol)
    prob = dfrhf.build_problem(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                               mol.n_alpha)
    guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    result = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, prob.n_alpha, guess=guess)
    assert result.energy == pytest.approx(float(ref["energy"]), abs=ENERGY_TOL)
    assert result.n_iterations == int(ref["n_iterations"])
    np.testing.assert_allclose(result.density, ref["density"], atol=1e-9)
    np.testing.assert_allclose([h.energy for h in result.history], ref["history"], atol=1e-9)


def test_lean_oracle_reproduces_the_reference_run_at_twelve_waters():
    """The memory-lean restatement (in-place fit, exchange through an occupied
    factor), which makes the (H2O)32 fixture, against the reference's own run on
    (H2O)12 (n = 288): the same energy, density and iteration count."""
    from tests.helpers import golden_run

    ref = golden_run("h2o12_s3")
    mol = molecule("h2o12_s3")
    np.testing.assert_allclose(mol.positions, ref["positions_bohr"], atol=1e-14)
    orb, aux = tables(mol)
    prob = dfrhf.build_problem_lean(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                                    mol.n_alpha)
    guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    result = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.LeanFittedJK(prob.b), prob.e_nuc, prob.n_alpha, guess=guess)
    assert result.energy == pytest.approx(float(ref["energy"]), abs=ENERGY_TOL)
    assert result.n_iterations == int(ref["n_iterations"])
    np.testing.assert_allclose(result.density, ref["density"], atol=1e-9)


def test_lean_exchange_refuses_an_indefinite_density():
    b = np.random.default_rng(0).normal(size=(3, 4, 4))
    with pytest.raises(ValueError, match="positive semidefinite"):
        dfrhf.LeanFittedJK(b).exchange(np.diag([1.0, -1.0, 0.5, 0.0]))


def test_planted_error_is_caught(pyscf_water):
    """A metric with one element perturbed by 1e-10 fails the 1e-12 check."""
    mol = water_sto3g_pyscf_geometry(pyscf_water["df_positions_bohr"])
    _, aux = tables(mol, "sto-3g")
    m = dfrhf.metric(aux)
    m[3, 5] += 1e-10
    with pytest.raises(AssertionError):
        np.testing.assert_allclose(m, pyscf_water["df_metric"], atol=INTEGRAL_TOL, rtol=0)


def test_oracle_dfmp2_matches_the_pyscf_fixture():
    """tests/reference/test_mp2_reference.py:37-60 (stored case): water/STO-3G with
    def2-universal-jkfit, the reference converged with TIGHT options."""
    g = golden("pyscf_water.npz")
    mol = water_sto3g_pyscf_geometry(g["df_positions_bohr"])
    orb, aux = tables(mol, "sto-3g")
    prob = dfrhf.build_problem(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                               mol.n_alpha)
    res = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, mol.n_alpha,
                          energy_tolerance=1e-13, gradient_tolerance=1e-9)
    assert abs(res.energy - float(g["dfrhf_energy_sto3g"])) < 1e-10
    e2 = dfrhf.df_mp2(prob.b, res.mo_energies, res.mo_coefficients, mol.n_alpha)
    assert abs(e2 - float(g["dfmp2_correlation_sto3g"])) < 1e-10
