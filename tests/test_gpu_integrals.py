"""Device integrals against the golden vectors and the oracle (B200).

Every call goes through the C ABI (libhfjk.so via ctypes).
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200 import _lib
from oracle import dfrhf, kernels
from tests.helpers import molecule, tables, water_sto3g_pyscf_geometry

pytestmark = pytest.mark.gpu
INTEGRAL_TOL = 1e-12  # reference tests/tolerances.py:4
ORACLE_TOL = 1e-11


def context_for(orb, aux):
    ctx = _lib.Context(0)
    ctx.upload(orb, aux)
    return ctx


def test_metric_and_three_center_match_pyscf(pyscf_water):
    mol = water_sto3g_pyscf_geometry(pyscf_water["df_positions_bohr"])
    orb, aux = tables(mol, "sto-3g")
    ctx = context_for(orb, aux)
    np.testing.assert_allclose(ctx.metric(), pyscf_water["df_metric"], atol=INTEGRAL_TOL, rtol=0)
    np.testing.assert_allclose(ctx.three_center(), pyscf_water["df_three_center"], atol=INTEGRAL_TOL, rtol=0)


def test_one_electron_matches_pyscf(pyscf_water):
    mol = water_sto3g_pyscf_geometry(pyscf_water["one_positions_bohr"])
    orb, aux = tables(mol, "cc-pvdz")
    ctx = context_for(orb, aux)
    np.testing.assert_allclose(ctx.one_electron(0), pyscf_water["one_overlap"], atol=INTEGRAL_TOL, rtol=0)
    np.testing.assert_allclose(ctx.one_electron(1), pyscf_water["one_kinetic"], atol=INTEGRAL_TOL, rtol=0)
    v = ctx.one_electron(2, mol.nuclear_charges, mol.positions)
    np.testing.assert_allclose(v, pyscf_water["one_nuclear"], atol=INTEGRAL_TOL, rtol=0)


@pytest.mark.parametrize("tag", ["water", "h2o2_s0"])
def test_integrals_match_oracle_cc_pvdz(tag):
    mol = molecule(tag)
    orb, aux = tables(mol)
    ctx = context_for(orb, aux)
    np.testing.assert_allclose(ctx.metric(), dfrhf.metric(aux), atol=ORACLE_TOL, rtol=0)
    np.testing.assert_allclose(ctx.three_center(), dfrhf.three_center(aux, orb), atol=ORACLE_TOL, rtol=0)
    t = dfrhf.kernel_table(orb)
    z = np.zeros((1, 3))
    np.testing.assert_allclose(ctx.one_electron(0), kernels.overlap(t, t, z)[0], atol=ORACLE_TOL, rtol=0)
    np.testing.assert_allclose(ctx.one_electron(1), kernels.kinetic(t, t, z)[0], atol=ORACLE_TOL, rtol=0)
    np.testing.assert_allclose(
        ctx.one_electron(2, mol.nuclear_charges, mol.positions),
        kernels.nuclear_attraction(t, t, z, mol.nuclear_charges, mol.positions)[0], atol=ORACLE_TOL, rtol=0)


def test_fitted_repulsion_is_factor_invariant(pyscf_water):
    """sum_P B B = (uv|P) M^-1 (P|wx): Cholesky replaces the reference's M^-1/2
    (tests/unit/test_density_fitting.py:177-195 of the reference)."""
    mol = water_sto3g_pyscf_geometry(pyscf_water["df_positions_bohr"])
    orb, aux = tables(mol, "sto-3g")
    ctx = context_for(orb, aux)
    ctx.build()
    b = dfrhf.df_tensor(dfrhf.metric(aux), dfrhf.three_center(aux, orb))
    expected = np.einsum("Puv,Pwx->uvwx", b, b)
    np.testing.assert_allclose(ctx.fitted_eri(), expected, atol=1e-10, rtol=0)


def test_bad_shell_tables_raise_input_error():
    from hafnium_b200.errors import InputError

    mol = molecule("water")
    orb, aux = tables(mol)
    ctx = _lib.Context(0)
    bad = type(orb)(orb.angular_momenta, orb.centers, orb.primitive_offsets, -orb.exponents, orb.coefficients,
                    orb.n_contractions, orb.shell_atoms)
    with pytest.raises(InputError, match="exponents are positive"):
        ctx.upload(bad, aux)
    with pytest.raises(InputError, match="upload shells first"):
        ctx.build()


def test_four_center_matches_oracle():
    mol = molecule("water")
    orb, _ = tables(mol)
    ctx = _lib.Context(0)
    ctx.upload(orb)
    np.testing.assert_allclose(ctx.four_center(), dfrhf.eri_exact(orb), atol=ORACLE_TOL, rtol=0)
