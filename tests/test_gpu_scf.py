"""Whole DF-RHF on the device against the reference's recorded runs (B200).

|dE| <= 1e-8 Eh and max|dD| <= 1e-6 against the reference's own DF-RHF
(tests/golden/reference_dfrhf_*.npz, made by tests/golden/make_golden.py).
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.scf import DeviceHamiltonian, ScfOptions, solve_rhf
from tests.conftest import golden
from tests.helpers import molecule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["water", "h2o2_s0", "h2o4_s1", "h2o8_s2"])
def test_device_dfrhf_matches_reference(tag):
    ref = golden(f"reference_dfrhf_{tag}.npz")
    mol = molecule(tag)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    result = solve_rhf(ham, options=ScfOptions(energy_tolerance=1e-11, gradient_tolerance=1e-8))
    assert result.converged
    assert abs(result.energy - float(ref["energy"])) <= 1e-8
    assert np.max(np.abs(result.density.cpu().numpy() - ref["density"])) <= 1e-6
