"""Whole DF-RHF on the device against the reference's recorded runs (B200).

|dE| <= 1e-8 Eh and max|dD| <= 1e-6 against the reference's own DF-RHF
(tests/golden/reference_dfrhf_*.npz, made by tests/golden/make_golden.py) up to
(H2O)16 (n = 384; (H2O)12 has n = 288, which the split-BF16 builds pad to an odd
multiple of 128), and against the oracle's lean restatement at (H2O)32 (n = 768,
oracle_dfrhf_h2o32_s0.npz), which the reference runs at 12 and 16 waters pin.
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.scf import DeviceHamiltonian, ScfOptions, solve_rhf
from tests.helpers import golden_run, molecule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["water", "h2o2_s0", "h2o4_s1", "h2o8_s2", "h2o12_s3", "h2o16_s0", "h2o32_s0"])
def test_device_dfrhf_matches_reference(tag):
    ref = golden_run(tag)
    mol = molecule(tag)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    result = solve_rhf(ham, options=ScfOptions(energy_tolerance=1e-11, gradient_tolerance=1e-8))
    assert result.converged
    assert abs(result.energy - float(ref["energy"])) <= 1e-8
    assert np.max(np.abs(result.density.cpu().numpy() - ref["density"])) <= 1e-6


def test_sad_guess_matches_oracle():
    """atoms.py:76-120 restated on the device against the oracle's restatement."""
    from hafnium_b200.basis import ShellTable
    from hafnium_b200.scf import atomic_density_guess
    from oracle import dfrhf

    mol = molecule("h2o2_s0")
    orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
    expected = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    got = atomic_density_guess(mol, "cc-pvdz").cpu().numpy()
    np.testing.assert_allclose(got, expected, atol=1e-8, rtol=0)


@pytest.mark.parametrize("tag", ["h2o4_s1", "h2o8_s2", "h2o12_s3", "h2o16_s0", "h2o32_s0"])
def test_sad_started_scf_follows_the_reference_iterations(tag):
    """With the reference's SAD guess the device SCF takes the reference's iterations."""
    from hafnium_b200.scf import atomic_density_guess

    ref = golden_run(tag)
    mol = molecule(tag)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    result = solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"))
    assert result.n_iterations == int(ref["n_iterations"])
    np.testing.assert_allclose([h.energy for h in result.history], ref["history"], atol=1e-8, rtol=0)
    assert abs(result.energy - float(ref["energy"])) <= 1e-8


@pytest.mark.parametrize("tag", ["h2o4_s1", "h2o8_s2", "h2o12_s3", "h2o16_s0", "h2o32_s0"])
def test_mixed_schedule_matches_reference(tag):
    """Split-BF16 builds, an FP64 anchor, incremental builds on the exactly
    factored difference density, then the finishing build in FP64, whose orbital
    gradient decides convergence (the reference's default tolerances): the
    reference's converged FP64 energy and density, with two FP64 exchange builds."""
    from hafnium_b200.scf import PrecisionSchedule, atomic_density_guess

    ref = golden_run(tag)
    mol = molecule(tag)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    result = solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"), schedule=PrecisionSchedule(mode="mixed"))
    assert result.converged
    assert {"bf16", "incremental", "fp64"} <= {h.precision for h in result.history}
    assert result.timings["exchange_builds_fp64"] == 2  # the anchor and the finishing build
    assert result.timings["final_gradient"] < 1e-6
    assert abs(result.energy - float(ref["energy"])) <= 1e-8
    assert np.max(np.abs(result.density.cpu().numpy() - ref["density"])) <= 1e-6


def test_mixed_schedule_at_tight_tolerances():
    """At tolerances far below the defaults the incremental builds still reach the
    gradient (re-anchoring if the BF16 rounding of a far anchor stalls them) and
    the FP64 finish confirms it."""
    from hafnium_b200.scf import PrecisionSchedule, atomic_density_guess

    ref = golden_run("h2o8_s2")
    mol = molecule("h2o8_s2")
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    result = solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"),
                       options=ScfOptions(energy_tolerance=1e-11, gradient_tolerance=1e-8),
                       schedule=PrecisionSchedule(mode="mixed"))
    assert result.converged and result.timings["final_gradient"] < 1e-8
    assert result.timings["exchange_builds_fp64"] <= 4
    assert abs(result.energy - float(ref["energy"])) <= 1e-8
    assert np.max(np.abs(result.density.cpu().numpy() - ref["density"])) <= 1e-6


@pytest.mark.parametrize("tag,schedule", [("h2o4_s1", "mixed"), ("h2o8_s2", "mixed"), ("h2o16_s0", "mixed"),
                                          ("h2o8_s2", "mixed-host")])
def test_reference_driver_with_the_mixed_builder_matches_reference(tag, schedule):
    """The reference's SCF loop (restated by the oracle: it calls nothing but
    coulomb(2 D) and exchange(D), with host NumPy arrays, and tests convergence
    on two consecutive energies) over the drop-in with schedule="mixed": the
    builder alone chooses split-BF16, anchored incremental and FP64 builds from
    the densities it is given, and the result is the reference's."""
    from hafnium_b200.basis import ShellTable
    from hafnium_b200.jk import B200DensityFittedCoulombExchange
    from oracle import dfrhf

    ref = golden_run(tag)
    mol = molecule(tag)
    orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
    aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
    two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux, schedule=schedule)
    s = dfrhf.overlap(orb)
    h = dfrhf.core_hamiltonian(orb, mol.nuclear_charges, mol.positions)
    guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    result = dfrhf.solve_rhf(s, h, two_body, mol.nuclear_repulsion_energy(), mol.n_alpha, guess=guess)
    kinds = [entry["precision"] for entry in two_body.schedule.log]
    assert kinds[0] == "bf16" and "incremental" in kinds
    assert 1 <= kinds.count("anchor") <= 2
    assert abs(result.energy - float(ref["energy"])) <= 1e-8
    assert np.max(np.abs(result.density - ref["density"])) <= 1e-6


@pytest.mark.parametrize("tag", ["h2o12_s3", "h2o32_s0"])
def test_protocol_only_device_driver_matches_reference(tag):
    """The device driver in protocol mode (only coulomb(2 D) / exchange(D) on host
    NumPy arrays, the reference's convergence test) over the mixed builder."""
    from hafnium_b200.scf import atomic_density_guess

    ref = golden_run(tag)
    mol = molecule(tag)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit", exchange_schedule="mixed")
    result = solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"), protocol=True, host_io=True)
    assert result.converged
    kinds = [h.precision for h in result.history]
    assert kinds[0] == "bf16" and "incremental" in kinds and "anchor" in kinds
    assert result.timings["h2d_bytes"] > 0 and result.timings["d2h_bytes"] > 0
    assert abs(result.energy - float(ref["energy"])) <= 1e-8
    assert np.max(np.abs(result.density.cpu().numpy() - ref["density"])) <= 1e-6


def test_host_array_path_matches_the_device_path():
    """Every J and K through the drop-in's host NumPy entry points (what the
    reference's driver calls) gives the device path's converged energy."""
    from hafnium_b200.scf import PrecisionSchedule, atomic_density_guess

    mol = molecule("h2o4_s1")
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    guess = atomic_density_guess(mol, "cc-pvdz")
    device = solve_rhf(ham, guess=guess, schedule=PrecisionSchedule(mode="mixed"))
    host = solve_rhf(ham, guess=guess, schedule=PrecisionSchedule(mode="mixed"), host_io=True)
    assert abs(host.energy - device.energy) <= 1e-8
    assert host.timings["h2d_bytes"] > 0 and host.timings["d2h_bytes"] > 0


def test_mixed_schedule_matches_plain_fp64_at_an_odd_padding():
    """(H2O)12: n = 288, padded to 384 for the split-BF16 builds (an odd multiple of
    128). The mixed schedule reaches the plain FP64 path's energy and density."""
    from hafnium_b200.molecule import water_cluster
    from hafnium_b200.scf import PrecisionSchedule, atomic_density_guess

    mol = water_cluster(12, 3)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    guess = atomic_density_guess(mol, "cc-pvdz")
    options = ScfOptions(energy_tolerance=1e-11, gradient_tolerance=1e-8)
    plain = solve_rhf(ham, guess=guess, options=options)
    mixed = solve_rhf(ham, guess=guess, options=options, schedule=PrecisionSchedule(mode="mixed"))
    assert plain.converged and mixed.converged
    assert {"bf16", "incremental", "fp64"} <= {h.precision for h in mixed.history}
    assert abs(mixed.energy - plain.energy) <= 1e-8
    assert float((mixed.density - plain.density).abs().max()) <= 1e-6


def test_library_and_host_schedules_agree():
    """hf_exchange_scheduled (the schedule inside the library, for C hosts) and its
    host-side restatement take the same decisions on the densities of an SCF and
    give the same K to far below the split-BF16 error."""
    import torch

    from hafnium_b200 import _lib
    from hafnium_b200.basis import ShellTable
    from hafnium_b200.errors import InputError
    from hafnium_b200.jk import B200DensityFittedCoulombExchange
    from hafnium_b200.scf import atomic_density_guess

    mol = molecule("h2o8_s2")
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    seen = []

    class Recorder:
        """The drop-in's protocol, recording every density it is given."""

        def __init__(self, inner):
            self.inner, self.n_ao = inner, inner.n_ao

        def coulomb(self, d):
            return self.inner.coulomb(d)

        def exchange(self, d):
            seen.append(d.clone())
            return self.inner.exchange(d)

    ham.two_body = Recorder(ham.two_body)
    solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"), protocol=True)
    orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
    aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
    library = B200DensityFittedCoulombExchange.from_tables(orb, aux, schedule="mixed")
    host = B200DensityFittedCoulombExchange.from_tables(orb, aux, schedule="mixed-host")
    for d in seen:
        k_lib, k_host = library.exchange(d), host.exchange(d)
        assert float((k_lib - k_host).abs().max()) <= 1e-9 * float(k_host.abs().max())
    kinds = [e["precision"] for e in library.schedule.log]
    assert kinds == [e["precision"] for e in host.schedule.log]
    assert kinds[0] == "bf16" and "anchor" in kinds and "incremental" in kinds
    with pytest.raises(InputError, match="final_change"):
        library.context.exchange_scheduled(seen[0], torch.empty_like(seen[0]), _lib.ScheduleC(_lib.SCHEDULE_MIXED, 1e-5, 1e-3))


def test_scheduled_exchange_of_an_indefinite_density_is_fp64():
    """The protocol allows any symmetric density; one without a factor (never an
    SCF's) goes through the signed FP64 path, with every schedule."""
    from oracle import dfrhf
    from tests.helpers import tables

    mol = molecule("h2o2_s0")
    orb, aux = tables(mol)
    b = dfrhf.df_tensor(dfrhf.metric(aux), dfrhf.three_center(aux, orb))
    rng = np.random.default_rng(9)
    c = rng.normal(size=(orb.n_functions, 6))
    d = c[:, :3] @ c[:, :3].T - c[:, 3:] @ c[:, 3:].T
    from hafnium_b200.jk import B200DensityFittedCoulombExchange

    for schedule in ("fp64", "mixed", "mixed-host"):
        two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux, schedule=schedule)
        np.testing.assert_allclose(two_body.exchange(d), dfrhf.exchange(b, d), atol=1e-10, rtol=0)
