"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run where the reference tree is mounted (it does not exist on the GPU hosts):

    python tests/golden/make_golden.py [/path/to/reference]

Two kinds of fixture are written:

* ``pyscf_*.npz``: the PySCF/libcint values the reference stores in
  tests/reference/data/*.json (metric and three-centre integrals of water in
  STO-3G / def2-universal-jkfit; S, T, V of water in cc-pVDZ), converted to
  NumPy arrays unchanged, with the reference's stored DF-RHF and exact RHF
  energies of water/STO-3G.
* ``reference_dfrhf_*.npz``: the reference's own DF-RHF (``hartree_fock`` with
  its SAD guess, DIIS 8, default tolerances; hafnium/scf/hartree_fock.py:24)
  run unchanged on seeded water clusters in cc-pVDZ / def2-universal-jkfit,
  its integrals supplied by the oracle's C++ restatement of the Rust kernels:
  geometry, total energy, alpha density, iteration energies. The same script
  checks the oracle's NumPy restatement (oracle/dfrhf.py) against each run.
* ``reference_gradient_*.npz``: the reference's own DF-RHF nuclear gradient at
  its converged state, with the state itself (see ``reference_gradients``).
* ``reference_dfrhf_h2o12_s3.npz``, ``reference_dfrhf_h2o16_s0.npz``: the
  reference's own DF-RHF as above on larger clusters (n = 288, 384), stored as
  an occupied factor F of the density (D = F F^T) to keep the files small; the
  oracle's memory-lean restatement (``LeanFittedJK``) is checked against each.
* ``oracle_dfrhf_h2o32_s0.npz``: (H2O)32 (n = 768), beyond what the reference's
  full-layout exchange runs in this container's memory in reasonable time, from
  the lean restatement that the two runs above pin (see ``large_runs``).

The reference tree is given as the first argument or by HF_REFERENCE_ROOT.
"""

from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

CLUSTERS = [(1, None), (2, 0), (4, 1), (8, 2)]  # (waters, seed); one water = the reference's water()


def molecule_for(n, seed):
    from hafnium_b200.molecule import water, water_cluster

    return water() if seed is None else water_cluster(n, seed)


def stored_pyscf(reference: pathlib.Path) -> None:
    data = reference / "tests" / "reference" / "data"
    df = json.loads((data / "density_fitting_water_sto-3g.json").read_text())
    one = json.loads((data / "one_electron_water_cc-pvdz.json").read_text())
    mp2 = json.loads((data / "mp2_water_sto-3g.json").read_text())
    scf = json.loads((data / "scf_water_sto-3g.json").read_text())
    np.savez_compressed(
        HERE / "pyscf_water.npz",
        df_positions_bohr=np.asarray(df["provenance"]["positions_bohr"]),
        df_metric=np.asarray(df["metric"]),
        df_three_center=np.asarray(df["three_center"]),
        one_positions_bohr=np.asarray(one["provenance"].get("positions_bohr", df["provenance"]["positions_bohr"])),
        one_overlap=np.asarray(one["overlap"]),
        one_kinetic=np.asarray(one["kinetic"]),
        one_nuclear=np.asarray(one["nuclear_attraction"]),
        dfrhf_energy_sto3g=np.asarray(mp2["reference_energy"]),
        dfmp2_correlation_sto3g=np.asarray(mp2["correlation_energy"]),
        rhf_energy_sto3g=np.asarray(scf["energy"] if "energy" in scf else scf["total_energy"]),
    )


def reference_runs(reference: pathlib.Path) -> None:
    from oracle import reference_env

    reference_env.install(reference)
    from hafnium.basis import BasisLibrary, BasisSet
    from hafnium.integrals import RustEngine
    from hafnium.molecule import Molecule as RefMolecule
    from hafnium.scf import hartree_fock

    from hafnium_b200.basis import ShellTable
    from oracle import dfrhf

    library = BasisLibrary(offline=True)
    engine = RustEngine()
    for n, seed in CLUSTERS:
        mol = molecule_for(n, seed)
        ref_mol = RefMolecule.from_atoms(list(zip(mol.symbols, map(tuple, mol.positions))), unit="bohr")
        basis = BasisSet.for_atoms(ref_mol, "cc-pvdz", library=library)
        aux = BasisSet.for_atoms(ref_mol, "def2-universal-jkfit", library=library)
        result = hartree_fock(engine, basis, ref_mol, auxiliary=aux)
        d_ref = np.asarray(result.density.blocks[0])
        hist = np.asarray([row.energy for row in result.history])
        # The oracle restatement on the same input.
        orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
        auxt = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
        prob = dfrhf.build_problem(orb, auxt, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                                   mol.n_alpha)
        guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
        ours = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, prob.n_alpha, guess=guess)
        de = abs(ours.energy - result.energy)
        dd = float(np.max(np.abs(ours.density - d_ref)))
        print(f"(H2O){n} seed {seed}: reference E = {result.energy:.12f} in {result.n_iterations} iterations; "
              f"oracle |dE| = {de:.2e}, max|dD| = {dd:.2e}, iterations {ours.n_iterations}; "
              f"metric eigenvalues dropped: {prob.dropped}")
        assert de < 1e-10 and dd < 1e-7 and ours.n_iterations == result.n_iterations
        tag = "water" if seed is None else f"h2o{n}_s{seed}"
        np.savez_compressed(
            HERE / f"reference_dfrhf_{tag}.npz",
            n_waters=np.asarray(n),
            seed=np.asarray(-1 if seed is None else seed),
            positions_bohr=mol.positions,
            energy=np.asarray(result.energy),
            density=d_ref,
            history=hist,
            n_iterations=np.asarray(result.n_iterations),
        )


LARGE_REFERENCE = [(12, 3), (16, 0)]  # n = 288 (pads to 384, an odd multiple of 128) and 384
LARGE_ORACLE = [(32, 0)]  # n = 768: the split-precision workload's size


def _save_large(path: pathlib.Path, n, seed, mol, energy, density, history, n_iterations, source: str) -> None:
    from oracle import dfrhf

    factor = dfrhf.psd_factor(density)
    assert factor.shape[1] == mol.n_alpha, factor.shape
    assert float(np.max(np.abs(factor @ factor.T - density))) < 1e-13
    np.savez_compressed(
        path,
        n_waters=np.asarray(n),
        seed=np.asarray(seed),
        positions_bohr=mol.positions,
        energy=np.asarray(energy),
        density_factor=factor,
        history=np.asarray(history),
        n_iterations=np.asarray(n_iterations),
        source=np.asarray(source),
    )


def large_runs(reference: pathlib.Path) -> None:
    """The reference's own ``hartree_fock`` on (H2O)12 and (H2O)16, and the oracle's
    lean restatement (in-place fit, exchange through an occupied factor) checked
    against both to |dE| < 1e-10, max|dD| < 1e-7 and the same iteration count; then
    the lean restatement alone on (H2O)32."""
    import time

    from oracle import reference_env

    reference_env.install(reference)
    from hafnium.basis import BasisLibrary, BasisSet
    from hafnium.integrals import RustEngine
    from hafnium.molecule import Molecule as RefMolecule
    from hafnium.scf import hartree_fock

    from hafnium_b200.basis import ShellTable
    from oracle import dfrhf

    library = BasisLibrary(offline=True)
    engine = RustEngine()

    def lean(mol):
        orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
        auxt = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
        prob = dfrhf.build_problem_lean(orb, auxt, mol.nuclear_charges, mol.positions,
                                        mol.nuclear_repulsion_energy(), mol.n_alpha)
        guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
        return dfrhf.solve_rhf(prob.s, prob.h, dfrhf.LeanFittedJK(prob.b), prob.e_nuc, prob.n_alpha,
                               guess=guess), prob.dropped

    for n, seed in LARGE_REFERENCE:
        mol = molecule_for(n, seed)
        t0 = time.perf_counter()
        ref_mol = RefMolecule.from_atoms(list(zip(mol.symbols, map(tuple, mol.positions))), unit="bohr")
        basis = BasisSet.for_atoms(ref_mol, "cc-pvdz", library=library)
        aux = BasisSet.for_atoms(ref_mol, "def2-universal-jkfit", library=library)
        result = hartree_fock(engine, basis, ref_mol, auxiliary=aux)
        t1 = time.perf_counter()
        d_ref = np.asarray(result.density.blocks[0])
        hist = [row.energy for row in result.history]
        ours, dropped = lean(mol)
        t2 = time.perf_counter()
        de = abs(ours.energy - result.energy)
        dd = float(np.max(np.abs(ours.density - d_ref)))
        print(f"(H2O){n} seed {seed}: reference E = {result.energy:.12f} in {result.n_iterations} iterations "
              f"({t1 - t0:.0f} s); lean oracle |dE| = {de:.2e}, max|dD| = {dd:.2e}, iterations "
              f"{ours.n_iterations} ({t2 - t1:.0f} s); metric eigenvalues dropped: {dropped}", flush=True)
        assert de < 1e-10 and dd < 1e-7 and ours.n_iterations == result.n_iterations
        _save_large(HERE / f"reference_dfrhf_h2o{n}_s{seed}.npz", n, seed, mol, result.energy, d_ref, hist,
                    result.n_iterations, "reference hartree_fock (hafnium/scf/hartree_fock.py:24)")
    for n, seed in LARGE_ORACLE:
        mol = molecule_for(n, seed)
        t0 = time.perf_counter()
        ours, dropped = lean(mol)
        print(f"(H2O){n} seed {seed}: lean oracle E = {ours.energy:.12f} in {ours.n_iterations} iterations "
              f"({time.perf_counter() - t0:.0f} s); metric eigenvalues dropped: {dropped}", flush=True)
        assert ours.converged
        _save_large(HERE / f"oracle_dfrhf_h2o{n}_s{seed}.npz", n, seed, mol, ours.energy, ours.density,
                    [row.energy for row in ours.history], ours.n_iterations,
                    "oracle restatement (oracle/dfrhf.py LeanFittedJK), pinned by the (H2O)12/16 reference runs")


GRADIENT_CASES = [("water_pyscf", "def2-svp"), ("water", "cc-pvdz"), ("h2o2_s0", "cc-pvdz"), ("h2o4_s1", "cc-pvdz")]


def reference_gradients(reference: pathlib.Path) -> None:
    """``reference_gradient_*.npz``: the reference's own DF-RHF nuclear gradient
    (``hafnium.properties.nuclear_gradient``, gradient.py:72-149) at its tightly
    converged state (the options of tests/reference/test_gradient_reference.py:38),
    with the oracle restatement checked against it term by term, and the
    water/def2-SVP run checked against the PySCF gradient the reference stores
    (tests/reference/data/gradient_water_def2-svp.json) at its GRADIENT_TOL 1e-7."""
    from oracle import reference_env

    reference_env.install(reference)
    from hafnium.basis import BasisLibrary, BasisSet
    from hafnium.integrals import RustEngine
    from hafnium.molecule import Molecule as RefMolecule
    from hafnium.properties import nuclear_gradient
    from hafnium.scf import ScfOptions, hartree_fock

    from hafnium_b200.basis import ShellTable
    from hafnium_b200.molecule import Molecule
    from oracle import dfrhf

    library = BasisLibrary(offline=True)
    engine = RustEngine()
    options = ScfOptions(gradient_tolerance=1e-10, energy_tolerance=1e-13, max_iterations=200)
    stored = json.loads((reference / "tests" / "reference" / "data" / "gradient_water_def2-svp.json").read_text())
    for tag, basis_name in GRADIENT_CASES:
        if tag == "water_pyscf":
            mol = Molecule(("O", "H", "H"), np.asarray(stored["provenance"]["positions_bohr"], dtype=np.float64))
        else:
            n, seed = {"water": (1, None), "h2o2_s0": (2, 0), "h2o4_s1": (4, 1)}[tag]
            mol = molecule_for(n, seed)
        ref_mol = RefMolecule.from_atoms(list(zip(mol.symbols, map(tuple, mol.positions))), unit="bohr")
        basis = BasisSet.for_atoms(ref_mol, basis_name, library=library)
        aux = BasisSet.for_atoms(ref_mol, "def2-universal-jkfit", library=library)
        result = hartree_fock(engine, basis, ref_mol, auxiliary=aux, options=options)
        grad = nuclear_gradient(engine, basis, aux, ref_mol, result)
        terms = {k: np.asarray(getattr(grad, k)) for k in
                 ("nuclear_repulsion", "one_electron", "overlap", "coulomb", "exchange")}
        total = np.asarray(grad.total)
        d_alpha = np.asarray(result.density.blocks[0])
        fock = np.asarray(result.fock.blocks[0])
        orb = ShellTable.build(basis_name, mol.symbols, mol.positions)
        auxt = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
        ours = dfrhf.nuclear_gradient(orb, auxt, mol.nuclear_charges, mol.positions, d_alpha, fock)
        worst = max(float(np.max(np.abs(ours[k] - terms[k]))) for k in terms)
        msg = f"{tag}/{basis_name}: E = {result.energy:.12f}, oracle vs reference max |dG| = {worst:.2e}"
        if tag == "water_pyscf":
            dp = float(np.max(np.abs(total - np.asarray(stored["gradient"]))))
            msg += f", reference vs stored PySCF max |dG| = {dp:.2e}"
            assert dp < 1e-7
        print(msg)
        assert worst < 1e-10
        np.savez_compressed(
            HERE / f"reference_gradient_{tag}.npz",
            basis=np.asarray(basis_name),
            symbols=np.asarray(mol.symbols),
            positions_bohr=mol.positions,
            energy=np.asarray(result.energy),
            density=d_alpha,
            fock=fock,
            total=total,
            pyscf_total=np.asarray(stored["gradient"]) if tag == "water_pyscf" else np.zeros((0, 3)),
            **terms,
        )


def reference_root() -> pathlib.Path:
    import os

    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("HF_REFERENCE_ROOT")
    if not root:
        raise SystemExit("give the reference tree as the first argument or in HF_REFERENCE_ROOT")
    return pathlib.Path(root)


if __name__ == "__main__":
    ref = reference_root()
    if "--large" in sys.argv:
        large_runs(ref)
    else:
        stored_pyscf(ref)
        reference_runs(ref)
        reference_gradients(ref)
