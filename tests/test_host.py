"""Host-side logic: the cluster generator, shell tables and the driver's host pieces (CPU)."""

from __future__ import annotations

import itertools

import numpy as np
import pytest

from hafnium_b200.basis import ShellTable, element_shells, primitive_norm
from hafnium_b200.molecule import ANGSTROM_IN_BOHR, cube_side_angstrom, water_cluster
from hafnium_b200.scf import fill_averaged, solve_diis
from oracle import dfrhf


@pytest.mark.parametrize("n,seed", [(8, 0), (32, 3), (64, 0)])
def test_water_cluster_geometry(n, seed):
    mol = water_cluster(n, seed)
    assert mol.symbols == ("O", "H", "H") * n
    pos = mol.positions / ANGSTROM_IN_BOHR
    oxygens = pos[0::3]
    for i, j in itertools.combinations(range(n), 2):
        assert np.linalg.norm(oxygens[i] - oxygens[j]) >= 2.7 - 1e-12
    side = cube_side_angstrom(n)
    assert np.all(oxygens >= 0.0) and np.all(oxygens <= side)
    for w in range(n):
        o, h1, h2 = pos[3 * w: 3 * w + 3]
        assert np.linalg.norm(h1 - o) == pytest.approx(0.9572, abs=1e-12)
        cos = np.dot(h1 - o, h2 - o) / 0.9572 ** 2
        assert np.degrees(np.arccos(cos)) == pytest.approx(104.52, abs=1e-9)
    assert mol.n_alpha == 5 * n


def test_cluster_sizes_match_the_configs():
    for n, nbf, naux in ((8, 192, 904), (32, 768, 3616), (64, 1536, 7232)):
        mol = water_cluster(n, 0)
        orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
        aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
        assert (orb.n_functions, aux.n_functions) == (nbf, naux)


def test_contractions_have_unit_norm():
    """<chi|chi> = 1 for every contracted spherical function (shell.py:87-104)."""
    for shells in element_shells("cc-pvdz").values():
        for shell in shells:
            for row in shell.primitive_coefficients():
                total = 0.0
                for ci, ai in zip(row, shell.exponents):
                    for cj, aj in zip(row, shell.exponents):
                        ni, nj = primitive_norm(ai, shell.l), primitive_norm(aj, shell.l)
                        total += ci * cj / (ni * nj) * (2 * np.sqrt(ai * aj) / (ai + aj)) ** (shell.l + 1.5)
                assert total == pytest.approx(1.0, abs=1e-12)


@pytest.mark.parametrize("basis", ["cc-pvdz", "def2-universal-jkfit", "sto-3g", "def2-svp"])
def test_shell_table_lays_out_each_atom_shell_by_shell(basis):
    """ShellTable.build (each element's block computed once) equals the table laid out
    shell by shell and atom by atom, as shell_table.py:84-116 does, for molecules of
    several elements; an element the basis lacks is refused."""
    from hafnium_b200.errors import InputError
    from hafnium_b200.molecule import Molecule, atomic_number

    rng = np.random.default_rng(5)
    mols = [water_cluster(3, 1), Molecule(("N", "H", "H", "H", "C", "O"), rng.normal(size=(6, 3)) * 2.0)]
    for mol in mols:
        ls, centers, offsets, exps, coefs, ks, atoms = [], [], [0], [], [], [], []
        for index, symbol in enumerate(mol.symbols):
            for shell in element_shells(basis)[atomic_number(symbol)]:
                rows = shell.primitive_coefficients()
                ls.append(shell.l)
                centers.append(mol.positions[index])
                exps.extend(shell.exponents)
                offsets.append(len(exps))
                for row in rows:
                    coefs.extend(row)
                ks.append(len(rows))
                atoms.append(index)
        t = ShellTable.build(basis, mol.symbols, mol.positions)
        np.testing.assert_array_equal(t.angular_momenta, ls)
        np.testing.assert_array_equal(t.centers, np.asarray(centers).reshape(-1, 3))
        np.testing.assert_array_equal(t.primitive_offsets, offsets)
        np.testing.assert_array_equal(t.exponents, exps)
        np.testing.assert_array_equal(t.coefficients, coefs)
        np.testing.assert_array_equal(t.n_contractions, ks)
        np.testing.assert_array_equal(t.shell_atoms, atoms)
    with pytest.raises(InputError):
        ShellTable.build(basis, ("O", "Xe"), np.zeros((2, 3)))


def test_diis_and_filling_match_the_oracle():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(5, 5))
    ov = a @ a.T
    np.testing.assert_allclose(solve_diis(ov), dfrhf.solve_diis(ov), atol=1e-14)
    e = np.array([-3.0, -1.0, 0.5, 0.5 + 1e-9, 0.5 - 1e-9, 2.0])
    np.testing.assert_allclose(fill_averaged(e, 3.0), dfrhf.fill_averaged(e, 3.0), atol=0)


def test_purification_gives_the_aufbau_projector():
    """scf.purify on the CPU: the projector onto the n_occ lowest eigenvectors."""
    import torch

    from hafnium_b200.scf import purify

    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(rng.normal(size=(60, 60)))
    levels = np.concatenate([np.sort(rng.uniform(-20.0, -0.4, 17)), np.sort(rng.uniform(0.2, 5.0, 43))])
    fo = (q * levels) @ q.T
    p, ok = purify(torch.as_tensor(fo), 17)
    assert ok
    expected = q[:, :17] @ q[:, :17].T
    np.testing.assert_allclose(p.numpy(), expected, atol=1e-11, rtol=0)


def test_purification_reports_a_missing_gap():
    import torch

    from hafnium_b200.scf import purify

    fo = np.diag(np.concatenate([np.full(3, -1.0), np.full(3, 0.5)]))
    fo[2, 2] = fo[3, 3] = 0.0  # degenerate HOMO/LUMO: no projector of rank 3 is singled out
    p, ok = purify(torch.as_tensor(fo), 3)
    assert not ok or abs(float(torch.trace(p)) - 3.0) < 1e-8


def test_occupied_factor_reproduces_an_idempotent_density():
    """hafnium_b200.gradient.occupied_factor: C C^T = D for D S D = D (the form in
    which the reference's ScfResult gives a state), and the five gradient terms
    add up to NuclearGradient.total."""
    from hafnium_b200.gradient import NuclearGradient, occupied_factor

    rng = np.random.default_rng(5)
    n, k = 12, 4
    a = rng.normal(size=(n, n))
    s = a @ a.T / n + np.eye(n)
    w, v = np.linalg.eigh(s)
    inv_half = (v / np.sqrt(w)) @ v.T
    q, _ = np.linalg.qr(rng.normal(size=(n, k)))
    c = inv_half @ q  # orthonormal in the S metric
    d = c @ c.T
    np.testing.assert_allclose(d @ s @ d, d, atol=1e-12)
    got = occupied_factor(d, s, k)
    np.testing.assert_allclose(got @ got.T, d, atol=1e-12)
    terms = [rng.normal(size=(3, 3)) for _ in range(5)]
    np.testing.assert_allclose(NuclearGradient(*terms).total, sum(terms), atol=0)
