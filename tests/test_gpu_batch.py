"""Batched DF-RHF (include/hfbatch.h) against the oracle and the per-cluster path (B200).

Mirrors the reference's SCF checks (tests/reference/test_mp2_reference.py:37-60,
tests/unit/test_scf_driver.py): the converged energy of every cluster matches
the oracle's restatement of the reference driver to 1e-8 Eh, with the same
number of Fock builds in the loop (len(history)) up to one.
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.molecule import water_cluster
from oracle import dfrhf
from tests.helpers import tables

pytestmark = pytest.mark.gpu
ENERGY_TOL = 1e-8
JK_TOL = 1e-11


def _oracle(mol):
    orb, aux = tables(mol)
    prob = dfrhf.build_problem(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                               mol.n_alpha)
    guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    return dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, mol.n_alpha, guess=guess)


@pytest.fixture(scope="module")
def small_clusters():
    mols = [water_cluster(2, 0), water_cluster(2, 5), water_cluster(3, 1), water_cluster(2, 9), water_cluster(3, 4)]
    return mols, [_oracle(m) for m in mols]


@pytest.mark.parametrize("tile", range(6))
def test_dgemm_tiles_match_torch(tile):
    import torch

    from hafnium_b200.batch import dgemm_nt

    gen = torch.Generator(device="cuda").manual_seed(tile)
    for m, n, k in ((96, 80, 72), (200, 136, 48), (17, 33, 9)):
        a = torch.rand((3, m, k), dtype=torch.float64, device="cuda", generator=gen)
        b = torch.rand((3, n, k), dtype=torch.float64, device="cuda", generator=gen)
        c = torch.rand((3, m, n), dtype=torch.float64, device="cuda", generator=gen)
        want = 0.5 * a @ b.transpose(1, 2) - 2.0 * c
        dgemm_nt(a, b, c, alpha=0.5, beta=-2.0, tile=tile)
        torch.testing.assert_close(c, want, rtol=0, atol=1e-12)


def test_batched_coulomb_and_exchange_match_single_cluster():
    import torch

    from hafnium_b200 import _lib
    from hafnium_b200.batch import Batch, _cluster

    mols = [water_cluster(2, 0), water_cluster(2, 5), water_cluster(2, 9)]
    clusters = [_cluster(m, "cc-pvdz", "def2-universal-jkfit", 0) for m in mols]
    batch = Batch([c[0] for c in clusters], 10)
    n = batch.n
    rng = np.random.default_rng(3)
    factors = [rng.normal(size=(n, 10)) / np.sqrt(n) for _ in mols]
    d = torch.as_tensor(np.stack([f @ f.T for f in factors]), device="cuda").contiguous()
    j = batch.coulomb(d, 2.0).cpu().numpy()
    k = batch.exchange(d, 10).cpu().numpy()
    for c, (ctx, _, _) in enumerate(clusters):
        dc = d[c].cpu().numpy()
        np.testing.assert_allclose(j[c], ctx.coulomb_host(2.0 * dc), atol=JK_TOL, rtol=0)
        np.testing.assert_allclose(k[c], ctx.exchange_host(dc, _lib.PREC_FP64), atol=JK_TOL, rtol=0)
    batch.close()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_scf_matches_oracle(small_clusters, use_graph):
    from hafnium_b200.batch import BatchOptions, solve_batch

    mols, refs = small_clusters
    result = solve_batch(mols, options=BatchOptions(use_graph=use_graph))
    assert all(s == "converged" for s in result.states), result.states
    for e, it, ref in zip(result.energies, result.iterations, refs):
        assert abs(e - ref.energy) < ENERGY_TOL, (e, ref.energy)
        assert abs(int(it) - len(ref.history)) <= 1, (int(it), len(ref.history))


def test_batched_density_matches_oracle():
    import torch

    from hafnium_b200.batch import Batch, BatchOptions, _Atoms, _cluster

    mols = [water_cluster(2, 0), water_cluster(2, 5)]
    refs = [_oracle(m) for m in mols]
    clusters = [_cluster(m, "cc-pvdz", "def2-universal-jkfit", 0) for m in mols]
    atoms = _Atoms("cc-pvdz", 0)
    batch = Batch([c[0] for c in clusters], mols[0].n_alpha)
    s = torch.stack([c[1] for c in clusters]).contiguous()
    h = torch.stack([c[2] for c in clusters]).contiguous()
    guess = torch.stack([atoms.guess(m) for m in mols]).contiguous()
    batch.load(s, h, guess, [m.nuclear_repulsion_energy() for m in mols], max(atoms.rank(m) for m in mols))
    batch.run(BatchOptions(), 0)
    dens = torch.empty_like(s)
    energies, _, states = batch.results(dens)
    for c, ref in enumerate(refs):
        assert states[c] == "converged"
        assert abs(energies[c] - ref.energy) < ENERGY_TOL
        np.testing.assert_allclose(dens[c].cpu().numpy(), ref.density, atol=1e-6, rtol=0)
    batch.close()


def test_iteration_limit_reports_not_converged():
    from hafnium_b200.batch import BatchOptions, solve_batch

    result = solve_batch([water_cluster(2, 0)], options=BatchOptions(max_iterations=3))
    assert result.states == ["not_converged"]
    assert int(result.iterations[0]) == 3


def test_tile_tuner_picks_a_timed_shape(tmp_path):
    from hafnium_b200.batch import TILE_SHAPES, TileTuner

    tuner = TileTuner(str(tmp_path / "tiles.json"), repeats=2)
    tile = tuner.choose(96, 4)
    assert 0 <= tile < len(TILE_SHAPES)
    again = TileTuner(str(tmp_path / "tiles.json"))
    assert again.choose(96, 4) == tile
