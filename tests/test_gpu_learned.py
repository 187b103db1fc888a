"""The learned guess's device kernels against the NumPy oracle, and what the
trained network gains over the SAD guess (B200)."""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.learned import model as M
from oracle import mpnn
from tests.test_learned import small_graph, small_params

pytestmark = pytest.mark.gpu


def test_device_forward_and_backward_match_the_oracle():
    import torch

    rng = np.random.default_rng(0)
    width, edge = 16, M.EDGE_FEATURES
    g = small_graph(rng, width=width, edge=edge)
    p = small_params(rng, width=width, edge=edge, layers=3, nd=7, no=5)
    t = {"d": rng.normal(size=(4, 7)), "o": rng.normal(size=(6, 5))}
    loss_ref, grads_ref = mpnn.loss_and_grad(p, g, t, 3, 1.0)
    net = M.DeviceNet({k: v.astype(np.float32) for k, v in p.items()}, layers=3)
    gd = net.upload_graph(g)
    td = {k: torch.as_tensor(v, dtype=torch.float32, device=net.dev) for k, v in t.items()}
    loss, grads = net.loss_and_grad(gd, td)
    assert float(loss.item()) == pytest.approx(loss_ref, rel=1e-4)
    for k, ref in grads_ref.items():
        got = grads[k].cpu().numpy().reshape(ref.shape)
        scale = max(1.0, float(np.max(np.abs(ref))))
        assert np.max(np.abs(got - ref)) <= 1e-4 * scale, k


def test_trained_network_beats_the_sad_guess():
    """Held-out (H2O)16: fewer SCF iterations from the learned guess, same energy."""
    from hafnium_b200.molecule import water_cluster
    from hafnium_b200.scf import DeviceHamiltonian, atomic_density_guess, learned_density_guess, solve_rhf

    weights = M.load_weights()
    if weights is None:
        pytest.skip("no trained weights shipped")
    mol = water_cluster(16, 90210)
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    r_sad = solve_rhf(ham, guess=atomic_density_guess(mol, "cc-pvdz"))
    r_ml = solve_rhf(ham, guess=learned_density_guess(mol, ham, weights=weights))
    assert abs(r_ml.energy - r_sad.energy) <= 1e-8
    assert r_ml.n_iterations < r_sad.n_iterations


def test_device_assembly_matches_the_host_blocks():
    """The predicted blocks become the same global density on the device as on the host."""
    import torch

    from hafnium_b200.molecule import water_cluster

    g = M.build_graph(water_cluster(6, 11))
    rng = np.random.default_rng(8)
    d = rng.normal(size=(g["n_nodes"], M.DIAG))
    o = rng.normal(size=(len(g["src"]), M.OFF))
    mean = rng.normal(size=(len(M.ELEMENTS), M.DIAG))
    want = M.blocks_to_density(g, d, o, mean)
    dev = torch.device("cuda", 0)
    got = M.assemble_density(g, torch.as_tensor(d, device=dev), torch.as_tensor(o, device=dev), mean, dev)
    np.testing.assert_allclose(got.cpu().numpy(), want, atol=1e-13)
