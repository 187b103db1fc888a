"""The learned guess's host pieces (CPU): the oracle's gradients, frame invariance,
block round trips."""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.learned import model as M
from hafnium_b200.learned.frames import ao_rotation, harmonic_rotation, solid_harmonics
from hafnium_b200.molecule import Molecule, water_cluster
from oracle import mpnn


def small_graph(rng, n=4, width=8, edge=5):
    src = np.array([0, 0, 1, 2, 3, 1], dtype=np.int32)
    dst = np.array([1, 2, 0, 3, 2, 3], dtype=np.int32)
    return {"src": src, "dst": dst, "edge": rng.normal(size=(6, edge)), "fcut": rng.uniform(0.2, 1, 6), "n_nodes": n}


def small_params(rng, width=8, edge=5, layers=2, nd=3, no=2):
    p = {"h0": rng.normal(size=width) * 0.5}
    for l in range(layers):
        p[f"Wm{l}"] = rng.normal(size=(2 * width + edge, width)) * 0.3
        p[f"bm{l}"] = rng.normal(size=width) * 0.1
        p[f"Wu{l}"] = rng.normal(size=(2 * width, width)) * 0.3
        p[f"bu{l}"] = rng.normal(size=width) * 0.1
    p["Wd"], p["bd"] = rng.normal(size=(width, nd)) * 0.3, rng.normal(size=nd) * 0.1
    p["We"], p["be"] = rng.normal(size=(2 * width + edge, width)) * 0.3, rng.normal(size=width) * 0.1
    p["Wo"], p["bo"] = rng.normal(size=(width, no)) * 0.3, rng.normal(size=no) * 0.1
    return p


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    g = small_graph(rng)
    p = small_params(rng)
    t = {"d": rng.normal(size=(4, 3)), "o": rng.normal(size=(6, 2))}
    _, grads = mpnn.loss_and_grad(p, g, t, 2, 0.7)
    worst = 0.0
    for k, v in p.items():
        flat = v.reshape(-1)
        for idx in range(0, flat.size, max(1, flat.size // 4)):
            old = flat[idx]
            flat[idx] = old + 1e-6
            lp, _ = mpnn.loss_and_grad(p, g, t, 2, 0.7)
            flat[idx] = old - 1e-6
            lm, _ = mpnn.loss_and_grad(p, g, t, 2, 0.7)
            flat[idx] = old
            fd = (lp - lm) / 2e-6
            worst = max(worst, abs(fd - grads[k].reshape(-1)[idx]) / max(1.0, abs(fd)))
    assert worst < 1e-6


def test_rotations_are_orthogonal_and_p_is_the_frame():
    rng = np.random.default_rng(1)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    q[:, 0] *= np.sign(np.linalg.det(q))
    for l in range(3):
        u = harmonic_rotation(q, l)
        np.testing.assert_allclose(u.T @ u, np.eye(2 * l + 1), atol=1e-12)
    np.testing.assert_allclose(harmonic_rotation(q, 1), q, atol=1e-12)
    assert solid_harmonics(2).shape == (5, 6)


def rotate(mol, r, shift):
    return Molecule(mol.symbols, mol.positions @ r.T + shift)


def test_edge_features_are_invariant_under_rigid_motions():
    mol = water_cluster(6, 3)
    rng = np.random.default_rng(2)
    r, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    r[:, 0] *= np.sign(np.linalg.det(r))
    g1 = M.build_graph(mol)
    g2 = M.build_graph(rotate(mol, r, np.array([1.0, -2.0, 0.5])))
    np.testing.assert_array_equal(g1["src"], g2["src"])
    np.testing.assert_allclose(g1["edge"], g2["edge"], atol=1e-12)


def test_local_blocks_round_trip_to_the_density():
    """Blocks within the cutoff map back to the global density unchanged."""
    mol = water_cluster(5, 4)
    g = M.build_graph(mol)
    n = 24 * g["n_nodes"]
    rng = np.random.default_rng(3)
    a = rng.normal(size=(n, n))
    dens = a + a.T
    # zero the blocks between waters beyond the cutoff: the network never predicts them
    keep = np.zeros((g["n_nodes"], g["n_nodes"]), dtype=bool)
    np.fill_diagonal(keep, True)
    keep[g["src"], g["dst"]] = True
    mask = np.kron(keep, np.ones((24, 24), dtype=bool))
    dens = np.where(mask, dens, 0.0)
    t = M.local_targets(g, dens)
    back = M.blocks_to_density(g, t["d"], t["o"], np.zeros(M.DIAG))
    np.testing.assert_allclose(back, dens, atol=1e-12)


def test_weights_checksum_detects_corruption(tmp_path):
    params = {k: v.astype(np.float32) for k, v in small_params(np.random.default_rng(4)).items()}
    path = tmp_path / "w.npz"
    M.save_weights(path, params, np.zeros(3), {"note": "test"})
    assert M.load_weights(path) is not None
    with np.load(path) as z:
        arrays = {k: z[k] for k in z.files}
    arrays["Wd"] = arrays["Wd"] + 1.0
    np.savez_compressed(path, **arrays)
    assert M.load_weights(path) is None


def test_non_water_molecules_fall_back():
    mol = Molecule(("N", "H", "H", "H"), np.zeros((4, 3)) + np.arange(4)[:, None])
    assert not M.is_water_cluster(mol)
    assert M.predict_density(mol) is None
