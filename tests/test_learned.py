"""The learned guess's host pieces (CPU): the oracle's gradients, atom frames and
the invariance of what the network sees and predicts, block round trips."""

from __future__ import annotations

import numpy as np

from hafnium_b200.learned import model as M
from hafnium_b200.learned.frames import ao_rotation, atom_frames, harmonic_rotation, shell_layout, solid_harmonics
from hafnium_b200.molecule import Molecule, water_cluster
from oracle import mpnn


def small_graph(rng, n=4, width=8, edge=5):
    src = np.array([0, 0, 1, 2, 3, 1], dtype=np.int32)
    dst = np.array([1, 2, 0, 3, 2, 3], dtype=np.int32)
    return {"src": src, "dst": dst, "edge": rng.normal(size=(6, edge)), "fcut": rng.uniform(0.2, 1, 6), "n_nodes": n,
            "elem": np.array([7, 0, 0, 5], dtype=np.int32)}


def small_params(rng, width=8, edge=5, layers=2, nd=3, no=2):
    p = {"h0": rng.normal(size=(len(M.ELEMENTS), width)) * 0.5}
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
    # the embedding rows of elements absent from the graph get no gradient
    absent = [e for e in range(len(M.ELEMENTS)) if e not in set(g["elem"].tolist())]
    assert np.all(grads["h0"][absent] == 0.0)


def random_rotation(rng):
    r, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    r[:, 0] *= np.sign(np.linalg.det(r))
    return r


def test_rotations_are_orthogonal_compose_and_p_is_the_frame():
    rng = np.random.default_rng(1)
    q, f = random_rotation(rng), random_rotation(rng)
    for l in range(3):
        u = harmonic_rotation(q, l)
        np.testing.assert_allclose(u.T @ u, np.eye(2 * l + 1), atol=1e-12)
        np.testing.assert_allclose(harmonic_rotation(q @ f, l), u @ harmonic_rotation(f, l), atol=1e-12)
    np.testing.assert_allclose(harmonic_rotation(q, 1), q, atol=1e-12)
    assert solid_harmonics(2).shape == (5, 6)


def rotate(mol, r, shift):
    return Molecule(mol.symbols, mol.positions @ r.T + shift)


def test_atom_frames_follow_the_molecule():
    mol = water_cluster(4, 2)
    rng = np.random.default_rng(5)
    r = random_rotation(rng)
    f1 = atom_frames(mol.positions)
    f2 = atom_frames(rotate(mol, r, np.array([0.3, 1.0, -2.0])).positions)
    for a, b in zip(f1, f2):
        np.testing.assert_allclose(a.T @ a, np.eye(3), atol=1e-12)
        assert np.linalg.det(a) > 0
        np.testing.assert_allclose(b, r @ a, atol=1e-10)
    # in a rigid water the oxygen's x axis points at the first hydrogen, y lies in the HOH plane
    o, h1, h2 = mol.positions[:3]
    np.testing.assert_allclose(f1[0][:, 0], (h1 - o) / np.linalg.norm(h1 - o), atol=1e-12)
    assert abs(np.dot(f1[0][:, 2], h2 - o)) < 1e-10
    # no frames for a linear molecule
    assert atom_frames(np.array([[0.0, 0, 0], [0, 0, 2.1], [0, 0, -2.1]])) is None


def test_edge_features_and_local_blocks_are_invariant_under_rigid_motions():
    from hafnium_b200.basis import ShellTable

    mol = water_cluster(6, 3)
    rng = np.random.default_rng(2)
    r = random_rotation(rng)
    moved = rotate(mol, r, np.array([1.0, -2.0, 0.5]))
    g1 = M.build_graph(mol)
    g2 = M.build_graph(moved)
    np.testing.assert_array_equal(g1["src"], g2["src"])
    np.testing.assert_array_equal(g1["elem"], g2["elem"])
    np.testing.assert_allclose(g1["edge"], g2["edge"], atol=1e-12)
    # a density that moves with the molecule (D' = W D W^T, W the AO rotation of r)
    # has the same local-frame blocks
    table = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
    n = g1["n_ao"]
    w = np.zeros((n, n))
    for a in range(mol.n_atoms):
        o, k = g1["offsets"][a], g1["nfun"][a]
        w[o:o + k, o:o + k] = ao_rotation(r, shell_layout(table, a))
    x = rng.normal(size=(n, n))
    dens = x + x.T
    t1 = M.local_targets(g1, dens)
    t2 = M.local_targets(g2, w @ dens @ w.T)
    np.testing.assert_allclose(t1["d"], t2["d"], atol=1e-10)
    np.testing.assert_allclose(t1["o"], t2["o"], atol=1e-10)


def test_local_blocks_round_trip_to_the_density():
    """Shell-pair blocks within the cutoff map back to the global density unchanged."""
    mol = water_cluster(5, 4)
    g = M.build_graph(mol)
    n = g["n_ao"]
    rng = np.random.default_rng(3)
    a = rng.normal(size=(n, n))
    dens = a + a.T
    # zero the blocks between atoms beyond the cutoff: the network never predicts them
    keep = np.zeros((g["n_nodes"], g["n_nodes"]), dtype=bool)
    np.fill_diagonal(keep, True)
    keep[g["src"], g["dst"]] = True
    atom = np.repeat(np.arange(g["n_nodes"]), g["nfun"])
    dens = np.where(keep[atom[:, None], atom[None, :]], dens, 0.0)
    mean = rng.normal(size=(len(M.ELEMENTS), M.DIAG))
    t = M.local_targets(g, dens, mean)
    back = M.blocks_to_density(g, t["d"], t["o"], mean)
    np.testing.assert_allclose(back, dens, atol=1e-12)
    # hydrogens have 5 of the 14 functions: their padding is zero
    h_rows = t["d"][g["elem"] == 0]
    pad = np.ones((M.NA_AO, M.NA_AO), dtype=bool)
    pad[:5, :5] = False
    assert np.allclose(h_rows[:, pad[np.triu_indices(M.NA_AO)]] + mean[0][pad[np.triu_indices(M.NA_AO)]], 0.0)


def test_weights_checksum_detects_corruption(tmp_path):
    params = {k: v.astype(np.float32) for k, v in small_params(np.random.default_rng(4)).items()}
    path = tmp_path / "w.npz"
    M.save_weights(path, params, np.zeros((len(M.ELEMENTS), 3)), {"note": "test", "elements": ["H", "O"]})
    assert M.load_weights(path) is not None
    with np.load(path) as z:
        arrays = {k: z[k] for k in z.files}
    arrays["Wd"] = arrays["Wd"] + 1.0
    np.savez_compressed(path, **arrays)
    assert M.load_weights(path) is None


def test_untrained_elements_and_linear_molecules_fall_back():
    weights = ({}, np.zeros((len(M.ELEMENTS), M.DIAG)), {"elements": ["H", "O"]})
    ammonia = Molecule(("N", "H", "H", "H"), np.array([[0.0, 0, 0], [1.9, 0, 0], [-0.6, 1.8, 0], [-0.6, -0.9, 1.5]]))
    assert M.predict_density(ammonia, weights) is None
    linear = Molecule(("O", "H", "H"), np.array([[0.0, 0, 0], [0, 0, 1.8], [0, 0, -1.8]]))
    assert M.build_graph(linear) is None
    assert M.predict_density(linear, weights) is None


def test_batched_rotations_and_the_torch_assembly_match_their_plain_forms():
    """harmonic_rotations (all frames at once) equals harmonic_rotation frame by frame, and
    assemble_density (torch, here on the CPU) equals blocks_to_density (NumPy)."""
    import torch

    from hafnium_b200.learned.frames import harmonic_rotations

    rng = np.random.default_rng(9)
    frames = [random_rotation(rng) for _ in range(5)]
    for l in range(3):
        batched = harmonic_rotations(frames, l)
        for f, u in zip(frames, batched):
            np.testing.assert_allclose(u, harmonic_rotation(f, l), atol=1e-13)
    g = M.build_graph(water_cluster(4, 6))
    d = rng.normal(size=(g["n_nodes"], M.DIAG))
    o = rng.normal(size=(len(g["src"]), M.OFF))
    mean = rng.normal(size=(len(M.ELEMENTS), M.DIAG))
    want = M.blocks_to_density(g, d, o, mean)
    got = M.assemble_density(g, torch.as_tensor(d), torch.as_tensor(o), mean, torch.device("cpu"))
    np.testing.assert_allclose(got.numpy(), want, atol=1e-13)
