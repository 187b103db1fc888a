"""Train the learned initial density on converged densities from this SCF.

    python -m hafnium_b200.learned.train [--clusters 16000] [--epochs 100] [--lr 3e-4] [--out weights.npz]

(the defaults are the recipe of the shipped weights, weights_ccpvdz_atoms.npz)

1. Seeded water clusters (H2O)n, n uniform in [2, 12], are converged together
   by the batched device DF-RHF (SAD guess, FP64, the reference's default
   tolerances). Their per-spin densities, expressed in the frames of their
   atoms (the shell-pair blocks of every atom and every atom pair within the
   cutoff), are the targets.
2. The network (hafnium_b200.learned.model) is trained with Adam on the device,
   forward and backward running on the hfnn kernels, several clusters per step.
3. Held-out (H2O)16-24 clusters are converged from the SAD guess and from the
   learned guess; iteration counts, first gradients, times (guess included)
   and energies are recorded in the weights file's metadata.
"""

from __future__ import annotations

import argparse
import json
import pathlib
import time

import numpy as np

from hafnium_b200.learned import model as M

BASIS, AUX = "cc-pvdz", "def2-universal-jkfit"


def converged_density(mol, device: int = 0):
    from hafnium_b200.scf import DeviceHamiltonian, atomic_density_guess, solve_rhf

    ham = DeviceHamiltonian.build(mol, BASIS, AUX, device=device)
    res = solve_rhf(ham, guess=atomic_density_guess(mol, BASIS, device=device))
    return res.density.cpu().numpy(), res


def make_dataset(count: int, seed0: int, n_range=(2, 12), device: int = 0, batched: bool = True):
    """Converged per-spin densities of seeded clusters as training targets: by
    default all clusters at once through the batched graph-resident SCF (the
    same converged densities as the per-cluster path, to 1e-6)."""
    from hafnium_b200.molecule import water_cluster

    rng = np.random.default_rng(seed0)
    mols = [water_cluster(int(rng.integers(n_range[0], n_range[1] + 1)), seed0 + 1000 + k) for k in range(count)]
    if batched:
        from hafnium_b200.batch import solve_batch

        res = solve_batch(mols, BASIS, AUX, device=device, keep_densities=True)
        keep = [i for i, s in enumerate(res.states) if s == "converged"]
        dens = [res.densities[i] for i in keep]
        mols = [mols[i] for i in keep]
    else:
        dens = [converged_density(m, device)[0] for m in mols]
    data = []
    for mol, d in zip(mols, dens):
        graph = M.build_graph(mol)
        if graph is None:
            continue
        tgt = M.local_targets(graph, d)
        # the training steps need neither the rotations nor FP64 targets
        graph = {k: v for k, v in graph.items() if k != "rot"}
        data.append((graph, {"d": tgt["d"], "o": tgt["o"].astype(np.float32)}))
    return data


def union(batch):
    """Disjoint union of several graphs and their targets (one training step)."""
    offset = 0
    elem, src, dst, edge, fcut, d, o = [], [], [], [], [], [], []
    for graph, tgt in batch:
        elem.append(graph["elem"])
        src.append(graph["src"] + offset)
        dst.append(graph["dst"] + offset)
        edge.append(graph["edge"])
        fcut.append(graph["fcut"])
        d.append(tgt["d"])
        o.append(tgt["o"])
        offset += graph["n_nodes"]
    g = {"n_nodes": offset, "elem": np.concatenate(elem).astype(np.int32),
         "src": np.concatenate(src).astype(np.int32), "dst": np.concatenate(dst).astype(np.int32),
         "edge": np.concatenate(edge), "fcut": np.concatenate(fcut)}
    return g, {"d": np.concatenate(d), "o": np.concatenate(o)}


def element_means(data) -> np.ndarray:
    """The mean diagonal block of each element over the training atoms (zero for
    elements that do not occur)."""
    total = np.zeros((len(M.ELEMENTS), M.DIAG))
    count = np.zeros(len(M.ELEMENTS))
    for graph, tgt in data:
        np.add.at(total, graph["elem"], tgt["d"])
        np.add.at(count, graph["elem"], 1.0)
    return total / np.maximum(count, 1.0)[:, None]


def train(data, epochs: int, batch: int = 8, lr: float = 1e-3, seed: int = 0, device: int = 0, log=print):
    import torch

    mean_diag = element_means(data)
    net = M.DeviceNet(M.init_params(seed), device=device)
    opt = M.Adam(net, lr)
    rng = np.random.default_rng(seed)
    dev = net.dev
    prepared = []
    for i in range(0, len(data), batch):
        g, t = union(data[i:i + batch])
        gd = net.upload_graph(g)
        td = {"d": torch.as_tensor(t["d"] - mean_diag[g["elem"]], dtype=torch.float32, device=dev).contiguous(),
              "o": torch.as_tensor(t["o"], dtype=torch.float32, device=dev).contiguous()}
        prepared.append((gd, td, float(len(t["d"]))))
    history = []
    for epoch in range(epochs):
        total, nodes = 0.0, 0.0
        for k in rng.permutation(len(prepared)):
            gd, td, nn = prepared[k]
            loss, grads = net.loss_and_grad(gd, td)
            opt.apply(grads, scale=1.0 / nn)
            total += float(loss.item())
            nodes += nn
        if epoch >= epochs // 2:
            opt.lr = lr * 0.5 * (1 + np.cos(np.pi * (epoch - epochs // 2) / max(1, epochs - epochs // 2)))
        history.append(total / nodes)
        log(f"epoch {epoch:3d}  loss per atom {total / nodes:.4e}")
    params = {k: v.cpu().numpy() for k, v in net.p.items()}
    return params, mean_diag, history


def evaluate(weights, sizes, seed0: int, device: int = 0, per_size: int = 3):
    """Plain FP64 SCF from the SAD guess and from the learned guess on held-out
    clusters (seeds disjoint from training): iterations, first-iteration
    gradient, and wall time including the guess itself, after a warm-up run."""
    import torch

    from hafnium_b200.molecule import water_cluster
    from hafnium_b200.scf import DeviceHamiltonian, atomic_density_guess, learned_density_guess, solve_rhf

    warm = water_cluster(4, seed0 + 49999)
    wham = DeviceHamiltonian.build(warm, BASIS, AUX, device=device)
    solve_rhf(wham, guess=learned_density_guess(warm, wham, weights=weights, device=device))
    solve_rhf(wham, guess=atomic_density_guess(warm, BASIS, device=device))
    del wham
    rows = []
    for k, n in enumerate(s for s in sizes for _ in range(per_size)):
        mol = water_cluster(n, seed0 + 50000 + k)
        ham = DeviceHamiltonian.build(mol, BASIS, AUX, device=device)
        out = {"n_waters": n}
        for name, make in (("sad", lambda: atomic_density_guess(mol, BASIS, device=device)),
                           ("learned", lambda: learned_density_guess(mol, ham, weights=weights, device=device))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = solve_rhf(ham, guess=make())
            torch.cuda.synchronize()
            out[f"{name}_iterations"] = res.n_iterations
            out[f"{name}_first_gradient"] = res.history[0].gradient_norm
            out[f"{name}_s"] = time.perf_counter() - t0
            out[f"{name}_energy"] = res.energy
        out["dE"] = out["learned_energy"] - out["sad_energy"]
        rows.append(out)
        del ham
    return rows


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=16000)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=3e-4)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--eval", type=str, default="16,20,24")
    ap.add_argument("--out", type=str, default=str(M.WEIGHTS))
    args = ap.parse_args()
    t0 = time.perf_counter()
    data = make_dataset(args.clusters, args.seed)
    t1 = time.perf_counter()
    print(f"dataset: {len(data)} clusters in {t1 - t0:.1f} s", flush=True)
    params, mean_diag, history = train(data, args.epochs, args.batch, args.lr, args.seed)
    t2 = time.perf_counter()
    trained = sorted({M.ELEMENTS[e] for graph, _ in data for e in graph["elem"]})
    meta = {"clusters": args.clusters, "n_range": [2, 12], "elements": trained, "epochs": args.epochs,
            "batch": args.batch, "lr": args.lr,
            "seed": args.seed, "basis": BASIS, "auxiliary": AUX, "loss_history": history,
            "dataset_s": t1 - t0, "train_s": t2 - t1}
    out = pathlib.Path(args.out)
    M.save_weights(out, params, mean_diag, meta)
    rows = evaluate((params, mean_diag, meta), [int(x) for x in args.eval.split(",") if x], args.seed)
    meta["evaluation"] = rows
    digest = M.save_weights(out, params, mean_diag, meta)
    print(json.dumps({"weights": str(out), "sha256": digest, "evaluation": rows, "final_loss": history[-1]}),
          flush=True)


if __name__ == "__main__":
    main()
