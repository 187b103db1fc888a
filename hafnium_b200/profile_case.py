"""A small, fixed workload for kernel profiling (ncu) and kernel timing.

    python -m hafnium_b200.profile_case [--waters 16] [--repeats 1] [--batched 0] [--gradient]
                                        [--columns 0]

Builds one seeded (H2O)n (one-electron integrals, metric, factor, three-centre
integrals, fitted tensor), then runs ``repeats`` of each build on the
occupied orbitals of a converged-looking density (the core-Hamiltonian
orbitals; the kernels do not depend on the values): J, FP64 K, split-BF16 K.
With ``--batched C`` it also converges C seeded (H2O)2 clusters through the
batched graph-resident SCF; with ``--gradient`` it times the DF-RHF nuclear
gradient of the same orbitals (the kernels do not depend on the values). With
``--columns W`` the K builds use a random factor of W columns instead of the
occupied orbitals. Prints one JSON line with the device time of each step (CUDA
events), so the same command gives both the timing and, under ``ncu``, the
launch list of a bounded number of kernels.
"""

from __future__ import annotations

import argparse
import json


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--waters", type=int, default=16)
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--batched", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--gradient", action="store_true", help="also time the DF-RHF nuclear gradient")
    ap.add_argument("--columns", type=int, default=0,
                    help="factor width of the K builds (default: the occupied orbitals), e.g. 320 to give a "
                         "smaller cluster the (H2O)64 tile shape")
    args = ap.parse_args()

    import torch

    from hafnium_b200 import _lib
    from hafnium_b200.molecule import water_cluster
    from hafnium_b200.scf import DeviceHamiltonian

    dev = torch.device("cuda", 0)
    mol = water_cluster(args.waters, args.seed)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"waters": args.waters}
    e0.record()
    ham = DeviceHamiltonian.build(mol, "cc-pvdz", "def2-universal-jkfit")
    e1.record()
    e1.synchronize()
    out["build_ms"] = e0.elapsed_time(e1)
    out["build_stages_ms"] = {k: ham.timings.get(k) for k in ("ms_metric", "ms_factor", "ms_three_center", "ms_fit")}
    w, v = torch.linalg.eigh(ham.s)
    x = v / torch.sqrt(w)[None, :]
    _, c = torch.linalg.eigh(x.T @ ham.h @ x)
    occ = (x @ c[:, : int(mol.n_alpha)]).contiguous()
    if args.columns:
        gen = torch.Generator(device=occ.device).manual_seed(args.seed)
        kfac = torch.randn((occ.shape[0], args.columns), generator=gen, dtype=torch.float64, device=occ.device)
        kfac = (kfac / (occ.shape[0] * args.columns) ** 0.5).contiguous()
    else:
        kfac = occ
    d = (occ @ occ.T).contiguous()
    two_body = ham.two_body
    steps = (("coulomb", lambda: two_body.coulomb(2.0 * d)),
             ("exchange_fp64", lambda: two_body.exchange_factored(kfac)),
             ("exchange_bf16", lambda: two_body.exchange_factored(kfac, precision=_lib.PREC_BF16X3)))
    for name, fn in steps:
        fn()  # first call allocates scratch (and the BF16 copy of B)
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(args.repeats):
            fn()
        e1.record()
        e1.synchronize()
        out[f"{name}_ms"] = e0.elapsed_time(e1) / args.repeats
    n, naux, o = ham.n_ao, two_body.n_aux, int(kfac.shape[1])
    out["exchange_fp64_tflops"] = 4.0 * naux * n * n * o / (out["exchange_fp64_ms"] / 1e3) / 1e12
    out["exchange_bf16_exec_tflops"] = 3 * 4.0 * naux * n * n * o / (out["exchange_bf16_ms"] / 1e3) / 1e12
    out["coulomb_gbs"] = 2.0 * two_body.stats()["b_bytes"] / (out["coulomb_ms"] / 1e3) / 1e9
    if args.gradient:
        from hafnium_b200.gradient import gradient_from_state

        gradient_from_state(two_body, occ, ham.h, mol)  # first call loads the kernels
        torch.cuda.synchronize(dev)
        e0.record()
        gradient_from_state(two_body, occ, ham.h, mol)
        e1.record()
        e1.synchronize()
        out["gradient_ms"] = e0.elapsed_time(e1)
        st = two_body.stats()
        out["gradient_stages_ms"] = {k: st[f"ms_gradient_{k}"] for k in
                                     ("weights", "metric", "three_center", "one_electron")}
    del ham, two_body
    torch.cuda.empty_cache()
    if args.batched:
        from hafnium_b200.batch import BatchOptions, solve_batch

        mols = [water_cluster(2, 1000 + i) for i in range(args.batched)]
        res = solve_batch(mols, options=BatchOptions(gemm_tile=1))
        out["batched"] = {"clusters": args.batched, "seconds": res.seconds, "run_s": res.timings["run_s"],
                          "converged": int(sum(s == "converged" for s in res.states)),
                          "iterations": [int(i) for i in res.iterations]}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
