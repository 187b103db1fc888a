"""A small, fixed workload for kernel profiling (ncu) and kernel timing.

    python -m hafnium_b200.profile_case [--waters 16] [--repeats 1] [--batched 0] [--gradient]
                                        [--columns 0]
    python -m hafnium_b200.profile_case --gemm M,N,K [--repeats 3]

Builds one seeded (H2O)n (one-electron integrals, metric, factor, three-centre
integrals, fitted tensor), then runs ``repeats`` of each build on the
occupied orbitals of a converged-looking density (the core-Hamiltonian
orbitals; the kernels do not depend on the values): J, FP64 K, split-BF16 K.
With ``--batched C`` it also converges C seeded (H2O)2 clusters through the
batched graph-resident SCF; with ``--gradient`` it times the DF-RHF nuclear
gradient of the same orbitals (the kernels do not depend on the values). With
``--columns W`` the K builds use a random factor of W columns instead of the
occupied orbitals. ``--gemm M,N,K`` times only the FP64 DMMA GEMM C = A B^T on
random operands, every CTA tile of ``hf_dgemm_nt`` in turn and then cuBLAS
(``torch.matmul``) on the same product, checking each against it. Prints one JSON line with the device time of each step (CUDA
events), so the same command gives both the timing and, under ``ncu``, the
launch list of a bounded number of kernels.
"""

from __future__ import annotations

import argparse
import json


def gemm_case(torch, shape, repeats: int) -> None:
    """TF/s of every hf_dgemm_nt tile and of cuBLAS on C[M][N] = A[M][K] B[N][K]^T."""
    from hafnium_b200.batch import TILE_SHAPES, dgemm_nt

    m, n, k = shape
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev).manual_seed(0)
    a = torch.randn((1, m, k), dtype=torch.float64, device=dev, generator=gen)
    b = torch.randn((1, n, k), dtype=torch.float64, device=dev, generator=gen)
    c = torch.empty((1, m, n), dtype=torch.float64, device=dev)
    ref = a[0] @ b[0].T
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"gemm": [m, n, k]}

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(repeats):
            fn()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / repeats
        return {"ms": ms, "tflops": 2.0 * m * n * k / ms / 1e9}

    for tile, (bm, bn) in enumerate(TILE_SHAPES):
        row = timed(lambda: dgemm_nt(a, b, c, tile=tile))
        row["max_abs_diff"] = float((c[0] - ref).abs().max())
        out[f"tile{tile}_{bm}x{bn}"] = row
    out["cublas"] = timed(lambda: torch.matmul(a[0], b[0].T, out=c[0]))
    print(json.dumps(out), flush=True)


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
    ap.add_argument("--gemm", type=str, default="",
                    help="M,N,K: time the FP64 DMMA GEMM tiles and cuBLAS on one product instead")
    args = ap.parse_args()

    import torch

    if args.gemm:
        gemm_case(torch, [int(x) for x in args.gemm.split(",")], max(1, args.repeats))
        return

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
