"""Benchmark: DF-RHF time-to-converge of a seeded water cluster on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--waters 64] [--impl b200|reference]

One step is one whole DF-RHF from the geometry: one-electron integrals, the
Coulomb metric, its Cholesky factor, the three-centre integrals, the packed
fitted tensor B = L^-1 (P|uv), and the SCF iterations (DIIS, reference default
tolerances |dE| < 1e-10 and gradient < 1e-6) to convergence; the clusters are
the seeded (H2O)n of hafnium_b200.molecule (cc-pVDZ / def2-universal-jkfit,
the stand-in for the unavailable cc-pVDZ-JKFIT). B is tens of GB, far above
the 126 MB L2, so no flush is needed between steps.

``value`` is the device-timed (CUDA events) time-to-converge of the learned
guess + mixed-precision schedule: the K timed steps as one region divided by K,
max over ranks, beside the plain FP64 path from the SAD guess timed the same
way (the slowest and per-step times are in the line too). ``e2e`` is the learned + mixed SCF as the reference's own
driver would run it: the driver calls nothing but the drop-in's ``coulomb(2 D)``
and ``exchange(D)`` with host NumPy arrays (host -> device copy of D, device ->
host of J and K inside the timed region), the drop-in choosing each build's
arithmetic itself (``schedule="mixed"``): wall clock around each run, the mean
of three runs after an untimed one (the slowest is in the line too). Several GPUs run independent replicas
(no collective on the path). ``--impl reference`` times the reference's CPU
path (the oracle's restatement: NumPy/OpenBLAS DF-RHF over C++/OpenMP
integrals) on the host cores.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DF-RHF (H2O)64 time-to-converge at |ΔE|≤1e-8 Eh: learned+mixed vs plain FP64 GPU"
BASIS, AUX = "cc-pvdz", "def2-universal-jkfit"
# DRAM bytes of one split-BF16 K build, k_tc_split3 stage 1 + stage 2 (ncu --set full,
# dram__bytes_read.sum + dram__bytes_write.sum) at n = 384, N = 1808 with a 320-column factor:
# the part that scales with the BF16 copy of B (N npad^2) and the part that scales with X (N npad ncols)
TC_TRAFFIC_B_H2O16 = 1.075544e9
TC_TRAFFIC_X_H2O16 = 0.842216e9 + 1.205165e9 + 0.020353e9
TC_UNITS_B_H2O16 = 1808 * 384 ** 2
TC_UNITS_X_H2O16 = 1808 * 384 * 320


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--waters", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ablation", action="store_true",
                    help="also run SAD+mixed and learned+plain once each (outside the timed steps)")
    ap.add_argument("--fit-waters", default="12,16",
                    help="--impl reference: the cluster sizes measured once each, beside the (H2O)8 steps, for the "
                         "scaling fit that carries the reference's time to the benchmark size")
    ap.add_argument("--batched", type=int, default=0,
                    help="run the batched workload instead: this many seeded (H2O)n, n uniform in [2, 16]")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(values, device=None):
    """Element-wise max of per-rank step times across the process group (a no-op
    without one): the whole-job time of replicas is the slowest rank's."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int) -> None:
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self) -> None:
        """Start sampling and return once the first sample is written, so that
        nvidia-smi's own start-up (NVML initialisation) is over before the timed
        region begins (at most 5 s)."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None
            return
        deadline = time.time() + 5.0
        while time.time() < deadline and self.proc.poll() is None:
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.05)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.flush()
        rows = []
        with open(self.file.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def measure_fp64_peak(torch, dev) -> float:
    """Dense FP64 tensor-core throughput of cuBLAS on this GPU (TFLOP/s), for the roofline."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = math.inf
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2 * 8192 ** 3 / best / 1e12


def exchange_kernel_ms(torch, ham, result, repeats: int = 3) -> dict:
    """Device time of one K build from the converged occupied orbitals, split-BF16
    and FP64 (CUDA events on the launching stream, after one warm-up call)."""
    from hafnium_b200 import _lib

    n_occ = int(ham.n_alpha)
    order = torch.argsort(result.mo_energies)[:n_occ]
    c = result.mo_coefficients[:, order].contiguous()
    out = {}
    for name, prec, reps in (("bf16", _lib.PREC_BF16X3, repeats), ("fp64", _lib.PREC_FP64, 1)):
        ham.two_body.exchange_factored(c, precision=prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            ham.two_body.exchange_factored(c, precision=prec)
        e1.record()
        e1.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    return out


def one_scf(torch, mol, dev, mode="mixed", guess_kind="sad", probe_kernels=False, protocol=False):
    """One whole DF-RHF from the geometry. ``protocol``: the driver calls only the
    drop-in's coulomb(2 D) / exchange(D) on host NumPy arrays and the drop-in's
    own mixed schedule chooses each build's arithmetic."""
    from hafnium_b200.scf import (DeviceHamiltonian, PrecisionSchedule, ScfOptions, atomic_density_guess,
                                  learned_density_guess, solve_rhf)

    t_ham = time.perf_counter()
    ham = DeviceHamiltonian.build(mol, BASIS, AUX, device=dev.index or 0,
                                  exchange_schedule="mixed" if protocol else "fp64")
    t_ham = time.perf_counter() - t_ham
    t_guess = time.perf_counter()
    if guess_kind == "learned":
        guess = learned_density_guess(mol, ham, device=dev.index or 0)
    else:
        guess = atomic_density_guess(mol, BASIS, device=dev.index or 0)
    torch.cuda.synchronize()
    t_guess = time.perf_counter() - t_guess
    result = solve_rhf(ham, guess=guess, options=ScfOptions(), host_io=protocol, protocol=protocol,
                       schedule=PrecisionSchedule(mode="fp64" if protocol else mode))
    kernel_ms = None
    if probe_kernels:
        kernel_ms = exchange_kernel_ms(torch, ham, result)
    stats = ham.two_body.stats()
    out = {"energy": result.energy, "iterations": result.n_iterations, "converged": result.converged,
           "ms_factorize_density_last": stats["ms_factorize_density"],
           "build": {k: ham.timings.get(k) for k in ("ms_metric", "ms_factor", "ms_three_center", "ms_fit",
                                                     "one_electron_s", "fitted_tensor_s")},
           "scf": {**result.timings, "guess_s": t_guess, "scf_s": result.seconds, "hamiltonian_s": t_ham},
           "launches": stats["kernel_launches"], "n_ao": ham.n_ao,
           "n_aux": ham.two_body.n_aux, "b_bytes": stats["b_bytes"],
           "precisions": [h.precision for h in result.history], "kernel_ms": kernel_ms,
           "density": result.density.detach().cpu().numpy()}
    t_free = time.perf_counter()
    del ham, result
    torch.cuda.synchronize()
    out["scf"]["teardown_s"] = time.perf_counter() - t_free
    return out


def step_breakdown(info: dict) -> dict:
    """Where one step's time went (seconds; the exchange by arithmetic)."""
    scf = info["scf"]
    out = {"hamiltonian": scf["hamiltonian_s"], "guess": scf["guess_s"], "scf": scf["scf_s"],
           "teardown": scf["teardown_s"], "coulomb": scf["coulomb_ms"] / 1e3, "eigh": scf["eigh_ms"] / 1e3,
           "exchange": scf["exchange_ms"] / 1e3}
    for key, value in scf.items():
        if key.startswith("exchange_ms_"):
            out["exchange_" + key[len("exchange_ms_"):]] = value / 1e3
    return {k: round(v, 4) for k, v in out.items()}


def tc_executed_flops(n: int, naux: int, ncols: int) -> float:
    """Tensor-core flops one split-BF16 K build executes (three BF16 products):
    stage 1 over the padded shapes, stage 2 over the output tiles it computes
    (those that touch the upper triangle)."""
    npad = (n + 127) // 128 * 128
    opad = max(64, (ncols + 63) // 64 * 64)
    stage1 = 2.0 * naux * npad * npad * opad
    bn2 = 256 if npad % 256 == 0 else 128
    upper = sum(1 for mt in range(npad // 128) for nt in range(npad // bn2) if (nt + 1) * bn2 > mt * 128)
    stage2 = 2.0 * upper * 128 * bn2 * naux * opad
    return 3.0 * (stage1 + stage2)


def timed_scf(torch, dev, mol, **kw):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    info = one_scf(torch, mol, dev, **kw)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, info


def run_b200(args) -> None:
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from hafnium_b200.molecule import water_cluster

    mol = water_cluster(args.waters, args.seed + rank)
    from hafnium_b200.learned.model import load_weights

    weights = load_weights()
    guess_kind = "learned" if weights is not None else "sad"
    for i in range(args.warmup):
        one_scf(torch, mol, dev, mode="mixed", guess_kind=guess_kind)
        if i == 0:
            one_scf(torch, mol, dev, mode="fp64")
            one_scf(torch, mol, dev, guess_kind=guess_kind, protocol=True)
    if world > 1:
        dist.barrier()
    import gc

    gc.collect()  # the warm-up's garbage, not the first timed step's
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local)
    sampler.start()

    def timed_region(**kw):
        """K whole SCFs as one timed region (CUDA events, synchronised on both sides,
        a barrier before under torchrun), each step also timed on its own."""
        steps, infos = [], []
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record()
        for _ in range(args.steps):
            t, info = timed_scf(torch, dev, mol, **kw)
            steps.append(t)
            infos.append(info)
        r1.record()
        r1.synchronize()
        return r0.elapsed_time(r1) / 1e3, steps, infos

    region, times, details = timed_region(mode="mixed", guess_kind=guess_kind)
    plain_region, plain_times, plain_details = timed_region(mode="fp64", guess_kind="sad")
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    # kernel-only timing of the exchange builds for the roofline, outside the timed steps
    probe = one_scf(torch, mol, dev, mode="mixed", guess_kind=guess_kind, probe_kernels=True)["kernel_ms"]
    ablation = None
    if args.ablation:
        # which part of the gain is the guess and which the precision schedule, one
        # run each (CUDA events around the whole SCF as above)
        ablation = {}
        for label, mode, kind in (("sad_mixed", "mixed", "sad"), ("learned_fp64", "fp64", guess_kind)):
            seconds, info = timed_scf(torch, dev, mol, mode=mode, guess_kind=kind)
            ablation[label] = {"seconds": seconds, "iterations": info["iterations"],
                               "energy": info["energy"], "precisions": info["precisions"],
                               "scf_s": info["scf"]["scf_s"], "hamiltonian_s": info["scf"]["hamiltonian_s"]}
    # seconds per step: each path's whole timed region over its K steps, max over ranks
    step_mean, plain_mean = max_over_ranks([region / args.steps, plain_region / args.steps], dev)
    if world > 1:
        dist.barrier()
    e2e = None
    if not args.no_e2e:
        # the reference's call pattern end to end: host NumPy D in, host NumPy J and K out,
        # the drop-in's own mixed schedule; wall clock around the whole run
        # one untimed run first (the protocol path's own first-call allocations), then the
        # timed runs as one region, divided by their count like ``value``
        one_scf(torch, mol, dev, guess_kind=guess_kind, protocol=True)
        e2e_times, e2e_info = [], None
        for _ in range(min(3, max(1, args.steps))):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            e2e_info = one_scf(torch, mol, dev, guess_kind=guess_kind, protocol=True)
            torch.cuda.synchronize(dev)
            e2e_times.append(time.perf_counter() - t0)
        e2e_mean, e2e_slowest = max_over_ranks([sum(e2e_times) / len(e2e_times), max(e2e_times)], dev)
        e2e = {"value": e2e_mean, "unit": "s", "slowest_s": e2e_slowest,
               "h2d_bytes_per_step": e2e_info["scf"]["h2d_bytes"],
               "d2h_bytes_per_step": e2e_info["scf"]["d2h_bytes"], "energy": e2e_info["energy"],
               "step_times_s": e2e_times, "iterations": e2e_info["iterations"],
               "precisions": e2e_info["precisions"], "step_breakdown_s": step_breakdown(e2e_info),
               "ms_factorize_density_last_call": e2e_info["ms_factorize_density_last"],
               "path": "learned guess; the device driver calls only coulomb(2D) and exchange(D) of the drop-in with "
                       "host NumPy arrays (host -> device D, device -> host J and K) and the reference's convergence "
                       "test; the drop-in (schedule='mixed') chooses split-BF16, anchored incremental or FP64 "
                       "arithmetic from the densities alone (its pivoted Cholesky of D included)"}
    # the GPU at the sizes the CPU baseline measures, one run each after a warm-up run
    same_size = {}
    for waters in (8, 16):
        small = water_cluster(waters, args.seed + rank)
        one_scf(torch, small, dev, mode="fp64")
        t_plain, _ = timed_scf(torch, dev, small, mode="fp64", guess_kind="sad")
        t_mixed, _ = timed_scf(torch, dev, small, mode="mixed", guess_kind=guess_kind)
        same_size[f"h2o{waters}"] = {"plain_fp64_s": t_plain, "learned_mixed_s": t_mixed}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    last = details[-1]
    plain = plain_details[-1]
    n, naux = last["n_ao"], last["n_aux"]
    o = mol.n_alpha
    fock_builds = plain["scf"]["fock_builds"]
    k64_ms = plain["scf"]["exchange_ms_fp64"] / plain["scf"]["exchange_builds_fp64"]
    j_ms = plain["scf"]["coulomb_ms"] / fock_builds
    k_flops = 4.0 * naux * n * n * o
    j_bytes = 2.0 * last["b_bytes"]
    k16_ms = probe["bf16"]
    k64_probe_ms = probe["fp64"]
    inc_builds = last["scf"].get("exchange_builds_incremental", 0)
    inc_ms = last["scf"]["exchange_ms_incremental"] / inc_builds if inc_builds else None
    fp64_peak = measure_fp64_peak(torch, dev)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    k64_tflops = k_flops / (k64_ms / 1e3) / 1e12
    j_gbs = j_bytes / (j_ms / 1e3) / 1e9
    npad = (n + 127) // 128 * 128
    traffic = (TC_TRAFFIC_B_H2O16 * naux * npad ** 2 / TC_UNITS_B_H2O16
               + TC_TRAFFIC_X_H2O16 * naux * npad * o / TC_UNITS_X_H2O16)
    algorithmic = 3.0 * k_flops
    executed = tc_executed_flops(n, naux, o)
    roofline = {"bound": "tensor", "kernel": "split-BF16 exchange on tcgen05 (k_tc_split3, both stages), "
                                             "one K build from the converged occupied orbitals",
                "achieved": algorithmic / (k16_ms / 1e3) / 1e12, "peak": bf16_peak, "unit": "TFLOP/s",
                "frac": algorithmic / (k16_ms / 1e3) / 1e12 / bf16_peak,
                "algorithmic": "3 x 4 naux n^2 nocc BF16 flops per K build (three split products of the "
                               "occupied-factor exchange)",
                "executed_tflops": executed / (k16_ms / 1e3) / 1e12,
                "frac_executed": executed / (k16_ms / 1e3) / 1e12 / bf16_peak,
                "executed": "flops the tensor cores run: stage 1 in full, stage 2 over the output tiles that "
                            "touch the upper triangle (%.3f of algorithmic)" % (executed / algorithmic),
                "traffic": traffic,
                "traffic_note": "DRAM bytes per K build: ncu dram__bytes_read.sum + dram__bytes_write.sum of both "
                                "stages at n=384, N=1808, 320 columns, scaled by N npad^2 (the BF16 copy of B) and "
                                "N npad nocc (X written by stage 1 and read by stage 2)",
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst, of measured)",
                "kernel_ms": k16_ms}
    setup_s = float(np.median([d["scf"]["hamiltonian_s"] for d in details + plain_details]))
    line = {
        "metric": METRIC,
        "value": step_mean,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_mean * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded rigid-water clusters (no dataset)",
        "config": {"workload": f"DF-RHF (H2O){args.waters} seed {args.seed}, cc-pVDZ/def2-universal-jkfit "
                               f"(n={n}, naux={naux}, nocc={o}), {guess_kind} guess, mixed split-BF16/FP64 "
                               f"exchange; compared with plain FP64 from the SAD guess",
                   "waters": args.waters, "basis": BASIS, "auxiliary": AUX, "precision_path": "mixed",
                   "guess": guess_kind if weights is None else
                   f"learned (weights sha256 {weights[2].get('sha256', '')[:12]}, trained on "
                   f"{weights[2].get('clusters')} clusters); SAD fallback",
                   "l2": "inputs larger than L2 (B tensor %.1f GB)" % (last["b_bytes"] / 1e9),
                   "sad_atoms": "converged once per process and element, then reused by every step (both paths)",
                   "parallelism": f"replicas x{world}"},
        "energy": last["energy"],
        "iterations": last["iterations"],
        "converged": last["converged"],
        "precisions": last["precisions"],
        "exchange_builds": {k[len("exchange_builds_"):]: v for k, v in last["scf"].items()
                            if k.startswith("exchange_builds_")},
        "step_times_s": times,
        "step_breakdown_s": [step_breakdown(d) for d in details],
        "plain_fp64": {"value": plain_mean, "step_times_s": plain_times, "energy": plain["energy"],
                       "iterations": plain["iterations"], "speedup_of_mixed": plain_mean / step_mean,
                       "speedup_of_mixed_slowest": max(plain_times) / max(times),
                       "speedup_of_mixed_median": float(np.median(plain_times) / np.median(times)),
                       "build": plain["build"],
                       "dE_mixed_vs_fp64": last["energy"] - plain["energy"],
                       "max_abs_dD_mixed_vs_fp64": float(np.max(np.abs(last["density"] - plain["density"])))},
        "ratio_bounds": {"shared_setup_s": setup_s,
                         "plain_over_setup": float(np.median(plain_times)) / setup_s,
                         "plain_over_setup_plus_two_fp64_k": float(np.median(plain_times)) /
                         (setup_s + 2.0 * k64_ms / 1e3),
                         "note": "the Hamiltonian (integrals, FP64 fit of B) is shared by both paths; with the two "
                                 "FP64 exchange builds the mixed path keeps, the speed-up cannot exceed "
                                 "plain_over_setup_plus_two_fp64_k however fast the rest becomes"},
        "same_size": same_size,
        "ablation": ablation,
        "stages": {"build": last["build"], "per_build_ms": {"coulomb": j_ms, "exchange_fp64": k64_ms,
                                                             "exchange_bf16_kernel": k16_ms,
                                                             "exchange_fp64_kernel": k64_probe_ms,
                                                             "exchange_incremental": inc_ms},
                   "mixed_scf": last["scf"], "plain_scf": plain["scf"]},
        "roofline": roofline,
        "roofline_exchange_fp64": {"bound": "tensor", "achieved": k64_tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                                   "frac": k64_tflops / fp64_peak, "algorithmic": "4 naux n^2 nocc flops per K (the "
                                   "SYRK half computes the upper tiles only, so executed flops are fewer)",
                                   "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run"},
        "roofline_coulomb": {"bound": "hbm", "achieved": j_gbs, "peak": hbm_peak, "unit": "GB/s",
                             "frac": j_gbs / hbm_peak, "algorithmic": "2 passes over packed B per J",
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
        "clocks": clocks,
        "gpu_launches": int(last["launches"]),
        "e2e": e2e,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.waters, (8, 12))
    print(json.dumps(line), flush=True)


def cpu_reference_scf(n_waters: int, seed: int) -> dict:
    """The reference's CPU path (oracle restatement) for one seeded cluster, timed."""
    from hafnium_b200.basis import ShellTable
    from hafnium_b200.molecule import water_cluster
    from oracle import dfrhf, kernels

    mol = water_cluster(n_waters, seed)
    t0 = time.perf_counter()
    orb = ShellTable.build(BASIS, mol.symbols, mol.positions)
    aux = ShellTable.build(AUX, mol.symbols, mol.positions)
    prob = dfrhf.build_problem(orb, aux, mol.nuclear_charges, mol.positions, mol.nuclear_repulsion_energy(),
                               mol.n_alpha)
    guess = dfrhf.atomic_density_guess(orb, mol.symbols, {"O": 8.0, "H": 1.0})
    t1 = time.perf_counter()
    # OpenBLAS runs the reference's stacked B @ D (coulomb_exchange.py:188) ~10x faster on one
    # thread than on all cores on these hosts, so the reference's SCF gets the faster setting.
    from threadpoolctl import threadpool_limits

    with threadpool_limits(limits=1, user_api="blas"):
        result = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, prob.n_alpha, guess=guess)
    t2 = time.perf_counter()
    return {"seconds": t2 - t0, "setup_s": t1 - t0, "scf_s": t2 - t1, "iterations": result.n_iterations,
            "energy": result.energy, "threads": kernels.threads(), "n": orb.n_functions, "waters": n_waters}


def scaling_fit(points: list[dict]) -> dict:
    """Least-squares exponent p of t = a n^p over the measured points."""
    x = np.log([p["n"] for p in points])
    y = np.log([p["seconds"] for p in points])
    slope, intercept = np.polyfit(x, y, 1) if len(points) > 1 else (4.0, y[0] - 4.0 * x[0])
    return {"exponent": float(slope), "log_prefactor": float(intercept)}


def cpu_baseline(n_target: int, sizes=(8, 12)) -> dict:
    """The reference CPU path measured on a bounded sample of clusters (about 30 s
    of CPU work for (H2O)8 and (H2O)12 here), and its time at the benchmark size
    from the fitted power law, labelled as an extrapolation: the reference's
    full-layout fitted tensor of (H2O)64 would need about 410 GB of host memory."""
    points = [cpu_reference_scf(w, 0) for w in sizes]
    fit = scaling_fit(points)
    n_target_ao = 24 * n_target
    value = float(math.exp(fit["log_prefactor"]) * n_target_ao ** fit["exponent"])
    return {"value": value, "unit": "s", "cores": points[0]["threads"], "kind": "port",
            "sample": "measured: " + ", ".join(f"(H2O){p['waters']} (n={p['n']}) {p['seconds']:.2f} s, "
                                               f"{p['iterations']} iterations" for p in points)
                      + f"; value = the fit t ~ n^{fit['exponent']:.2f} extrapolated to (H2O){n_target} "
                        f"(n={n_target_ao}); integrals on all OpenMP threads, SCF BLAS on 1 thread (its fastest)",
            "measured": [{k: p[k] for k in ("waters", "n", "seconds", "setup_s", "scf_s", "iterations")}
                         for p in points],
            "fit": fit, "extrapolated": True}


def run_reference(args) -> None:
    """The reference's CPU path on the host cores: each timed step one (H2O)8 DF-RHF
    (the reference's CPU-sized case); the ``--fit-waters`` sizes ((H2O)12 and
    (H2O)16 by default) once each for the scaling fit that carries the value to
    the benchmark size."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(threads))
    times = []
    sample = None
    for i in range(args.warmup + args.steps):
        sample = cpu_reference_scf(8, args.seed)
        if i >= args.warmup:
            times.append(sample["seconds"])
    points = [dict(sample, seconds=statistics.median(times))]
    points += [cpu_reference_scf(int(w), args.seed) for w in args.fit_waters.split(",") if w.strip()]
    fit = scaling_fit(points)
    n_target_ao = 24 * args.waters
    value = float(math.exp(fit["log_prefactor"]) * n_target_ao ** fit["exponent"])
    desc = ("measured on the host cores: " + ", ".join(f"(H2O){p['waters']} (n={p['n']}) {p['seconds']:.2f} s"
                                                       for p in points)
            + f" ((H2O)8 the median of {args.steps} steps); value = the fit t ~ n^{fit['exponent']:.2f} "
              f"extrapolated to (H2O){args.waters} (the reference layout of (H2O)64 needs ~410 GB of host memory)")
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded rigid-water clusters",
        "config": {"workload": f"DF-RHF (H2O){args.waters} seed {args.seed}, cc-pVDZ/def2-universal-jkfit",
                   "waters": args.waters},
        "step_times_s": times,
        "measured": [{k: p[k] for k in ("waters", "n", "seconds", "setup_s", "scf_s", "iterations", "energy")}
                     for p in points],
        "fit": fit,
        "cpu_baseline": {"value": value, "unit": "s", "cores": sample["threads"], "kind": "port", "sample": desc,
                         "extrapolated": True},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


BATCH_METRIC = "batched DF-RHF throughput: seeded (H2O)n clusters, n uniform in [2,16], converged per second"


def batched_clusters(count: int, seed: int):
    from hafnium_b200.molecule import water_cluster

    rng = np.random.default_rng(seed)
    sizes = rng.integers(2, 17, size=count)
    return [water_cluster(int(n), seed * 100000 + i) for i, n in enumerate(sizes)]


def run_batched(args) -> None:
    """Many clusters of uneven size through the graph-resident batched SCF (one
    graph launch per wave). value = clusters converged per second, from the
    geometries (integrals, fitted tensors, SCF) to host energies."""
    import torch

    from hafnium_b200 import batch as hb

    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    mols = batched_clusters(args.batched, args.seed + rank)
    tuner = hb.TileTuner()
    # warm-up: library load, SAD atoms, and the tile choice of every shape at its batch size
    hb.solve_batch(mols[:4], device=local, tuner=tuner)
    counts = {}
    for m in mols:
        counts[m.n_atoms] = counts.get(m.n_atoms, 0) + 1
    for atoms, c in counts.items():
        tuner.choose(24 * atoms // 3, min(c, 256), local)
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local)
    sampler.start()
    t0 = time.perf_counter()
    res = hb.solve_batch(mols, device=local, tuner=tuner)
    torch.cuda.synchronize(dev)
    seconds = time.perf_counter() - t0
    clocks = sampler.stop()
    # accuracy: the plain per-cluster FP64 path (pinned to the oracle) on one cluster of each size,
    # and the oracle itself on the two smallest clusters
    from hafnium_b200.scf import DeviceHamiltonian, atomic_density_guess, solve_rhf

    checked, worst = 0, 0.0
    seen = set()
    for i, m in enumerate(mols):
        if m.n_atoms in seen:
            continue
        seen.add(m.n_atoms)
        ham = DeviceHamiltonian.build(m, BASIS, AUX, device=local)
        ref = solve_rhf(ham, guess=atomic_density_guess(m, BASIS, device=local))
        worst = max(worst, abs(ref.energy - res.energies[i]))
        checked += 1
        del ham
    torch.cuda.empty_cache()
    oracle_worst = 0.0
    small = sorted(range(len(mols)), key=lambda i: mols[i].n_atoms)[:2]
    from oracle import dfrhf
    from hafnium_b200.basis import ShellTable

    for i in small:
        m = mols[i]
        orb = ShellTable.build(BASIS, m.symbols, m.positions)
        aux = ShellTable.build(AUX, m.symbols, m.positions)
        prob = dfrhf.build_problem(orb, aux, m.nuclear_charges, m.positions, m.nuclear_repulsion_energy(), m.n_alpha)
        guess = dfrhf.atomic_density_guess(orb, m.symbols, {"O": 8.0, "H": 1.0})
        ref = dfrhf.solve_rhf(prob.s, prob.h, dfrhf.FittedJK(prob.b), prob.e_nuc, m.n_alpha, guess=guess)
        oracle_worst = max(oracle_worst, abs(ref.energy - res.energies[i]))
    waters = [m.n_atoms // 3 for m in mols]
    k_flops = sum(4.0 * (113 * w) * (24 * w) ** 2 * (5 * w) * int(it) for w, it in zip(waters, res.iterations))
    fp64_peak = measure_fp64_peak(torch, dev)
    k_tflops = k_flops / res.timings["run_s"] / 1e12
    line = {
        "metric": BATCH_METRIC, "value": len(mols) / seconds, "unit": "clusters/s", "n_gpus": world, "steps": 1,
        "warmup": 1, "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded rigid-water clusters (no dataset)",
        "config": {"workload": f"{len(mols)} seeded (H2O)n, n uniform in [2,16] (48-384 functions), "
                               "cc-pVDZ/def2-universal-jkfit, SAD guess, FP64, one graph launch per wave",
                   "clusters": len(mols), "parallelism": f"replicas x{world}",
                   "l2": "per-wave tensors of tens of GB, larger than L2"},
        "converged": int(sum(s == "converged" for s in res.states)),
        "states": {st: int(sum(s == st for s in res.states)) for st in sorted(set(res.states))},
        "not_converged": [{"index": i, "waters": mols[i].n_atoms // 3, "state": res.states[i],
                           "iterations": int(res.iterations[i])}
                          for i in range(len(mols)) if res.states[i] != "converged"][:16],
        "iterations": {"mean": float(np.mean(res.iterations)), "max": int(np.max(res.iterations))},
        "timings": {k: v for k, v in res.timings.items()},
        "scf_only_clusters_per_s": len(mols) / res.timings["run_s"],
        "max_abs_dE_vs_fp64_single_cluster": worst, "clusters_checked_fp64": checked,
        "max_abs_dE_vs_oracle": oracle_worst, "clusters_checked_oracle": len(small),
        "roofline": {"bound": "tensor", "kernel": "batched FP64 exchange (DMMA half-transform + SYRK), whole run",
                     "achieved": k_tflops, "peak": fp64_peak, "unit": "TFLOP/s", "frac": k_tflops / fp64_peak,
                     "traffic": None, "algorithmic": "sum over clusters and Fock builds of 4 naux n^2 nocc",
                     "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run"},
        "clocks": clocks,
        "e2e": {"value": len(mols) / seconds, "unit": "clusters/s",
                "h2d_bytes_per_step": int(sum(m.positions.nbytes for m in mols)),
                "d2h_bytes_per_step": int(8 * len(mols))},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.batched:
        run_batched(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
