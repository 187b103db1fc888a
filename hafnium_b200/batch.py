"""Batched DF-RHF over many clusters: one CUDA graph per wave of clusters.

``solve_batch`` converges the restricted SCF of many molecules at once through
the ``hf_batch_*`` C ABI (include/hfbatch.h). Clusters are grouped by shape
(orbital count, auxiliary count, occupied count); each group is one batch, and
all batches of a wave run in one graph launch whose loop over SCF iterations is
a device-side conditional node. A wave holds as many clusters as the device
memory budget admits.

Each cluster follows the reference driver (hafnium/scf/driver.py:154-213,
331-366) from the SAD guess (hafnium/scf/atoms.py:76-120); the differences the
batched form makes are stated in include/hfbatch.h (Cholesky orthonormal basis,
aufbau density by purification).

The DMMA tile shape of the n x n products is chosen per shape by ``TileTuner``,
which times every tile on the batch's own problem size.
"""

from __future__ import annotations

import ctypes
import json
import os
import time
from dataclasses import dataclass, field

import numpy as np

from hafnium_b200 import _lib
from hafnium_b200.basis import ShellTable
from hafnium_b200.errors import BackendError, ConvergenceError, InputError

# CTA tiles of hf_dgemm_nt: 0-4 with 3 stages of 16-wide k slices, 5 with 2 stages of 32
TILE_SHAPES = ((128, 64), (64, 64), (64, 32), (32, 32), (128, 128), (64, 64))
STATE_NAMES = {0: "iterating", 1: "finishing", 2: "converged", 3: "not_converged", 4: "purification_failed"}


def _torch():
    import torch

    return torch


@dataclass
class BatchOptions:
    max_iterations: int = 100
    diis_size: int = 8
    energy_tolerance: float = 1e-10
    gradient_tolerance: float = 1e-6
    purify_steps: int = 64
    purify_tolerance: float = 1e-9
    gemm_tile: int | None = None  # None: chosen by the tile tuner
    use_graph: bool = True

    def to_c(self, tile: int) -> _lib.BatchOptionsC:
        return _lib.BatchOptionsC(self.max_iterations, self.diis_size, self.energy_tolerance,
                                  self.gradient_tolerance, self.purify_steps, self.purify_tolerance, int(tile),
                                  1 if self.use_graph else 0)


@dataclass
class BatchResult:
    energies: np.ndarray
    iterations: np.ndarray
    states: list
    seconds: float
    timings: dict = field(default_factory=dict)
    densities: list | None = None  # per-spin densities (host), when requested

    @property
    def converged(self) -> np.ndarray:
        return np.array([s == "converged" for s in self.states])


class Batch:
    """One ``hf_batch``: clusters of one shape sharing a graph-resident SCF."""

    def __init__(self, contexts, n_occ: int) -> None:
        self.lib = _lib.load()
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c.handle.value for c in self.contexts])
        handle = ctypes.c_void_p()
        status = self.lib.hf_batch_create(arr, len(self.contexts), int(n_occ), ctypes.byref(handle))
        if status != _lib.HF_OK:
            raise (InputError if status in (_lib.HF_ERR_ARG, _lib.HF_ERR_STATE) else BackendError)(
                f"hf_batch_create failed with status {status}")
        self.handle = handle
        count, n, naux, nocc = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self.lib.hf_batch_dims(handle, ctypes.byref(count), ctypes.byref(n), ctypes.byref(naux), ctypes.byref(nocc))
        self.count, self.n, self.naux, self.nocc = count.value, n.value, naux.value, nocc.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.hf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:  # pragma: no cover
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def check(self, status: int, what: str) -> None:
        if status == _lib.HF_OK:
            return
        message = (self.lib.hf_batch_last_error(self.handle) or b"").decode()
        text = f"{what}: {message}" if message else f"{what} failed with status {status}"
        if status in (_lib.HF_ERR_ARG, _lib.HF_ERR_NUMERIC, _lib.HF_ERR_STATE):
            raise InputError(text)
        raise BackendError(text)

    def set_stream(self, stream_handle: int | None) -> None:
        self.check(self.lib.hf_batch_set_stream(self.handle, stream_handle or None), "hf_batch_set_stream")

    def load(self, overlap, core, guess, nuclear_repulsion, guess_rank: int) -> None:
        """overlap, core, guess: CUDA float64 tensors [count, n, n]."""
        e = np.ascontiguousarray(nuclear_repulsion, dtype=np.float64)
        for t in (overlap, core, guess):
            if tuple(t.shape) != (self.count, self.n, self.n) or not t.is_contiguous():
                raise InputError(f"expected a contiguous [{self.count}, {self.n}, {self.n}] tensor")
        _torch().cuda.synchronize(overlap.device)  # the batch reads them on its own stream
        self.check(self.lib.hf_batch_load(self.handle, overlap.data_ptr(), core.data_ptr(), guess.data_ptr(),
                                          e.ctypes.data, int(guess_rank)), "hf_batch_load")

    def run(self, options: BatchOptions, tile: int) -> None:
        opts = options.to_c(tile)
        self.check(self.lib.hf_batch_run(self.handle, ctypes.byref(opts)), "hf_batch_run")

    def results(self, densities=None):
        if densities is not None:
            _torch().cuda.synchronize(densities.device)  # the copy runs on the batch's stream
        e = np.empty(self.count)
        it = np.empty(self.count, dtype=np.int32)
        st = np.empty(self.count, dtype=np.int32)
        self.check(self.lib.hf_batch_results(self.handle, e.ctypes.data, it.ctypes.data, st.ctypes.data,
                                             None if densities is None else densities.data_ptr()),
                   "hf_batch_results")
        return e, it, [STATE_NAMES.get(int(s), str(int(s))) for s in st]

    def coulomb(self, density, scale: float = 1.0):
        out = _torch().empty_like(density)
        _torch().cuda.synchronize(density.device)
        self.check(self.lib.hf_batch_coulomb(self.handle, density.data_ptr(), float(scale), out.data_ptr()),
                   "hf_batch_coulomb")
        return out

    def exchange(self, density, max_rank: int):
        out = _torch().empty_like(density)
        _torch().cuda.synchronize(density.device)
        self.check(self.lib.hf_batch_exchange(self.handle, density.data_ptr(), int(max_rank), out.data_ptr()),
                   "hf_batch_exchange")
        return out


def run_group(batches, options: BatchOptions, tile: int) -> None:
    """Every batch converged in one graph launch."""
    lib = _lib.load()
    arr = (ctypes.c_void_p * len(batches))(*[b.handle.value for b in batches])
    opts = options.to_c(tile)
    status = lib.hf_batch_run_group(arr, len(batches), ctypes.byref(opts))
    if status != _lib.HF_OK:
        batches[0].check(status, "hf_batch_run_group")


def dgemm_nt(a, b, c, *, alpha: float = 1.0, beta: float = 0.0, tile: int = 0, stream=None) -> None:
    """c = alpha a b^T + beta c on the DMMA kernel; a [batch, m, k], b [batch, n, k], c [batch, m, n]."""
    lib = _lib.load()
    batch, m, k = a.shape
    n = b.shape[1]
    status = lib.hf_dgemm_nt(m, n, k, a.data_ptr(), k, m * k, b.data_ptr(), k, n * k, c.data_ptr(), n, m * n,
                             float(alpha), float(beta), batch, int(tile), stream)
    if status != _lib.HF_OK:
        raise BackendError(f"hf_dgemm_nt failed with status {status}")


class TileTuner:
    """Chooses the DMMA tile shape for batched n x n products by timing each
    shape on the problem itself (CUDA events, after a warm-up). Choices are kept
    per (device name, n, batch) in memory and, when ``path`` is given, in a JSON
    file."""

    def __init__(self, path: str | None = None, repeats: int = 5) -> None:
        self.path = path or os.environ.get("HAFNIUM_B200_TILE_CACHE")
        self.repeats = repeats
        self.choices: dict[str, dict] = {}
        if self.path and os.path.exists(self.path):
            with open(self.path) as f:
                self.choices = json.load(f)

    def choose(self, n: int, batch: int, device: int = 0) -> int:
        torch = _torch()
        key = f"{torch.cuda.get_device_name(device)}|{n}|{batch}"
        if key in self.choices:
            return int(self.choices[key]["tile"])
        dev = torch.device("cuda", device)
        gen = torch.Generator(device=dev).manual_seed(n)
        a = torch.rand((batch, n, n), dtype=torch.float64, device=dev, generator=gen)
        c = torch.empty_like(a)
        times = []
        for tile in range(len(TILE_SHAPES)):
            dgemm_nt(a, a, c, tile=tile)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.repeats):
                dgemm_nt(a, a, c, tile=tile)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / self.repeats)
        best = int(np.argmin(times))
        self.choices[key] = {"tile": best, "shape": list(TILE_SHAPES[best]), "ms": times}
        if self.path:
            with open(self.path, "w") as f:
                json.dump(self.choices, f, indent=1)
        return best


_DEFAULT_TUNER: TileTuner | None = None


def default_tuner() -> TileTuner:
    global _DEFAULT_TUNER
    if _DEFAULT_TUNER is None:
        _DEFAULT_TUNER = TileTuner()
    return _DEFAULT_TUNER


# ----------------------------------------------------------------- clusters
class _Atoms:
    """SAD blocks per element (hafnium/scf/atoms.py:55-120), converged once."""

    def __init__(self, basis: str, device: int) -> None:
        self.basis, self.device = basis, device
        self.blocks: dict[str, object] = {}
        self.ranks: dict[str, int] = {}

    def block(self, symbol: str):
        if symbol not in self.blocks:
            from hafnium_b200.scf import atomic_block

            d = atomic_block(symbol, self.basis, self.device)
            w = _torch().linalg.eigvalsh(0.5 * (d + d.T))
            self.blocks[symbol] = d
            self.ranks[symbol] = int((w > 1e-14 * float(w.abs().max())).sum())
        return self.blocks[symbol]

    def guess(self, molecule):
        torch = _torch()
        return torch.block_diag(*[self.block(s) for s in molecule.symbols])

    def rank(self, molecule) -> int:
        for s in molecule.symbols:
            self.block(s)
        return sum(self.ranks[s] for s in molecule.symbols)


def _cluster(molecule, basis: str, auxiliary: str, device: int, tables=None):
    """(context with B built, S, H) for one molecule; ``tables`` = (orbital,
    auxiliary) shell tables when the caller has them already."""
    torch = _torch()
    if tables is None:
        tables = (ShellTable.build(basis, molecule.symbols, molecule.positions),
                  ShellTable.build(auxiliary, molecule.symbols, molecule.positions))
    orb, aux = tables
    ctx = _lib.Context(device)
    ctx.upload(orb, aux)
    dev = torch.device("cuda", device)
    n = orb.n_functions
    s = torch.empty((n, n), dtype=torch.float64, device=dev)
    t = torch.empty_like(s)
    v = torch.empty_like(s)
    q = torch.as_tensor(molecule.nuclear_charges, dtype=torch.float64, device=dev)
    r = torch.as_tensor(np.ascontiguousarray(molecule.positions), dtype=torch.float64, device=dev)
    _lib.torch_sync(s)
    for kind, out in ((0, s), (1, t), (2, v)):
        ctx.check(ctx.lib.hf_one_electron(ctx.handle, kind, q.data_ptr() if kind == 2 else None,
                                          r.data_ptr() if kind == 2 else None, q.shape[0] if kind == 2 else 0,
                                          out.data_ptr(), 1), "hf_one_electron")
    ctx.build()
    return ctx, s, t + v


def _b_bytes(n: int, naux: int) -> int:
    nt = (n + 63) // 64
    return naux * nt * (nt + 1) // 2 * 4096 * 8


def _cluster_state_bytes(n: int) -> int:
    """Device bytes of one cluster's batch state (matrices, DIIS rings, K scratch)."""
    npad = (n + 63) // 64 * 64
    return (34 * n * n + 2 * npad * npad) * 8


BATCH_FIXED_BYTES = 2 << 30  # the K chunk buffer of one batch


def solve_batch(molecules, basis: str = "cc-pvdz", auxiliary: str = "def2-universal-jkfit", *, device: int = 0,
                options: BatchOptions | None = None, tuner: TileTuner | None = None,
                memory_fraction: float = 0.6, max_batch: int = 256, keep_densities: bool = False,
                setup_threads: int = 16, retry_failed: bool = True) -> BatchResult:
    """Converge every molecule's restricted DF-RHF; energies (and, with
    ``keep_densities``, the converged per-spin densities) in input order."""
    torch = _torch()
    _lib.load()  # before any worker thread touches the library
    options = options or BatchOptions()
    tuner = tuner or default_tuner()
    dev = torch.device("cuda", device)
    t_start = time.perf_counter()
    atoms = _Atoms(basis, device)
    shapes: dict[tuple, list[int]] = {}
    tables: dict[int, tuple] = {}
    for i, mol in enumerate(molecules):
        tables[i] = (ShellTable.build(basis, mol.symbols, mol.positions),
                     ShellTable.build(auxiliary, mol.symbols, mol.positions))
        orb_n, aux_n = tables[i][0].n_functions, tables[i][1].n_functions
        if 2 * int(mol.n_alpha) != mol.n_electrons:
            raise InputError("the batched SCF is restricted: every molecule needs an even electron count")
        shapes.setdefault((orb_n, aux_n, int(mol.n_alpha)), []).append(i)
    energies = np.full(len(molecules), np.nan)
    iterations = np.zeros(len(molecules), dtype=np.int32)
    states = ["not_run"] * len(molecules)
    densities = [None] * len(molecules) if keep_densities else None
    timings = {"tables_s": time.perf_counter() - t_start, "setup_s": 0.0, "run_s": 0.0, "results_s": 0.0,
               "waves": 0, "tiles": {}}
    # waves: groups in order of size, split to fit the memory budget
    pending = []
    for key in sorted(shapes):
        idx = shapes[key]
        for k in range(0, len(idx), max_batch):
            pending.append((key, idx[k:k + max_batch]))
    free, _ = torch.cuda.mem_get_info(dev)
    budget = memory_fraction * free
    from concurrent.futures import ThreadPoolExecutor

    pool = ThreadPoolExecutor(max_workers=setup_threads)
    while pending:
        wave, used = [], 0.0
        while pending:
            (n, naux, nocc), idx = pending[0]
            per = _b_bytes(n, naux) + _cluster_state_bytes(n)
            fit = int(max(0, (budget - used - BATCH_FIXED_BYTES) // per))
            if fit <= 0 and wave:
                break
            take = max(1, min(len(idx), fit))
            wave.append(((n, naux, nocc), idx[:take]))
            used += take * per + BATCH_FIXED_BYTES
            if take < len(idx):
                pending[0] = ((n, naux, nocc), idx[take:])
                break
            pending.pop(0)
        t0 = time.perf_counter()
        batches, keep = [], []
        for (n, naux, nocc), idx in wave:
            # each cluster's integrals and fitted tensor on its own stream, several at once
            clusters = list(pool.map(lambda i: _cluster(molecules[i], basis, auxiliary, device, tables.pop(i)), idx))
            ctxs = [c[0] for c in clusters]
            s = torch.stack([c[1] for c in clusters]).contiguous()
            h = torch.stack([c[2] for c in clusters]).contiguous()
            guess = torch.stack([atoms.guess(molecules[i]) for i in idx]).contiguous()
            rank = max(atoms.rank(molecules[i]) for i in idx)
            e_nuc = np.array([molecules[i].nuclear_repulsion_energy() for i in idx])
            b = Batch(ctxs, nocc)
            b.load(s, h, guess, e_nuc, rank)
            tile = options.gemm_tile if options.gemm_tile is not None else tuner.choose(n, len(idx), device)
            timings["tiles"][str(n)] = list(TILE_SHAPES[tile])
            batches.append((b, idx, tile))
            keep.append((ctxs, s, h, guess))
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        # one graph launch per wave; batches whose tuned tiles differ run as separate groups
        by_tile: dict[int, list] = {}
        for b, idx, tile in batches:
            by_tile.setdefault(tile, []).append(b)
        for tile, group in by_tile.items():
            run_group(group, options, tile)
        torch.cuda.synchronize(dev)
        t2 = time.perf_counter()
        for b, idx, _ in batches:
            dens = torch.empty((b.count, b.n, b.n), dtype=torch.float64, device=dev) if keep_densities else None
            e, it, st = b.results(dens)
            for j, i in enumerate(idx):
                energies[i], iterations[i], states[i] = e[j], it[j], st[j]
                if keep_densities:
                    densities[i] = dens[j].cpu().numpy()
            b.close()
        for ctxs, *_ in keep:
            for c in ctxs:
                c.close()
        del keep, batches
        t3 = time.perf_counter()
        if retry_failed:
            # a cluster the batch could not converge (no gap for purification, or
            # the iteration limit) goes through the per-cluster driver instead
            from hafnium_b200.scf import DeviceHamiltonian, ScfOptions, atomic_density_guess, solve_rhf

            for _, idx in wave:
                for i in idx:
                    if states[i] == "converged":
                        continue
                    mol = molecules[i]
                    ham = DeviceHamiltonian.build(mol, basis, auxiliary, device=device)
                    try:
                        res = solve_rhf(ham, guess=atomic_density_guess(mol, basis, device=device),
                                        options=ScfOptions(max_iterations=options.max_iterations,
                                                           energy_tolerance=options.energy_tolerance,
                                                           gradient_tolerance=options.gradient_tolerance,
                                                           diis_size=options.diis_size))
                    except ConvergenceError as error:
                        res = getattr(error, "last", None)
                    if res is None:
                        continue
                    energies[i], iterations[i] = res.energy, res.n_iterations
                    timings.setdefault("retried", []).append({"index": i, "batch_state": states[i]})
                    states[i] = "converged" if res.converged else "not_converged"
                    if keep_densities:
                        densities[i] = res.density.cpu().numpy()
                    del ham
        timings["setup_s"] += t1 - t0
        timings["run_s"] += t2 - t1
        timings["results_s"] += t3 - t2
        timings["waves"] += 1
    pool.shutdown()
    return BatchResult(energies, iterations, states, time.perf_counter() - t_start, timings, densities)
