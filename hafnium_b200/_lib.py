"""ctypes binding of ``libhfjk.so`` (include/hfjk.h).

The library is built in-tree (``python -m hafnium_b200.build``) and loaded by
path. There is no fallback: if the library or a CUDA device is missing, the
calls raise ``BackendError``.
"""

from __future__ import annotations

import ctypes
import pathlib

import numpy as np

from hafnium_b200.errors import BackendError, InputError

HERE = pathlib.Path(__file__).resolve().parent
LIBRARY = HERE / "_build" / "libhfjk.so"

HF_OK, HF_ERR_ARG, HF_ERR_OOM, HF_ERR_CUDA, HF_ERR_TIMEOUT, HF_ERR_NUMERIC, HF_ERR_STATE = range(7)
PREC_FP64, PREC_BF16X3 = 0, 1

EXPORTS = (
    "hf_ctx_create", "hf_ctx_destroy", "hf_last_error", "hf_set_stream", "hf_shells_upload",
    "hf_build_fitted_tensor", "hf_dims", "hf_coulomb", "hf_exchange", "hf_exchange_factored",
    "hf_metric", "hf_three_center", "hf_fitted_eri", "hf_one_electron", "hf_four_center", "hf_get_stats",
    "hf_coulomb_static", "hf_mp2_energy", "hf_nuclear_gradient", "hf_mo_fitted_tensor", "hf_set_wait_limit",
    "hf_boys", "hf_release_retained", "hf_density_factor", "hf_set_fitted_rows", "hf_exchange_scheduled",
    "hf_schedule_reset",
)

BATCH_EXPORTS = (
    "hf_batch_default_options", "hf_batch_create", "hf_batch_destroy", "hf_batch_last_error", "hf_batch_set_stream",
    "hf_batch_dims", "hf_batch_load", "hf_batch_run", "hf_batch_run_group", "hf_batch_results", "hf_batch_coulomb",
    "hf_batch_exchange", "hf_dgemm_nt",
)


class BatchOptionsC(ctypes.Structure):
    _fields_ = [
        ("max_iterations", ctypes.c_int),
        ("diis_size", ctypes.c_int),
        ("energy_tolerance", ctypes.c_double),
        ("gradient_tolerance", ctypes.c_double),
        ("purify_steps", ctypes.c_int),
        ("purify_tolerance", ctypes.c_double),
        ("gemm_tile", ctypes.c_int),
        ("use_graph", ctypes.c_int),
    ]


class ShellTableC(ctypes.Structure):
    _fields_ = [
        ("n_shells", ctypes.c_int64),
        ("angular_momenta", ctypes.c_void_p),
        ("centers", ctypes.c_void_p),
        ("primitive_offsets", ctypes.c_void_p),
        ("exponents", ctypes.c_void_p),
        ("coefficients", ctypes.c_void_p),
        ("n_contractions", ctypes.c_void_p),
    ]


class ScheduleC(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("anchor_change", ctypes.c_double), ("final_change", ctypes.c_double)]


SCHEDULE_FP64, SCHEDULE_MIXED = 0, 1
BUILD_KINDS = {0: "fp64", 1: "bf16", 2: "anchor", 3: "incremental"}


class StatsC(ctypes.Structure):
    _fields_ = [
        ("ms_metric", ctypes.c_double),
        ("ms_factor", ctypes.c_double),
        ("ms_three_center", ctypes.c_double),
        ("ms_fit", ctypes.c_double),
        ("ms_coulomb", ctypes.c_double),
        ("ms_exchange", ctypes.c_double),
        ("ms_factorize_density", ctypes.c_double),
        ("min_pivot_ratio", ctypes.c_double),
        ("n_ao", ctypes.c_int64),
        ("n_aux", ctypes.c_int64),
        ("n_tiles", ctypes.c_int64),
        ("b_bytes", ctypes.c_int64),
        ("exchange_rank", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64),
        ("ms_gradient_weights", ctypes.c_double),
        ("ms_gradient_metric", ctypes.c_double),
        ("ms_gradient_three_center", ctypes.c_double),
        ("ms_gradient_one_electron", ctypes.c_double),
        ("device_allocations", ctypes.c_int64),
    ]


_lib: ctypes.CDLL | None = None


def load(path: pathlib.Path | str | None = None) -> ctypes.CDLL:
    """Load the library (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    target = pathlib.Path(path) if path else LIBRARY
    if path is None:
        from hafnium_b200 import build

        if build.needs_build():
            try:
                build.build()
            except Exception as error:  # noqa: BLE001
                if not target.exists():
                    raise BackendError(f"libhfjk.so is missing and could not be built: {error}") from error
    if not target.exists():
        raise BackendError(f"libhfjk.so not found at {target}; run python -m hafnium_b200.build")
    lib = ctypes.CDLL(str(target))
    v, p, i64, i = ctypes.c_void_p, ctypes.POINTER, ctypes.c_int64, ctypes.c_int
    lib.hf_ctx_create.argtypes = [i, p(v)]
    lib.hf_ctx_destroy.argtypes = [v]
    lib.hf_last_error.argtypes = [v]
    lib.hf_last_error.restype = ctypes.c_char_p
    lib.hf_set_stream.argtypes = [v, v]
    lib.hf_shells_upload.argtypes = [v, p(ShellTableC), p(ShellTableC)]
    lib.hf_build_fitted_tensor.argtypes = [v]
    lib.hf_dims.argtypes = [v, p(i64), p(i64)]
    lib.hf_coulomb.argtypes = [v, v, v, i]
    lib.hf_exchange.argtypes = [v, v, v, i, i]
    lib.hf_exchange_factored.argtypes = [v, v, i64, v, v, i, i]
    lib.hf_metric.argtypes = [v, v]
    lib.hf_three_center.argtypes = [v, v]
    lib.hf_fitted_eri.argtypes = [v, v]
    lib.hf_one_electron.argtypes = [v, i, v, v, i64, v, i]
    lib.hf_four_center.argtypes = [v, v, i]
    lib.hf_coulomb_static.argtypes = [v, v, v]
    lib.hf_set_wait_limit.argtypes = [v, i64, i]
    lib.hf_boys.argtypes = [v, v, i64, i, v]
    lib.hf_release_retained.argtypes = [i]
    lib.hf_density_factor.argtypes = [v, v, v, i64, p(i64), i]
    lib.hf_set_fitted_rows.argtypes = [v, i64, i64]
    lib.hf_exchange_scheduled.argtypes = [v, v, v, i, p(ScheduleC), p(i)]
    lib.hf_schedule_reset.argtypes = [v]
    lib.hf_mp2_energy.argtypes = [v, v, v, i64, i64, ctypes.POINTER(ctypes.c_double), i]
    lib.hf_nuclear_gradient.argtypes = [v, v, i64, v, v, v, i64, v, i]
    lib.hf_mo_fitted_tensor.argtypes = [v, v, i64, v, i64, v, i]
    lib.hf_get_stats.argtypes = [v, p(StatsC)]
    d = ctypes.c_double
    lib.hf_batch_default_options.argtypes = [p(BatchOptionsC)]
    lib.hf_batch_create.argtypes = [p(v), i, i64, p(v)]
    lib.hf_batch_destroy.argtypes = [v]
    lib.hf_batch_last_error.argtypes = [v]
    lib.hf_batch_set_stream.argtypes = [v, v]
    lib.hf_batch_dims.argtypes = [v, p(i), p(i64), p(i64), p(i64)]
    lib.hf_batch_load.argtypes = [v, v, v, v, v, i64]
    lib.hf_batch_run.argtypes = [v, p(BatchOptionsC)]
    lib.hf_batch_run_group.argtypes = [p(v), i, p(BatchOptionsC)]
    lib.hf_batch_results.argtypes = [v, v, v, v, v]
    lib.hf_batch_coulomb.argtypes = [v, v, d, v]
    lib.hf_batch_exchange.argtypes = [v, v, i64, v]
    lib.hf_dgemm_nt.argtypes = [i64, i64, i64, v, i64, i64, v, i64, i64, v, i64, i64, d, d, i, i, v]
    for name in EXPORTS + BATCH_EXPORTS:
        text = name in ("hf_last_error", "hf_batch_last_error")
        getattr(lib, name).restype = ctypes.c_char_p if text else ctypes.c_int
    _lib = lib
    return lib


def shell_struct(table) -> tuple[ShellTableC, tuple]:
    """A C view of a ShellTable-like object; the tuple keeps the arrays alive."""
    counts = getattr(table, "n_contractions", None)
    if counts is None:
        counts = table.contraction_counts
    arrays = (
        np.ascontiguousarray(table.angular_momenta, dtype=np.int64),
        np.ascontiguousarray(table.centers, dtype=np.float64),
        np.ascontiguousarray(table.primitive_offsets, dtype=np.int64),
        np.ascontiguousarray(table.exponents, dtype=np.float64),
        np.ascontiguousarray(table.coefficients, dtype=np.float64),
        np.ascontiguousarray(counts, dtype=np.int64),
    )
    s = ShellTableC(arrays[0].shape[0], *(a.ctypes.data for a in arrays))
    return s, arrays


def torch_sync(tensor) -> None:
    """Wait for the work torch has queued on ``tensor``'s device (its current stream)."""
    import torch

    torch.cuda.current_stream(tensor.device).synchronize()


def host_empty(shape) -> np.ndarray:
    """An uninitialised FP64 host array in page-locked memory (torch's caching
    pinned-memory allocator, so repeated calls reuse blocks), into which the
    device-to-host copy of a result runs at full bus speed instead of through
    the driver's staging of pageable memory; plain NumPy memory without a GPU."""
    try:
        import torch

        if torch.cuda.is_available():
            return torch.empty(tuple(shape), dtype=torch.float64, pin_memory=True).numpy()
    except (ImportError, RuntimeError):  # pragma: no cover - a GPU process has torch and CUDA
        pass
    return np.empty(tuple(shape))


def to_host(tensor) -> np.ndarray:
    """A device tensor's values as a NumPy array in page-locked memory."""
    out = host_empty(tensor.shape)
    import torch

    torch.from_numpy(out).copy_(tensor)
    return out


def release_retained(device: int = 0) -> None:
    """Free the fitted-tensor blocks the library keeps on ``device`` for the next
    context of the same size (see hf_release_retained in include/hfjk.h)."""
    status = load().hf_release_retained(int(device))
    if status != HF_OK:
        raise InputError(f"hf_release_retained({device}) failed with status {status}")


class Context:
    """One ``hf_ctx``: the device-resident fitted tensor and its J/K builds."""

    def __init__(self, device: int = 0) -> None:
        self.lib = load()
        handle = ctypes.c_void_p()
        status = self.lib.hf_ctx_create(int(device), ctypes.byref(handle))
        if status != HF_OK:
            raise BackendError(f"hf_ctx_create failed with status {status} (no usable CUDA device {device}?)")
        self.handle = handle
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.hf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order varies
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def check(self, status: int, what: str) -> None:
        if status == HF_OK:
            return
        message = (self.lib.hf_last_error(self.handle) or b"").decode()
        text = f"{what}: {message}" if message else f"{what} failed with status {status}"
        if status in (HF_ERR_ARG, HF_ERR_NUMERIC, HF_ERR_STATE):
            raise InputError(text)
        raise BackendError(text)

    def set_stream(self, stream_handle: int | None) -> None:
        self.check(self.lib.hf_set_stream(self.handle, stream_handle or None), "hf_set_stream")

    def upload(self, orbital, auxiliary=None) -> None:
        o, keep_o = shell_struct(orbital)
        if auxiliary is None:
            self.check(self.lib.hf_shells_upload(self.handle, ctypes.byref(o), None), "hf_shells_upload")
            return
        a, keep_a = shell_struct(auxiliary)
        self.check(self.lib.hf_shells_upload(self.handle, ctypes.byref(o), ctypes.byref(a)), "hf_shells_upload")
        del keep_o, keep_a

    def set_fitted_rows(self, row0: int, row1: int) -> None:
        """Hold only rows [row0, row1) of the fitted tensor (a shard by auxiliary index)."""
        self.check(self.lib.hf_set_fitted_rows(self.handle, int(row0), int(row1)), "hf_set_fitted_rows")

    def build(self) -> None:
        """The fitted tensor on the device. When the device is out of memory, the
        contexts Python no longer references are collected (their tensors freed)
        and torch's cached blocks released before one more attempt."""
        status = self.lib.hf_build_fitted_tensor(self.handle)
        if status == HF_ERR_OOM:
            import gc

            gc.collect()
            try:
                import torch

                if torch.cuda.is_available():
                    torch.cuda.empty_cache()
            except ImportError:  # pragma: no cover - torch is a dependency of the device path
                pass
            status = self.lib.hf_build_fitted_tensor(self.handle)
        self.check(status, "hf_build_fitted_tensor")

    def dims(self) -> tuple[int, int]:
        n, naux = ctypes.c_int64(), ctypes.c_int64()
        self.check(self.lib.hf_dims(self.handle, ctypes.byref(n), ctypes.byref(naux)), "hf_dims")
        return int(n.value), int(naux.value)

    def stats(self) -> dict:
        s = StatsC()
        self.check(self.lib.hf_get_stats(self.handle, ctypes.byref(s)), "hf_get_stats")
        return {name: getattr(s, name) for name, _ in StatsC._fields_}

    # -- host-array entry points (numpy in, numpy out) ---------------------
    def coulomb_host(self, d: np.ndarray) -> np.ndarray:
        d = np.ascontiguousarray(d, dtype=np.float64)
        out = host_empty(d.shape)
        self.check(self.lib.hf_coulomb(self.handle, d.ctypes.data, out.ctypes.data, 0), "hf_coulomb")
        return out

    def exchange_host(self, d: np.ndarray, precision: int = PREC_FP64) -> np.ndarray:
        d = np.ascontiguousarray(d, dtype=np.float64)
        out = host_empty(d.shape)
        self.check(self.lib.hf_exchange(self.handle, d.ctypes.data, out.ctypes.data, precision, 0), "hf_exchange")
        return out

    def exchange_factored_host(self, c: np.ndarray, weights=None, precision: int = PREC_FP64) -> np.ndarray:  # noqa: E501
        c = np.ascontiguousarray(c, dtype=np.float64)
        n = c.shape[0]
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        out = host_empty((n, n))
        self.check(
            self.lib.hf_exchange_factored(
                self.handle, c.ctypes.data, c.shape[1], None if w is None else w.ctypes.data, out.ctypes.data,
                precision, 0,
            ),
            "hf_exchange_factored",
        )
        return out

    # -- device entry points (torch CUDA tensors) ---------------------------
    # The library works on its own stream and synchronises it before returning;
    # torch's stream is synchronised first, so inputs written by torch kernels
    # are complete and no memory torch recycles is still in use.
    def coulomb_device(self, d, out) -> None:
        torch_sync(d)
        self.check(self.lib.hf_coulomb(self.handle, d.data_ptr(), out.data_ptr(), 1), "hf_coulomb")

    def boys(self, t, n_max: int) -> np.ndarray:
        """F_0..F_n_max at each argument in ``t`` from the device evaluation:
        ``[len(t), n_max + 1]``."""
        t = np.ascontiguousarray(np.atleast_1d(np.asarray(t, dtype=np.float64)))
        out = np.empty((t.shape[0], n_max + 1))
        self.check(self.lib.hf_boys(self.handle, t.ctypes.data, t.shape[0], int(n_max), out.ctypes.data), "hf_boys")
        return out

    def set_wait_limit(self, seconds: float, stall_next_build: bool = False) -> None:
        """Limit of the split-BF16 exchange's device waits; ``stall_next_build``
        makes the next split-BF16 build wait once on a barrier that nothing
        completes (it then returns HF_ERR_TIMEOUT, raised as BackendError)."""
        self.check(self.lib.hf_set_wait_limit(self.handle, int(round(seconds * 1e9)), int(stall_next_build)),
                   "hf_set_wait_limit")

    def coulomb_static_device(self, d, out) -> None:
        """J into ``out`` through hf_coulomb_static, the build that allocates no
        device memory (its scratch is a static device array). Torch's pending
        work on ``d`` and ``out`` is waited for first: the library runs on its
        own stream."""
        torch_sync(d)
        torch_sync(out)
        self.check(self.lib.hf_coulomb_static(self.handle, d.data_ptr(), out.data_ptr()), "hf_coulomb_static")

    def overlap_device(self):
        """The orbital overlap matrix S as a torch CUDA tensor (hf_one_electron)."""
        import torch

        n, _ = self.dims()
        s = torch.empty((n, n), dtype=torch.float64, device=torch.device("cuda", self.device))
        torch_sync(s)
        self.check(self.lib.hf_one_electron(self.handle, 0, None, None, 0, s.data_ptr(), 1), "hf_one_electron")
        return s

    def exchange_scheduled(self, d, out, schedule: "ScheduleC") -> str:
        """K of ``d`` into ``out`` through hf_exchange_scheduled (torch CUDA tensors,
        or host NumPy arrays); returns the arithmetic the schedule chose."""
        kind = ctypes.c_int(-1)
        if hasattr(d, "data_ptr"):
            torch_sync(d)
            status = self.lib.hf_exchange_scheduled(self.handle, d.data_ptr(), out.data_ptr(), 1,
                                                    ctypes.byref(schedule), ctypes.byref(kind))
        else:
            status = self.lib.hf_exchange_scheduled(self.handle, d.ctypes.data, out.ctypes.data, 0,
                                                    ctypes.byref(schedule), ctypes.byref(kind))
        self.check(status, "hf_exchange_scheduled")
        return BUILD_KINDS.get(kind.value, str(kind.value))

    def schedule_reset(self) -> None:
        self.check(self.lib.hf_schedule_reset(self.handle), "hf_schedule_reset")

    def density_factor_device(self, d, max_rank: int):
        """``F`` ([n_ao, rank], a torch CUDA tensor) with ``F F^T = D`` for a
        positive semidefinite device density, by the library's pivoted Cholesky."""
        import torch

        torch_sync(d)
        n = d.shape[0]
        rows = torch.empty((max(1, min(int(max_rank), n)), n), dtype=torch.float64, device=d.device)
        rank = ctypes.c_int64()
        self.check(self.lib.hf_density_factor(self.handle, d.data_ptr(), rows.data_ptr(), rows.shape[0],
                                              ctypes.byref(rank), 1), "hf_density_factor")
        return rows[: rank.value].T.contiguous()

    def exchange_device(self, d, out, precision: int = PREC_FP64) -> None:
        torch_sync(d)
        self.check(self.lib.hf_exchange(self.handle, d.data_ptr(), out.data_ptr(), precision, 1), "hf_exchange")

    def exchange_factored_device(self, c, out, weights=None, precision: int = PREC_FP64) -> None:
        torch_sync(c)
        self.check(
            self.lib.hf_exchange_factored(
                self.handle, c.data_ptr(), c.shape[1], None if weights is None else weights.data_ptr(),
                out.data_ptr(), precision, 1,
            ),
            "hf_exchange_factored",
        )

    def mp2_energy(self, mo_coefficients, mo_energies, n_occ: int) -> float:
        """DF-MP2 correlation energy (torch CUDA tensors or NumPy arrays)."""
        out = ctypes.c_double()
        if hasattr(mo_coefficients, "data_ptr"):
            c = mo_coefficients.contiguous()
            e = mo_energies.contiguous()
            torch_sync(c)
            status = self.lib.hf_mp2_energy(self.handle, c.data_ptr(), e.data_ptr(), c.shape[1], int(n_occ),
                                            ctypes.byref(out), 1)
        else:
            c = np.ascontiguousarray(mo_coefficients, dtype=np.float64)
            e = np.ascontiguousarray(mo_energies, dtype=np.float64)
            status = self.lib.hf_mp2_energy(self.handle, c.ctypes.data, e.ctypes.data, c.shape[1], int(n_occ),
                                            ctypes.byref(out), 0)
        self.check(status, "hf_mp2_energy")
        return float(out.value)

    def mo_fitted_tensor(self, c_bra, c_ket):
        """B[P, p, q] in an orbital basis, [aux, n_bra, n_ket] (torch CUDA tensors in,
        a torch CUDA tensor out; or NumPy in and out)."""
        _, naux = self.dims()
        if hasattr(c_bra, "data_ptr"):
            import torch

            cb = c_bra.contiguous()
            ck = c_ket.contiguous()
            out = torch.empty((naux, cb.shape[1], ck.shape[1]), dtype=torch.float64, device=cb.device)
            torch_sync(cb)
            torch_sync(ck)
            status = self.lib.hf_mo_fitted_tensor(self.handle, cb.data_ptr(), cb.shape[1], ck.data_ptr(), ck.shape[1],
                                                  out.data_ptr(), 1)
        else:
            cb = np.ascontiguousarray(c_bra, dtype=np.float64)
            ck = np.ascontiguousarray(c_ket, dtype=np.float64)
            out = np.empty((naux, cb.shape[1], ck.shape[1]))
            status = self.lib.hf_mo_fitted_tensor(self.handle, cb.ctypes.data, cb.shape[1], ck.ctypes.data, ck.shape[1],
                                                  out.ctypes.data, 0)
        self.check(status, "hf_mo_fitted_tensor")
        return out

    def nuclear_gradient(self, occupied, weighted, charges, positions) -> np.ndarray:
        """The five DF-RHF gradient terms [5, atom, 3] (torch CUDA tensors or NumPy
        arrays for the occupied orbitals and the energy-weighted density)."""
        q = np.ascontiguousarray(charges, dtype=np.float64)
        r = np.ascontiguousarray(positions, dtype=np.float64)
        out = np.empty((5, q.shape[0], 3))
        if hasattr(occupied, "data_ptr"):
            c = occupied.contiguous()
            w = weighted.contiguous()
            torch_sync(c)
            torch_sync(w)
            status = self.lib.hf_nuclear_gradient(self.handle, c.data_ptr(), c.shape[1], w.data_ptr(), q.ctypes.data,
                                                  r.ctypes.data, q.shape[0], out.ctypes.data, 0)
        else:
            c = np.ascontiguousarray(occupied, dtype=np.float64)
            w = np.ascontiguousarray(weighted, dtype=np.float64)
            status = self.lib.hf_nuclear_gradient(self.handle, c.ctypes.data, c.shape[1], w.ctypes.data, q.ctypes.data,
                                                  r.ctypes.data, q.shape[0], out.ctypes.data, 0)
        self.check(status, "hf_nuclear_gradient")
        return out

    # -- inspection ----------------------------------------------------------
    def metric(self) -> np.ndarray:
        _, naux = self.dims()
        out = np.empty((naux, naux))
        self.check(self.lib.hf_metric(self.handle, out.ctypes.data), "hf_metric")
        return out

    def three_center(self) -> np.ndarray:
        n, naux = self.dims()
        out = np.empty((naux, n, n))
        self.check(self.lib.hf_three_center(self.handle, out.ctypes.data), "hf_three_center")
        return out

    def fitted_eri(self) -> np.ndarray:
        n, _ = self.dims()
        out = np.empty((n, n, n, n))
        self.check(self.lib.hf_fitted_eri(self.handle, out.ctypes.data), "hf_fitted_eri")
        return out

    def four_center(self) -> np.ndarray:
        n, _ = self.dims()
        out = np.empty((n, n, n, n))
        self.check(self.lib.hf_four_center(self.handle, out.ctypes.data, 0), "hf_four_center")
        return out

    def one_electron(self, kind: int, charges=None, positions=None) -> np.ndarray:
        n, _ = self.dims()
        out = np.empty((n, n))
        q = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        r = None if positions is None else np.ascontiguousarray(positions, dtype=np.float64)
        natoms = 0 if q is None else q.shape[0]
        self.check(
            self.lib.hf_one_electron(
                self.handle, int(kind), None if q is None else q.ctypes.data, None if r is None else r.ctypes.data,
                natoms, out.ctypes.data, 0,
            ),
            "hf_one_electron",
        )
        return out
