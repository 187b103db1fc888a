"""Oracle stand-in for the reference's compiled ``hafnium._kernels`` module.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker, never by the product.

The reference builds ``hafnium._kernels`` from Rust (crates/hafnium-py/src/lib.rs)
and no Rust toolchain exists here. This module exposes the subset of that
module's API the molecular DF-RHF path touches, with the same names, argument
meaning, output shapes and error behaviour (``ValueError`` for invalid input,
lib.rs:1118), computed by ``oracle/md_oracle.cpp`` through ctypes:

- ``kernel_version``, ``dot``, ``boys_function``, ``spherical_transformation``
  (lib.rs:17-61)
- ``ShellTable`` with the validation of integrals/mod.rs:111-173 (lib.rs:66-108)
- ``overlap``, ``kinetic``, ``nuclear_attraction`` (lib.rs:111-186)
- ``coulomb_two_center``, ``coulomb_three_center`` (lib.rs:352-423)
- ``coulomb_four_center``, ``schwarz_bounds`` (lib.rs:503-562)
- ``overlap_derivative``, ``kinetic_derivative``, ``nuclear_attraction_derivative``,
  ``coulomb_two_center_derivative``, ``coulomb_three_center_derivative``
  (hafnium/_kernels.pyi:71-140; two_electron.rs:132-394)
- ``configure_threads`` (lib.rs:1110; integrals/mod.rs:43-49)
"""

from __future__ import annotations

import ctypes
import pathlib

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libmd_oracle.so"
_lib: ctypes.CDLL | None = None


class _Shells(ctypes.Structure):
    _fields_ = [
        ("n_shells", ctypes.c_int64),
        ("angular_momenta", ctypes.c_void_p),
        ("centers", ctypes.c_void_p),
        ("primitive_offsets", ctypes.c_void_p),
        ("exponents", ctypes.c_void_p),
        ("coefficients", ctypes.c_void_p),
        ("n_contractions", ctypes.c_void_p),
    ]


def library() -> ctypes.CDLL:
    """Load (building on first use if needed) the oracle's shared library."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            import subprocess

            subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
        lib = ctypes.CDLL(str(_LIB_PATH))
        p = ctypes.POINTER(_Shells)
        d = ctypes.c_void_p
        i64 = ctypes.c_int64
        lib.md_boys.argtypes = [ctypes.c_int, ctypes.c_double, d]
        lib.md_spherical_transformation.argtypes = [ctypes.c_int, d]
        lib.md_overlap.argtypes = [p, p, i64, d, d]
        lib.md_kinetic.argtypes = [p, p, i64, d, d]
        lib.md_nuclear_attraction.argtypes = [p, p, i64, d, i64, d, d, ctypes.c_int, ctypes.c_double, d]
        lib.md_coulomb_two_center.argtypes = [p, p, i64, d, ctypes.c_int, ctypes.c_double, d]
        lib.md_coulomb_three_center.argtypes = [p, p, p, i64, d, ctypes.c_int, ctypes.c_double, d]
        lib.md_coulomb_four_center.argtypes = [p, p, p, p, i64, d, ctypes.c_int, ctypes.c_double, ctypes.c_double, d]
        lib.md_schwarz_bounds.argtypes = [p, p, i64, d, ctypes.c_int, ctypes.c_double, d]
        lib.md_overlap_derivative.argtypes = [p, p, i64, d, d]
        lib.md_kinetic_derivative.argtypes = [p, p, i64, d, d]
        lib.md_nuclear_attraction_derivative.argtypes = [p, p, i64, d, i64, d, d, ctypes.c_int, ctypes.c_double, d, d]
        lib.md_coulomb_two_center_derivative.argtypes = [p, p, i64, d, ctypes.c_int, ctypes.c_double, d]
        lib.md_coulomb_three_center_derivative.argtypes = [p, p, p, i64, d, ctypes.c_int, ctypes.c_double, d]
        lib.md_set_threads.argtypes = [ctypes.c_int]
        lib.md_get_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def kernel_version() -> str:
    """Version string of the kernel provider (the oracle restatement)."""
    return "0.0.1"


def dot(a, b) -> float:
    """Dot product of two contiguous one-dimensional float64 arrays (lib.rs:26-35)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype != np.float64 or b.dtype != np.float64:
        raise TypeError("float64 arrays expected")
    if not (a.flags.c_contiguous and b.flags.c_contiguous):
        raise TypeError("the arrays must be contiguous")
    if a.shape != b.shape:
        raise ValueError(f"length mismatch: {a.shape[0]} and {b.shape[0]}")
    return float(np.dot(a, b))


def boys_function(n_max: int, t: float) -> np.ndarray:
    """``F_n(t)`` for ``n = 0..n_max`` (special.rs:34-51)."""
    if not (t >= 0.0):
        raise ValueError("the Boys function argument is non-negative")
    out = np.empty(n_max + 1)
    library().md_boys(int(n_max), float(t), _ptr(out))
    return out


def spherical_transformation(l: int) -> np.ndarray:
    """Cartesian-to-solid-harmonic matrix ``[2l + 1, n_cartesian]`` (cartesian.rs:93-110)."""
    if l < 0 or l > 16:
        raise ValueError("angular momentum exceeds the supported maximum")
    out = np.empty((2 * l + 1, (l + 1) * (l + 2) // 2))
    library().md_spherical_transformation(int(l), _ptr(out))
    return out


_MAX_L = 8  # the oracle library's per-shell limit (the reference allows 16)


class ShellTable:
    """Contracted shells in structure-of-arrays form (integrals/mod.rs:63-173)."""

    def __init__(self, angular_momenta, centers, primitive_offsets, exponents, coefficients, n_contractions):
        l = np.ascontiguousarray(angular_momenta, dtype=np.int64)
        c = np.ascontiguousarray(centers, dtype=np.float64)
        off = np.ascontiguousarray(primitive_offsets, dtype=np.int64)
        e = np.ascontiguousarray(exponents, dtype=np.float64)
        k = np.ascontiguousarray(n_contractions, dtype=np.int64)
        co = np.ascontiguousarray(coefficients, dtype=np.float64)
        n = l.shape[0]
        if np.any(l < 0) or np.any(off < 0) or np.any(k < 0):
            raise ValueError("angular momenta are non-negative integers")
        if c.ndim != 2 or c.shape != (n, 3):
            raise ValueError("invalid shell table: one centre per shell")
        if off.shape != (n + 1,) or off[0] != 0:
            raise ValueError("invalid shell table: primitive offsets start at zero and have one entry per shell plus one")
        if np.any(np.diff(off) <= 0):
            raise ValueError("invalid shell table: every shell needs at least one primitive")
        if off[-1] != e.shape[0]:
            raise ValueError("invalid shell table: exponents cover exactly the primitives of the shells")
        if k.shape != (n,) or np.any(k == 0):
            raise ValueError("invalid shell table: every shell needs at least one contraction")
        if co.shape[0] != int((k * np.diff(off)).sum()):
            raise ValueError("invalid shell table: coefficients hold one row per contraction, one entry per primitive")
        if np.any(~(e > 0.0)):
            raise ValueError("invalid shell table: exponents are positive")
        if not np.all(np.isfinite(co)):
            raise ValueError("invalid shell table: coefficients are finite")
        if not np.all(np.isfinite(c)):
            raise ValueError("invalid shell table: centres are finite")
        if np.any(l > 16):
            raise ValueError("invalid shell table: angular momentum exceeds the supported maximum")
        if np.any(l > _MAX_L):
            raise ValueError("the oracle supports angular momentum up to 8")
        self._arrays = (l, c, off, e, co, k)
        self._struct = _Shells(n, _ptr(l), _ptr(c), _ptr(off), _ptr(e), _ptr(co), _ptr(k))
        self._n_functions = int(np.sum(k * (2 * l + 1)))

    @property
    def n_shells(self) -> int:
        return int(self._arrays[0].shape[0])

    @property
    def n_functions(self) -> int:
        return self._n_functions

    def __eq__(self, other) -> bool:
        if not isinstance(other, ShellTable):
            return NotImplemented
        return all(np.array_equal(a, b) for a, b in zip(self._arrays, other._arrays))

    __hash__ = None  # type: ignore[assignment]


def _vectors(a, name: str, width: int = 3) -> np.ndarray:
    v = np.ascontiguousarray(a, dtype=np.float64)
    if v.ndim != 2 or v.shape[1] != width:
        raise ValueError(f"{name} must have shape [n, {width}]")
    if not np.all(np.isfinite(v)):
        raise ValueError(f"{name} are finite")
    return v


def _vector_sets(a, count: int) -> np.ndarray:
    v = np.ascontiguousarray(a, dtype=np.float64)
    if v.ndim != 3 or v.shape[1:] != (count, 3):
        raise ValueError(f"translations must have shape [n, {count}, 3]")
    if not np.all(np.isfinite(v)):
        raise ValueError("translations are finite")
    return v


def _kernel(omega, short_range: bool) -> tuple[int, float]:
    """Kernel selector of coulomb.rs:34-49: Full, LongRange(omega), ShortRange(omega)."""
    if omega is not None and (not np.isfinite(omega) or omega <= 0.0):
        raise ValueError("the range-separation parameter omega is positive")
    if omega is None:
        if short_range:
            raise ValueError("the short-range kernel needs the range-separation parameter omega")
        return 0, 0.0
    return (2 if short_range else 1), float(omega)


def _threshold(threshold: float) -> None:
    if not np.isfinite(threshold) or threshold < 0.0:
        raise ValueError("the screening threshold is finite and non-negative")


def _check(status: int) -> None:
    if status != 0:
        raise ValueError("invalid shell table for the oracle")


def overlap(bra: ShellTable, ket: ShellTable, translations) -> np.ndarray:
    tr = _vectors(translations, "translations")
    out = np.empty((tr.shape[0], bra.n_functions, ket.n_functions))
    _check(library().md_overlap(ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), _ptr(out)))
    return out


def kinetic(bra: ShellTable, ket: ShellTable, translations) -> np.ndarray:
    tr = _vectors(translations, "translations")
    out = np.empty((tr.shape[0], bra.n_functions, ket.n_functions))
    _check(library().md_kinetic(ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), _ptr(out)))
    return out


def nuclear_attraction(bra, ket, translations, charges, positions, omega=None, short_range=False, threshold=0.0):
    tr = _vectors(translations, "translations")
    pos = _vectors(positions, "positions")
    q = np.ascontiguousarray(charges, dtype=np.float64)
    if q.shape[0] != pos.shape[0]:
        raise ValueError(f"length mismatch: {q.shape[0]} and {pos.shape[0]}")
    kind, w = _kernel(omega, short_range)
    _threshold(threshold)
    out = np.empty((tr.shape[0], bra.n_functions, ket.n_functions))
    _check(
        library().md_nuclear_attraction(
            ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), q.shape[0], _ptr(q), _ptr(pos),
            kind, w, _ptr(out),
        )
    )
    return out


def coulomb_two_center(bra, ket, translations, omega=None, short_range=False, threshold=0.0):
    tr = _vectors(translations, "translations")
    kind, w = _kernel(omega, short_range)
    _threshold(threshold)
    out = np.empty((tr.shape[0], bra.n_functions, ket.n_functions))
    _check(
        library().md_coulomb_two_center(
            ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), kind, w, _ptr(out)
        )
    )
    return out


def coulomb_three_center(auxiliary, bra, ket, translations, omega=None, short_range=False, threshold=0.0):
    tr = _vector_sets(translations, 2)
    kind, w = _kernel(omega, short_range)
    _threshold(threshold)
    out = np.empty((tr.shape[0], auxiliary.n_functions, bra.n_functions, ket.n_functions))
    _check(
        library().md_coulomb_three_center(
            ctypes.byref(auxiliary._struct), ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0],
            _ptr(tr), kind, w, _ptr(out),
        )
    )
    return out


def overlap_derivative(bra: ShellTable, ket: ShellTable, translations) -> np.ndarray:
    """``<d_A mu | nu>`` as ``[image, 3, bra, ket]``."""
    tr = _vectors(translations, "translations")
    out = np.empty((tr.shape[0], 3, bra.n_functions, ket.n_functions))
    _check(library().md_overlap_derivative(ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr),
                                           _ptr(out)))
    return out


def kinetic_derivative(bra: ShellTable, ket: ShellTable, translations) -> np.ndarray:
    """``<d_A mu | -1/2 nabla^2 | nu>`` as ``[image, 3, bra, ket]``."""
    tr = _vectors(translations, "translations")
    out = np.empty((tr.shape[0], 3, bra.n_functions, ket.n_functions))
    _check(library().md_kinetic_derivative(ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr),
                                           _ptr(out)))
    return out


def nuclear_attraction_derivative(bra, ket, translations, charges, positions, omega=None, short_range=False):
    """By the bra centres ``[image, 3, bra, ket]`` and by the charge positions
    ``[image, charge, 3, bra, ket]``."""
    tr = _vectors(translations, "translations")
    pos = _vectors(positions, "positions")
    q = np.ascontiguousarray(charges, dtype=np.float64)
    if q.shape[0] != pos.shape[0]:
        raise ValueError(f"length mismatch: {q.shape[0]} and {pos.shape[0]}")
    kind, w = _kernel(omega, short_range)
    by_center = np.empty((tr.shape[0], 3, bra.n_functions, ket.n_functions))
    by_nucleus = np.empty((tr.shape[0], q.shape[0], 3, bra.n_functions, ket.n_functions))
    _check(
        library().md_nuclear_attraction_derivative(
            ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), q.shape[0], _ptr(q), _ptr(pos),
            kind, w, _ptr(by_center), _ptr(by_nucleus),
        )
    )
    return by_center, by_nucleus


def coulomb_two_center_derivative(bra, ket, translations, omega=None, short_range=False):
    """``(d_P P | Q)`` as ``[image, 3, bra, ket]``."""
    tr = _vectors(translations, "translations")
    kind, w = _kernel(omega, short_range)
    out = np.empty((tr.shape[0], 3, bra.n_functions, ket.n_functions))
    _check(
        library().md_coulomb_two_center_derivative(
            ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), kind, w, _ptr(out)
        )
    )
    return out


def coulomb_three_center_derivative(auxiliary, bra, ket, translations, omega=None, short_range=False):
    """``(d_P P | uv)`` and ``(P | d_A u v)``, each ``[image, 3, aux, bra, ket]``."""
    tr = _vector_sets(translations, 2)
    kind, w = _kernel(omega, short_range)
    out = np.empty((tr.shape[0], 6, auxiliary.n_functions, bra.n_functions, ket.n_functions))
    _check(
        library().md_coulomb_three_center_derivative(
            ctypes.byref(auxiliary._struct), ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0],
            _ptr(tr), kind, w, _ptr(out),
        )
    )
    return np.ascontiguousarray(out[:, :3]), np.ascontiguousarray(out[:, 3:])


def coulomb_four_center(bra, ket, translations, omega=None, short_range=False, threshold=0.0):
    tr = _vector_sets(translations, 3)
    kind, w = _kernel(omega, short_range)
    _threshold(threshold)
    b0, b1 = bra
    k0, k1 = ket
    out = np.empty((tr.shape[0], b0.n_functions, b1.n_functions, k0.n_functions, k1.n_functions))
    _check(
        library().md_coulomb_four_center(
            ctypes.byref(b0._struct), ctypes.byref(b1._struct), ctypes.byref(k0._struct), ctypes.byref(k1._struct),
            tr.shape[0], _ptr(tr), kind, w, float(threshold), _ptr(out),
        )
    )
    return out


def schwarz_bounds(bra, ket, translations, omega=None, short_range=False):
    tr = _vectors(translations, "translations")
    kind, w = _kernel(omega, short_range)
    out = np.empty((tr.shape[0], bra.n_shells, ket.n_shells))
    _check(
        library().md_schwarz_bounds(
            ctypes.byref(bra._struct), ctypes.byref(ket._struct), tr.shape[0], _ptr(tr), kind, w, _ptr(out)
        )
    )
    return out


_threads_configured = False


def configure_threads(n_threads: int) -> None:
    """Size the thread pool once per process, as integrals/mod.rs:43-49 does."""
    global _threads_configured
    if _threads_configured:
        raise ValueError("thread pool: the global thread pool has already been initialized")
    _threads_configured = True
    library().md_set_threads(int(n_threads))


def threads() -> int:
    """Threads the oracle library runs on."""
    return int(library().md_get_threads())
