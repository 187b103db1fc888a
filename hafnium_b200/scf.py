"""A device-resident restatement of the reference's restricted SCF driver.

Follows hafnium/scf/driver.py:154-213 (loop), 248-260 (orbital gradient),
307-329 (canonically orthogonalised eigh, next density), 331-366 (finish),
385-389 (convergence test); hafnium/scf/diis.py:55-106 (Pulay DIIS, bordered
system by eigh with the null space dropped); hafnium/scf/orthogonalization.py:16-42;
hafnium/scf/hamiltonian.py:331-370 (restricted Fock build and energy terms);
hafnium/scf/occupation.py:321-370 (aufbau and averaged filling). Every matrix
stays on the GPU in float64 (torch for the eigensolves); J and K come from
``libhfjk.so``. The exchange is built from the occupied orbitals the driver
already holds (D = C_occ C_occ^T), which is the same contraction as K(D).

The reference driver itself is unchanged and can use the drop-in builder
directly; this module exists so that a whole SCF runs on the device, which the
benchmarks and the mixed-precision schedule need.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from hafnium_b200 import _lib
from hafnium_b200.basis import ShellTable
from hafnium_b200.errors import ConvergenceError, InputError
from hafnium_b200.jk import B200DensityFittedCoulombExchange, difference_factors

NULL_SPACE_TOLERANCE = 1e-14  # diis.py:17
DEFAULT_OVERLAP_THRESHOLD = 1e-10  # orthogonalization.py:12
FILL_TOLERANCE = 1e-12  # occupation.py:285


def _torch():
    import torch

    return torch


@dataclass(frozen=True)
class ScfOptions:
    """driver.py:38-66 (no level shift or damping on the device path)."""

    max_iterations: int = 100
    energy_tolerance: float = 1e-10
    gradient_tolerance: float = 1e-6
    diis_size: int = 8
    overlap_threshold: float = DEFAULT_OVERLAP_THRESHOLD
    purify: bool = False  # density by purification after the first iteration (same projector)

    def __post_init__(self) -> None:
        if self.max_iterations < 1:
            raise InputError("at least one iteration is needed")
        if self.energy_tolerance <= 0.0 or self.gradient_tolerance <= 0.0:
            raise InputError("tolerances must be positive")
        if self.diis_size < 1:
            raise InputError("the DIIS subspace holds at least one matrix")


@dataclass(frozen=True)
class PrecisionSchedule:
    """Which arithmetic each exchange build uses.

    ``fp64``: every build in FP64 (the plain path).

    ``mixed``: split-BF16 builds (three BF16 products, FP32 accumulation) from
    the occupied orbitals while the orbital gradient is at or above
    ``anchor_gradient``. The next build is an FP64 anchor K64(D_a), where the
    DIIS history restarts (it held BF16-accurate matrices). After it every
    build is incremental, K(D_n) = K64(D_a) + K16(D_n - D_a), with the
    difference density factored exactly (``jk.difference_factors``), so the
    BF16 error scales with |D_n - D_a| rather than with |D_n|. Once the
    gradient of an incremental build is below the convergence tolerance, the
    finishing build (driver.py:336) is made in FP64 at the aufbau density of
    that Fock matrix; its FP64 orbital gradient decides convergence. A gradient
    below the tolerance bounds the energy error quadratically (far below the
    energy tolerance), so this replaces the reference's test on two
    consecutive FP64 energies, and the reported energy and density are FP64.
    Otherwise that FP64 build becomes the new anchor and the iterations go on.
    If the gradient stops falling (``stall_window`` builds without halving),
    the BF16 phase moves to the anchor and the incremental phase re-anchors.
    DIIS, the eigensolves, J and the energy are FP64 throughout; a mixed run
    makes two FP64 exchange builds when nothing stalls.
    """

    mode: str = "fp64"
    anchor_gradient: float = 1e-3
    stall_window: int = 4
    restart_diis_at_anchor: bool = True

    def __post_init__(self) -> None:
        if self.mode not in ("fp64", "mixed"):
            raise InputError("the precision schedule is 'fp64' or 'mixed'")


@dataclass
class Iteration:
    index: int
    energy: float
    energy_change: float
    gradient_norm: float
    precision: str = "fp64"


@dataclass
class ScfResult:
    energy: float
    density: object  # torch [n, n], per spin
    fock: object
    mo_energies: object
    mo_coefficients: object
    converged: bool
    history: list = field(default_factory=list)
    energy_terms: tuple = ()
    seconds: float = 0.0
    timings: dict = field(default_factory=dict)

    @property
    def n_iterations(self) -> int:
        return len(self.history)


class DeviceHamiltonian:
    """Overlap, core Hamiltonian, nuclear repulsion and the fitted two-body term."""

    def __init__(self, s, h, two_body: B200DensityFittedCoulombExchange, e_nuc: float, n_alpha: int,
                 timings: dict | None = None) -> None:
        self.s, self.h, self.two_body, self.e_nuc, self.n_alpha = s, h, two_body, e_nuc, n_alpha
        self.timings = timings or {}

    @property
    def n_ao(self) -> int:
        return self.two_body.n_ao

    def orthogonalizer(self, threshold: float = DEFAULT_OVERLAP_THRESHOLD):
        """The canonical X of S (orthogonalization.py:16-42), computed once per threshold."""
        cache = self.__dict__.setdefault("_x_cache", {})
        if threshold not in cache:
            cache[threshold] = canonical_orthogonalizer(self.s, threshold)
        return cache[threshold]

    @classmethod
    def build(cls, molecule, basis: str, auxiliary: str, *, device: int = 0,
              exchange_schedule: str = "fp64") -> "DeviceHamiltonian":
        """One-electron integrals and the fitted two-body term of ``molecule``;
        ``exchange_schedule`` is the builder's own schedule for ``exchange(D)``
        (``"mixed"`` for the protocol-driven mixed-precision path)."""
        torch = _torch()
        t0 = time.perf_counter()
        orb = ShellTable.build(basis, molecule.symbols, molecule.positions)
        aux = ShellTable.build(auxiliary, molecule.symbols, molecule.positions)
        ctx = _lib.Context(device)
        ctx.upload(orb, aux)
        dev = torch.device("cuda", device)
        n = orb.n_functions
        s = torch.empty((n, n), dtype=torch.float64, device=dev)
        t = torch.empty_like(s)
        v = torch.empty_like(s)
        charges = torch.as_tensor(molecule.nuclear_charges, dtype=torch.float64, device=dev)
        positions = torch.as_tensor(np.ascontiguousarray(molecule.positions), dtype=torch.float64, device=dev)
        _lib.torch_sync(s)  # the library reads these on its own stream
        for kind, out, args in ((0, s, ()), (1, t, ()), (2, v, (charges, positions))):
            q, r = args if args else (None, None)
            ctx.check(
                ctx.lib.hf_one_electron(ctx.handle, kind, None if q is None else q.data_ptr(),
                                        None if r is None else r.data_ptr(), 0 if q is None else q.shape[0],
                                        out.data_ptr(), 1),
                "hf_one_electron",
            )
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        ctx.build()
        torch.cuda.synchronize(dev)
        t2 = time.perf_counter()
        two_body = B200DensityFittedCoulombExchange(ctx, schedule=exchange_schedule)
        timings = {"one_electron_s": t1 - t0, "fitted_tensor_s": t2 - t1, **ctx.stats()}
        return cls(s, t + v, two_body, molecule.nuclear_repulsion_energy(), molecule.n_alpha, timings)


def canonical_orthogonalizer(s, threshold: float = DEFAULT_OVERLAP_THRESHOLD):
    """orthogonalization.py:16-42."""
    torch = _torch()
    w, v = torch.linalg.eigh(s)
    n = s.shape[-1]
    kept = int((w > threshold).sum())
    if kept == 0:
        raise InputError("no eigenvalue of the overlap exceeds the threshold")
    return v[:, n - kept:] / torch.sqrt(w[n - kept:])[None, :]


def solve_diis(overlaps: np.ndarray) -> np.ndarray:
    """diis.py:82-106 on the host (an m x m system, m <= diis_size)."""
    m = overlaps.shape[0]
    scale = np.max(np.diagonal(overlaps))
    b = overlaps / (scale if scale > 0.0 else 1.0)
    system = np.zeros((m + 1, m + 1))
    system[:m, :m] = b
    system[:m, m] = -1.0
    system[m, :m] = -1.0
    right = np.zeros(m + 1)
    right[m] = -1.0
    w, v = np.linalg.eigh(system)
    keep = np.abs(w) > NULL_SPACE_TOLERANCE * np.max(np.abs(w))
    inv = np.where(keep, 1.0 / np.where(keep, w, 1.0), 0.0)
    return (v @ (inv * (v.T @ right)))[:m]


def purify(fo, n_occ: int, tolerance: float = 1e-9, max_steps: int = 100):
    """Canonical purification of a symmetric matrix ``fo`` (orthonormal basis) to
    the projector onto its n_occ lowest eigenvectors (Palser and Manolopoulos,
    PRB 58, 12704 (1998), eq. 13-16): P0 from Gershgorin bounds, then
    P <- (P^2 ((1 + c) I - P)) / c or its c < 1/2 form, c = tr(P^2 - P^3) / tr(P - P^2),
    until tr(P - P^2) < tolerance, plus one more (quadratic) step. Returns
    (P, converged)."""
    torch = _torch()
    m = fo.shape[0]
    diag = torch.diagonal(fo)
    radius = fo.abs().sum(dim=1) - diag.abs()
    lo, hi, mu = float((diag - radius).min()), float((diag + radius).max()), float(diag.sum()) / m
    if not (hi > mu > lo) or not 0 < n_occ < m:
        return fo, False
    lam = min(n_occ / (hi - mu), (m - n_occ) / (mu - lo))
    eye = torch.eye(m, dtype=fo.dtype, device=fo.device)
    p = (lam / m) * (mu * eye - fo) + (n_occ / m) * eye
    crossed = False
    for _ in range(max_steps):
        p2 = p @ p
        t1 = float(torch.diagonal(p).sum() - torch.diagonal(p2).sum())
        t2 = float(torch.diagonal(p2).sum() - (p2 * p).sum())
        if crossed:
            return 0.5 * (p + p.T), True
        if t1 < tolerance:
            crossed = True
        if t1 > 0.0:
            c = min(1.0, max(0.0, t2 / t1))
        elif abs(t1) < tolerance:
            c = 0.5
        else:
            return p, False
        if c >= 0.5:
            p = p2 @ (((1.0 + c) * eye - p) / c)
        else:
            p = p2 @ (((1.0 + c) * eye - p) / (1.0 - c)) + ((1.0 - 2.0 * c) / (1.0 - c)) * p
    return p, False


def fill_averaged(energies: np.ndarray, count: float, tolerance: float = 1e-6) -> np.ndarray:
    """occupation.py:342-370: degenerate groups share electrons equally."""
    order = np.argsort(energies, kind="stable")
    values = energies[order]
    spread = max(1.0, float(values[-1] - values[0])) if len(values) else 1.0
    occ = np.zeros(len(energies))
    remaining = count
    start = 0
    while start < len(order):
        end = start + 1
        while end < len(order) and values[end] - values[end - 1] <= tolerance * spread:
            end += 1
        group = order[start:end]
        share = min(remaining, float(len(group))) / len(group)
        occ[group] = share
        remaining = max(remaining - share * len(group), 0.0)
        start = end
    if not math.isclose(remaining, 0.0, abs_tol=FILL_TOLERANCE):
        raise InputError(f"cannot place {count} electrons in {len(energies)} levels")
    return occ


class _ExactTwoBody:
    """Exact J/K from four-centre integrals held on the device (coulomb_exchange.py:75-121)."""

    def __init__(self, eri) -> None:
        self.eri = eri
        self.n_ao = eri.shape[0]

    def coulomb(self, d):
        return _torch().einsum("uvwx,wx->uv", self.eri, d)

    def exchange(self, d):
        return _torch().einsum("uwxv,wx->uv", self.eri, d)

    def exchange_factored(self, factor, weights=None):
        return self.exchange(factor @ factor.T)


def _spherical_atom(symbol: str, basis: str, device: int):
    """atoms.py:55-73: the neutral atom with exact J/K and averaged occupations."""
    torch = _torch()
    from hafnium_b200.molecule import Molecule, atomic_number

    z = atomic_number(symbol)
    atom = Molecule((symbol,), np.zeros((1, 3)))
    orb = ShellTable.build(basis, atom.symbols, atom.positions)
    ctx = _lib.Context(device)
    ctx.upload(orb)
    dev = torch.device("cuda", device)
    s = torch.as_tensor(ctx.one_electron(0), device=dev)
    h = torch.as_tensor(ctx.one_electron(1) + ctx.one_electron(2, np.array([float(z)]), np.zeros((1, 3))), device=dev)
    eri = torch.as_tensor(ctx.four_center(), device=dev)
    ctx.close()
    ham = DeviceHamiltonian(s, h, _ExactTwoBody(eri), 0.0, z / 2.0)
    return _Rhf(ham, ScfOptions(), PrecisionSchedule(), averaged=True).run(None).density


_ATOM_CACHE: dict[tuple, object] = {}


def atomic_density_guess(molecule, basis: str, *, device: int = 0):
    """atoms.py:76-120: converge each distinct element once, place the per-spin
    atomic densities on the diagonal in atom order (molecular case). An
    element's atomic density depends only on the element and the basis, so it
    is converged once per process and device and kept."""
    torch = _torch()
    return torch.block_diag(*[atomic_block(symbol, basis, device) for symbol in molecule.symbols]).contiguous()


def atomic_block(symbol: str, basis: str, device: int = 0):
    """The converged per-spin density of one neutral atom (atoms.py:55-73), cached."""
    key = (symbol, basis.lower(), device)
    if key not in _ATOM_CACHE:
        _ATOM_CACHE[key] = _spherical_atom(symbol, basis, device)
    return _ATOM_CACHE[key]


def project_occupied(ham: DeviceHamiltonian, density, threshold: float = DEFAULT_OVERLAP_THRESHOLD):
    """The idempotent density of the n_alpha leading natural orbitals of ``density``
    in the overlap metric: D' = C C^T with X^T S D S X = V diag(w) V^T, C = X V_top."""
    torch = _torch()
    x = ham.orthogonalizer(threshold)
    d = torch.as_tensor(density, dtype=torch.float64, device=ham.s.device)
    d = 0.5 * (d + d.T)
    m = x.T @ ham.s @ d @ ham.s @ x
    w, v = torch.linalg.eigh(0.5 * (m + m.T))
    c = x @ v[:, -int(ham.n_alpha):]
    return (c @ c.T).contiguous()


def learned_density_guess(molecule, ham: DeviceHamiltonian, *, weights=None, basis: str = "cc-pvdz",
                          device: int = 0):
    """The learned network's density projected onto the occupied space; the SAD
    guess (atoms.py:76-120) when the network does not apply (no weights, another
    basis than cc-pVDZ, an element it was not trained on, a linear molecule)."""
    from hafnium_b200.learned.model import predict_density

    predicted = predict_density(molecule, weights, device=device) if basis == "cc-pvdz" else None
    if predicted is None or not bool(_torch().isfinite(predicted).all()):
        return atomic_density_guess(molecule, basis, device=device)
    return project_occupied(ham, predicted)


class _HostTwoBody:
    """The drop-in's host-array API (coulomb_exchange.py:176-190) seen from the
    device driver: device inputs are copied to host NumPy arrays, passed to the
    builder's host entry points, and the results copied back; the bytes each way
    are counted on the driver."""

    def __init__(self, two_body, rhf) -> None:
        self.two_body, self.rhf = two_body, rhf

    def _down(self, t):
        a = t.detach().cpu().numpy()
        self.rhf.h2d_bytes += a.nbytes
        return a

    def _up(self, a, device):
        self.rhf.d2h_bytes += a.nbytes
        return _torch().as_tensor(a, device=device)

    def coulomb(self, d):
        return self._up(self.two_body.coulomb(self._down(d)), d.device)

    def exchange(self, d):
        return self._up(self.two_body.exchange(self._down(d)), d.device)

    def exchange_factored(self, factor, weights=None, precision=None):
        w = None if weights is None else self._down(weights)
        return self._up(self.two_body.exchange_factored(self._down(factor), w, precision), factor.device)

    def context_exchange_bf16(self, d):
        return self._up(self.two_body.context.exchange_host(self._down(d), _lib.PREC_BF16X3), d.device)


class _Rhf:
    def __init__(self, ham: DeviceHamiltonian, options: ScfOptions, schedule: PrecisionSchedule,
                 host_io: bool = False, averaged: bool = False, protocol: bool = False) -> None:
        torch = _torch()
        self.torch = torch
        self.host_io = host_io
        self.protocol = protocol
        self.last_precision = "fp64"
        self.averaged = averaged
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.ham = ham
        self.options = options
        self.schedule = schedule
        self.x = ham.orthogonalizer(options.overlap_threshold)
        self.n = ham.n_ao
        self.z = None  # occupied orbitals of the last iteration, orthonormal basis
        self.purify = options.purify
        self.anchor_k = None  # K64(D_a) of the last FP64 anchor
        self.anchor_factor = None  # C_a with D_a = C_a C_a^T
        self.timings = {"coulomb_ms": 0.0, "exchange_ms": 0.0, "eigh_ms": 0.0, "fock_builds": 0}

    def solve(self, f):
        torch = self.torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        w, v = torch.linalg.eigh(self.x.T @ f @ self.x)
        c = self.x @ v
        e1.record()
        e1.synchronize()
        self.timings["eigh_ms"] += e0.elapsed_time(e1)
        return w, c

    def next_density(self, f):
        """(D, C) of the aufbau state of Fock matrix ``f``: the reference's
        eigensolve (driver.py:307-329) on the first iteration, afterwards canonical
        purification (Palser and Manolopoulos, PRB 58, 12704 (1998)) of X^T f X on
        the tensor cores and the occupied orbitals as the span of P Z, Z the
        previous occupied orbitals, orthonormalised by a Cholesky factor. With a
        HOMO-LUMO gap both give the same projector; without one, or when P Z loses
        rank, the eigensolve is used."""
        torch = self.torch
        if self.averaged or self.z is None or not self.purify:
            w, c = self.solve(f)
            d, factor = self.density(w, c, averaged=False)
            self.z = self.x.T @ self.ham.s @ factor  # the occupied orbitals in the orthonormal basis
            return d, factor
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fo = self.x.T @ f @ self.x
        p, ok = purify(0.5 * (fo + fo.T), int(self.ham.n_alpha))
        if ok:
            y = p @ self.z
            g = y.T @ y
            low, info = torch.linalg.cholesky_ex(0.5 * (g + g.T))
            ok = int(info) == 0 and float(torch.diagonal(low).min()) > 1e-3
        if ok:
            z = torch.linalg.solve_triangular(low, y.T, upper=False).T.contiguous()
            self.z = z
            factor = (self.x @ z).contiguous()
        e1.record()
        e1.synchronize()
        self.timings["purify_ms"] = self.timings.get("purify_ms", 0.0) + e0.elapsed_time(e1)
        if not ok:
            self.timings["purify_fallbacks"] = self.timings.get("purify_fallbacks", 0) + 1
            self.z = None
            return self.next_density(f)
        return factor @ factor.T, factor

    def density(self, w, c, averaged: bool):
        if averaged or self.averaged:
            occ = fill_averaged(w.cpu().numpy(), float(self.ham.n_alpha))
        else:
            occ = np.zeros(w.shape[0])
            occ[np.argsort(w.cpu().numpy(), kind="stable")[: int(self.ham.n_alpha)]] = 1.0
        keep = np.nonzero(occ > 0.0)[0]
        idx = self.torch.as_tensor(keep, device=c.device)
        occ_t = self.torch.as_tensor(occ[keep], dtype=self.torch.float64, device=c.device)
        factor = (c[:, idx] * self.torch.sqrt(occ_t)[None, :]).contiguous()
        return factor @ factor.T, factor

    def _timed(self, key: str, fn):
        torch = self.torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        e1.synchronize()
        self.timings[f"exchange_ms_{key}"] = self.timings.get(f"exchange_ms_{key}", 0.0) + e0.elapsed_time(e1)
        self.timings[f"exchange_builds_{key}"] = self.timings.get(f"exchange_builds_{key}", 0) + 1
        return out

    def difference_factors(self, factor):
        """(V+, V-) with D_n - D_a = V+ V+^T - V- V-^T (``jk.difference_factors``:
        the anchor's orbitals rotated onto the current ones, then matrix products)."""
        return difference_factors(factor, self.anchor_factor, self.ham.s)

    def gradient_norm(self, f, d) -> float:
        """driver.py:248-260: |X^T (F D S - S D F) X| with the factor 2 of the restricted trace."""
        s = self.ham.s
        g = self.x.T @ (f @ d @ s - s @ d @ f) @ self.x
        return math.sqrt(2.0 * float(self.torch.sum(g * g))), g

    def exchange(self, d, factor, precision: str, two_body=None):
        """K for this iteration in the arithmetic ``precision`` names: ``fp64``,
        ``bf16`` (split-BF16 from the orbitals), ``anchor`` (FP64, kept as the
        base of the increments) or ``incremental``."""
        two_body = two_body or self.ham.two_body
        if precision in ("fp64", "anchor"):
            k = self._timed("fp64", lambda: two_body.exchange(d) if factor is None else
                            two_body.exchange_factored(factor))
            if precision == "anchor":
                self.anchor_k, self.anchor_factor = k, factor
                self.timings["anchors"] = self.timings.get("anchors", 0) + 1
            return k
        if precision == "bf16":
            if factor is None:
                return self._timed("bf16", lambda: two_body.context_exchange_bf16(d))
            return self._timed("bf16", lambda: two_body.exchange_factored(factor, precision=_lib.PREC_BF16X3))
        vp, vm = self.difference_factors(factor)

        def increment():
            # the positive and negative parts as two unsigned split-BF16 builds of
            # n_occ columns each (a single signed build over 2 n_occ columns measured
            # 2.6x slower at (H2O)64: its X chunks are four times smaller)
            out = self.anchor_k.clone()
            out += two_body.exchange_factored(vp, precision=_lib.PREC_BF16X3)
            out -= two_body.exchange_factored(vm, precision=_lib.PREC_BF16X3)
            return out

        return self._timed("incremental", increment)

    def fock(self, d, factor, precision: str = "fp64"):
        """hamiltonian.py:331-370 for one restricted block."""
        torch = self.torch
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        if self.protocol:
            # the reference's calls only: coulomb(2 D) and exchange(D), the builder
            # choosing its own arithmetic (coulomb_exchange.py:426, 509)
            two_body = _HostTwoBody(self.ham.two_body, self) if self.host_io else self.ham.two_body
            j = two_body.coulomb((2.0 * d).contiguous())
            ev[1].record()
            k = two_body.exchange(d.contiguous())
            log = getattr(getattr(self.ham.two_body, "schedule", None), "log", None)
            self.last_precision = log[-1]["precision"] if log else "fp64"
        elif self.host_io:
            # the reference-facing calls: host NumPy arrays in, host NumPy J/K out
            host = _HostTwoBody(self.ham.two_body, self)
            j = host.coulomb((2.0 * d).contiguous())
            ev[1].record()
            k = self.exchange(d, factor, precision, host)
        else:
            j = self.ham.two_body.coulomb((2.0 * d).contiguous())
            ev[1].record()
            k = self.exchange(d, factor, precision)
        ev[2].record()
        f = self.ham.h + j - k
        e1 = 2.0 * torch.sum(d * self.ham.h)
        ej = torch.sum(d * j)
        ek = -torch.sum(d * k)
        terms = torch.stack([e1, ej, ek]).cpu().numpy()
        self.timings["coulomb_ms"] += ev[0].elapsed_time(ev[1])
        self.timings["exchange_ms"] += ev[1].elapsed_time(ev[2])
        self.timings["fock_builds"] += 1
        energy = self.ham.e_nuc + float(terms.sum())
        return f, (self.ham.e_nuc, *map(float, terms)), energy

    def run(self, guess) -> ScfResult:
        torch = self.torch
        opts = self.options
        t_start = time.perf_counter()
        if guess is None:  # driver.py:230-236 averaged core-Hamiltonian density
            w, c = self.solve(self.ham.h)
            d, factor = self.density(w, c, averaged=True)
        else:
            d = torch.as_tensor(guess, dtype=torch.float64, device=self.ham.s.device)
            factor = None
        focks, errors, history = [], [], []
        mixed = self.schedule.mode == "mixed" and not self.protocol
        precision = "bf16" if mixed else "fp64"
        pending = None  # a Fock build already made for d (after an FP64 finish that did not converge)
        f = None
        for index in range(opts.max_iterations):
            if pending is not None:
                f, energy = pending
                pending = None
            else:
                f, _, energy = self.fock(d, factor, precision)
            gnorm, g = self.gradient_norm(f, d)
            previous = history[-1] if history else None
            change = energy - previous.energy if previous else math.inf
            built = self.last_precision if self.protocol else ("fp64" if precision == "anchor" else precision)
            history.append(Iteration(index, energy, change, gnorm, built))
            converged = abs(change) < opts.energy_tolerance and gnorm < opts.gradient_tolerance
            if not mixed:
                if converged:
                    return self.finish(f, history, True, t_start)
            elif built != "bf16" and gnorm < opts.gradient_tolerance:
                if built == "fp64" and converged:
                    return self.finish(f, history, True, t_start)
                # the finishing build (driver.py:336) in FP64 at the aufbau density
                # of f; its exact orbital gradient decides convergence
                w, c = self.solve(f)
                d2, factor2 = self.density(w, c, averaged=False)
                f2, terms2, e2 = self.fock(d2, factor2, "anchor")
                g2, _ = self.gradient_norm(f2, d2)
                if g2 < opts.gradient_tolerance:
                    self.torch.cuda.synchronize()
                    self.timings["final_gradient"] = g2
                    return ScfResult(e2, d2, f2, w, c, True, history, terms2, time.perf_counter() - t_start,
                                     dict(self.timings))
                # not yet: that FP64 build is the new anchor and the iterations go on
                d, factor, pending = d2, factor2, (f2, e2)
                precision = "anchor"
                continue
            if precision == "anchor":
                precision = "incremental"
                if self.schedule.restart_diis_at_anchor:
                    focks, errors = [], []  # the history held BF16-accurate matrices
            elif precision == "bf16" and gnorm < self.schedule.anchor_gradient:
                precision = "anchor"
            elif precision in ("bf16", "incremental"):
                window = self.schedule.stall_window
                recent = [h for h in history[-window - 1:] if h.precision == built]
                if len(recent) > window and gnorm > 0.5 * recent[0].gradient_norm:
                    # the gradient stopped halving: BF16 noise (or a far anchor) bounds it
                    precision = "anchor"
            focks = (focks + [f])[-opts.diis_size:]
            errors = (errors + [g])[-opts.diis_size:]
            if len(focks) == 1:
                extrapolated = focks[0]
            else:
                ov = torch.stack([torch.stack([2.0 * torch.sum(a * b) for b in errors]) for a in errors]).cpu().numpy()
                coef = solve_diis(ov)
                extrapolated = sum(float(cf) * fk for cf, fk in zip(coef, focks))
            d, factor = self.next_density(extrapolated)
        result = self.finish(focks[-1] if focks else f, history, False, t_start)
        raise ConvergenceError(f"the SCF did not converge in {opts.max_iterations} iterations", result)

    def finish(self, f, history, converged: bool, t_start: float) -> ScfResult:
        """driver.py:331-366: one more Fock build from the aufbau density of ``f``."""
        w, c = self.solve(f)
        d, factor = self.density(w, c, averaged=False)
        final_f, terms, energy = self.fock(d, factor, "fp64")
        self.torch.cuda.synchronize()
        return ScfResult(energy, d, final_f, w, c, converged, history, terms, time.perf_counter() - t_start,
                         dict(self.timings))


def solve_rhf(ham: DeviceHamiltonian, *, guess=None, options: ScfOptions | None = None,
              schedule: PrecisionSchedule | None = None, host_io: bool = False, protocol: bool = False) -> ScfResult:
    """Converge the restricted state of ``ham`` on the device (driver.py:154-213).

    ``host_io`` routes every J and K through the drop-in's host-array API (NumPy
    density in, NumPy J/K out), as the unchanged reference driver would call it.
    ``protocol`` makes the driver call nothing but ``coulomb(2 D)`` and
    ``exchange(D)`` of the two-body builder, with the reference's convergence
    test: the builder's own schedule (``B200DensityFittedCoulombExchange``
    with ``schedule="mixed"``) then chooses each build's arithmetic, and
    ``schedule`` is not used.
    """
    rhf = _Rhf(ham, options or ScfOptions(), schedule or PrecisionSchedule(), host_io, protocol=protocol)
    result = rhf.run(guess)
    result.timings["h2d_bytes"] = rhf.h2d_bytes
    result.timings["d2h_bytes"] = rhf.d2h_bytes
    return result
