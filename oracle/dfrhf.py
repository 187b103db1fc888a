"""Oracle: a NumPy FP64 restatement of the reference's molecular DF-RHF.

TEST INFRASTRUCTURE ONLY (the checker for ``tests/``, ``smoke()`` and the CPU
baseline of ``bench.py``); the product never imports it.

Each function restates one piece of the reference, cited by file:line. Integrals
come from ``oracle.kernels`` (the C++ restatement of the Rust kernels). The
restatement is pinned against the reference itself: ``tests/golden/make_golden.py``
runs the reference's own ``solve_scf`` on the same inputs in a container where
the reference tree is mounted and stores energies, densities and iteration
counts as fixtures, which ``tests/test_oracle.py`` compares against.

Shell tables are passed as objects with the SoA attributes of
``hafnium/integrals/shell_table.py:14-82`` (``angular_momenta``, ``centers``,
``primitive_offsets``, ``exponents``, ``coefficients``, ``n_contractions``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from oracle import kernels

DEFAULT_METRIC_THRESHOLD = 1e-10  # density_fitting.py:32
DEFAULT_OVERLAP_THRESHOLD = 1e-10  # orthogonalization.py:12
NULL_SPACE_TOLERANCE = 1e-14  # diis.py:17
DEFAULT_SCHWARZ_THRESHOLD = 1e-14  # integrals/two_electron.py:17
FILL_TOLERANCE = 1e-12  # occupation.py:285
ZERO = np.zeros((1, 3))


def kernel_table(table) -> kernels.ShellTable:
    """native.py:16-24: marshal the SoA arrays into the kernel module's table."""
    counts = getattr(table, "n_contractions", None)
    if counts is None:
        counts = table.contraction_counts
    return kernels.ShellTable(
        table.angular_momenta, table.centers, table.primitive_offsets, table.exponents, table.coefficients, counts
    )


# ------------------------------------------------------------------ integrals
def overlap(table) -> np.ndarray:
    t = kernel_table(table)
    return kernels.overlap(t, t, ZERO)[0]


def core_hamiltonian(table, charges, positions) -> np.ndarray:
    """one_electron.py:65-75: kinetic plus attraction to the nuclei."""
    t = kernel_table(table)
    return kernels.kinetic(t, t, ZERO)[0] + kernels.nuclear_attraction(t, t, ZERO, charges, positions)[0]


def metric(aux) -> np.ndarray:
    """density_fitting.py:77: (P|Q) with the full kernel."""
    a = kernel_table(aux)
    return kernels.coulomb_two_center(a, a, ZERO)[0]


def three_center(aux, orb) -> np.ndarray:
    """density_fitting.py:78-84: (P|uv) as [aux, ao, ao], both triangles."""
    a, o = kernel_table(aux), kernel_table(orb)
    return kernels.coulomb_three_center(a, o, o, np.zeros((1, 2, 3)))[0]


def inverse_square_root(m: np.ndarray, threshold: float = DEFAULT_METRIC_THRESHOLD) -> tuple[np.ndarray, int]:
    """density_fitting.py:181-197: M^{-1/2}, eigenvalues below threshold*max dropped."""
    w, v = np.linalg.eigh(m)
    keep = w > threshold * np.max(w)
    safe = np.where(keep, w, 1.0)
    inv = np.where(keep, 1.0 / np.sqrt(safe), 0.0)
    return (v * inv) @ v.T, int(m.shape[0] - keep.sum())


def df_tensor(m: np.ndarray, t3: np.ndarray, threshold: float = DEFAULT_METRIC_THRESHOLD) -> np.ndarray:
    """density_fitting.py:97-107: B = M^{-1/2} (P|uv)."""
    half, _ = inverse_square_root(m, threshold)
    return (half @ t3.reshape(t3.shape[0], -1)).reshape(t3.shape)


def coulomb(b: np.ndarray, d: np.ndarray) -> np.ndarray:
    """coulomb_exchange.py:176-182: charges = B.vec(D); J = charges.B."""
    naux, n = b.shape[0], b.shape[1]
    flat = b.reshape(naux, n * n)
    return (((flat @ d.reshape(n * n)) @ flat)).reshape(n, n)


def exchange(b: np.ndarray, d: np.ndarray) -> np.ndarray:
    """coulomb_exchange.py:184-190: K = sum_P B_P D B_P."""
    naux, n = b.shape[0], b.shape[1]
    half = b @ d
    left = np.transpose(half, (1, 0, 2)).reshape(n, naux * n)
    return left @ b.reshape(naux * n, n)


def eri_exact(table) -> np.ndarray:
    """two_electron.py (hafnium/integrals): (uv|wx) with Schwarz threshold 1e-14."""
    t = kernel_table(table)
    return kernels.coulomb_four_center((t, t), (t, t), np.zeros((1, 3, 3)), threshold=DEFAULT_SCHWARZ_THRESHOLD)[0]


# ---------------------------------------------------------------- SCF pieces
def canonical_orthogonalizer(s: np.ndarray, threshold: float = DEFAULT_OVERLAP_THRESHOLD) -> np.ndarray:
    """orthogonalization.py:16-42: X = V s^{-1/2} over eigenvalues above threshold."""
    w, v = np.linalg.eigh(s)
    n = s.shape[-1]
    kept = int(np.sum(w > threshold))
    if kept == 0:
        raise ValueError("no eigenvalue of the overlap exceeds the threshold")
    return v[:, n - kept:] / np.sqrt(w[n - kept:])[None, :]


def solve_diis(overlaps: np.ndarray) -> np.ndarray:
    """diis.py:82-106: bordered system solved by eigh, null space dropped."""
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


def fill_aufbau(energies: np.ndarray, count: int) -> np.ndarray:
    """occupation.py:321-339 for a molecule: the lowest ``count`` levels get one."""
    occ = np.zeros(energies.shape[0])
    occ[np.argsort(energies, kind="stable")[:count]] = 1.0
    return occ


def fill_averaged(energies: np.ndarray, count: float, tolerance: float = 1e-6) -> np.ndarray:
    """occupation.py:342-370: degenerate groups share electrons equally."""
    order = sorted(range(len(energies)), key=lambda i: float(energies[i]))
    values = [float(energies[i]) for i in order]
    spread = max(1.0, values[-1] - values[0]) if values else 1.0
    occ = np.zeros(len(energies))
    remaining = count
    start = 0
    while start < len(order):
        end = start + 1
        while end < len(order) and values[end] - values[end - 1] <= tolerance * spread:
            end += 1
        group = order[start:end]
        capacity = float(len(group))
        share = min(remaining, capacity) / capacity
        occ[group] = share
        remaining = max(remaining - share * capacity, 0.0)
        start = end
    if not math.isclose(remaining, 0.0, abs_tol=FILL_TOLERANCE):
        raise ValueError(f"cannot place {count} electrons in {len(energies)} levels")
    return occ


@dataclass
class Iteration:
    index: int
    energy: float
    energy_change: float
    gradient_norm: float


@dataclass
class RhfResult:
    energy: float
    density: np.ndarray  # per-spin D_alpha
    fock: np.ndarray
    mo_energies: np.ndarray
    mo_coefficients: np.ndarray
    converged: bool
    history: list = field(default_factory=list)
    energy_terms: tuple = ()

    @property
    def n_iterations(self) -> int:
        return len(self.history)


class ExactJK:
    """coulomb_exchange.py:75-121 restricted to what the SAD atoms need."""

    def __init__(self, eri: np.ndarray) -> None:
        self.eri = eri

    def coulomb(self, d):
        return np.einsum("uvwx,wx->uv", self.eri, d)

    def exchange(self, d):
        return np.einsum("uwxv,wx->uv", self.eri, d)


class FittedJK:
    """coulomb_exchange.py:125-190: J and K from the fitted tensor B[aux, ao, ao]."""

    def __init__(self, b: np.ndarray) -> None:
        self.b = b

    def coulomb(self, d):
        return coulomb(self.b, d)

    def exchange(self, d):
        return exchange(self.b, d)


def psd_factor(d: np.ndarray, tolerance: float = 1e-14) -> np.ndarray:
    """``F`` with ``F F^T = D`` for a symmetric positive semidefinite ``D``: the
    eigenvectors of the eigenvalues above ``tolerance`` times the largest,
    scaled by their square roots."""
    w, v = np.linalg.eigh(0.5 * (d + d.T))
    keep = w > tolerance * max(float(np.max(np.abs(w))), 1e-300)
    return v[:, keep] * np.sqrt(w[keep])[None, :]


class LeanFittedJK:
    """coulomb_exchange.py:176-190 with the exchange contracted through an
    occupied factor of the density: ``K = sum_P (B_P F)(B_P F)^T`` for
    ``D = F F^T`` (the same sum as ``sum_P B_P D B_P``, at 4 N n^2 r instead of
    4 N n^3 flops and without B-sized temporaries). The densities of the
    restricted driver are positive semidefinite (aufbau projectors, the SAD
    guess), so the factor exists; an indefinite input raises."""

    def __init__(self, b: np.ndarray) -> None:
        self.b = b

    def coulomb(self, d):
        return coulomb(self.b, d)

    def exchange(self, d):
        w = np.linalg.eigvalsh(0.5 * (d + d.T))
        if w[0] < -1e-10 * max(float(np.max(np.abs(w))), 1e-300):
            raise ValueError("the lean exchange needs a positive semidefinite density")
        f = psd_factor(d)
        naux, n = self.b.shape[0], self.b.shape[1]
        k = np.zeros((n, n))
        step = max(1, int(2**28 // max(1, 8 * n * f.shape[1])))  # about 256 MB of B_P F at a time
        for start in range(0, naux, step):
            x = self.b[start:start + step] @ f  # [chunk, n, r]
            flat = np.ascontiguousarray(np.transpose(x, (1, 0, 2))).reshape(n, -1)
            k += flat @ flat.T
        return 0.5 * (k + k.T)


def build_problem_lean(orb, aux, charges, positions, e_nuc: float, n_alpha: int) -> "DfRhfProblem":
    """``build_problem`` with B = M^{-1/2} (P|uv) formed in place over column
    blocks of the three-centre tensor (one [aux, ao, ao] array in memory instead
    of two); ``metric`` is kept and ``three_center`` is not (it is B)."""
    s = overlap(orb)
    h = core_hamiltonian(orb, charges, positions)
    m = metric(aux)
    b = three_center(aux, orb)
    half, dropped = inverse_square_root(m)
    flat = b.reshape(b.shape[0], -1)
    for start in range(0, flat.shape[1], 8192):
        flat[:, start:start + 8192] = half @ flat[:, start:start + 8192]
    return DfRhfProblem(s, h, b, e_nuc, n_alpha, m, np.zeros((0,)), dropped)


def fock_rhf(h, jk, d_alpha, e_nuc):
    """hamiltonian.py:331-370 for the restricted class: J from 2 D_a, K from D_a.

    The structured trace of a restricted matrix counts both spins, so
    E = E_nuc + 2 tr(D h) + tr(D J) - tr(D K) with J = J(2 D).
    """
    j = jk.coulomb(2.0 * d_alpha)
    k = jk.exchange(d_alpha)
    f = h + j - k
    e1 = 2.0 * float(np.sum(d_alpha * h))
    ej = 2.0 * float(np.sum(d_alpha * j)) / 2.0
    ek = -2.0 * float(np.sum(d_alpha * k)) / 2.0
    return f, (e_nuc, e1, ej, ek), e_nuc + e1 + ej + ek


def solve_rhf(
    s,
    h,
    jk,
    e_nuc: float,
    n_alpha: float,
    *,
    guess=None,
    averaged: bool = False,
    max_iterations: int = 100,
    energy_tolerance: float = 1e-10,
    gradient_tolerance: float = 1e-6,
    diis_size: int = 8,
) -> RhfResult:
    """driver.py:154-213 + 331-366 for one restricted block.

    ``averaged`` selects AveragedOccupation (the SAD atoms) over aufbau.
    Raises RuntimeError with ``.last`` when the iteration does not converge.
    """
    x = canonical_orthogonalizer(s)

    def solve(f):
        w, v = np.linalg.eigh(x.T @ f @ x)
        return w, x @ v

    def occupy(w):
        return fill_averaged(w, n_alpha) if averaged else fill_aufbau(w, int(n_alpha))

    if guess is None:  # driver.py:230-236 _averaged_core_density
        w, c = solve(h)
        d = (c * fill_averaged(w, n_alpha)[None, :]) @ c.T
    else:
        d = guess
    focks: list[np.ndarray] = []
    errors: list[np.ndarray] = []
    history: list[Iteration] = []
    f = None
    for index in range(max_iterations):
        f, _, energy = fock_rhf(h, jk, d, e_nuc)
        g = x.T @ (f @ d @ s - s @ d @ f) @ x
        gnorm = math.sqrt(2.0 * float(np.sum(g * g)))
        change = energy - history[-1].energy if history else math.inf
        history.append(Iteration(index, energy, change, gnorm))
        if abs(change) < energy_tolerance and gnorm < gradient_tolerance:
            return _finish(f, solve, occupy, h, jk, e_nuc, history, True)
        focks = (focks + [f])[-diis_size:]
        errors = (errors + [g])[-diis_size:]
        if len(focks) == 1:
            extrapolated = focks[0]
        else:
            ov = np.array([[2.0 * float(np.sum(a * b)) for b in errors] for a in errors])
            coef = solve_diis(ov)
            extrapolated = sum(c * fk for c, fk in zip(coef, focks))
        w, c = solve(extrapolated)
        d = (c * occupy(w)[None, :]) @ c.T
    result = _finish(focks[-1], solve, occupy, h, jk, e_nuc, history, False)
    error = RuntimeError(f"the SCF did not converge in {max_iterations} iterations")
    error.last = result  # type: ignore[attr-defined]
    raise error


def _finish(f, solve, occupy, h, jk, e_nuc, history, converged) -> RhfResult:
    w, c = solve(f)
    d = (c * occupy(w)[None, :]) @ c.T
    final_f, terms, energy = fock_rhf(h, jk, d, e_nuc)
    return RhfResult(energy, d, final_f, w, c, converged, history, terms)


# --------------------------------------------------------------- SAD guess
def atomic_density_guess(orb, symbols, charges_by_symbol) -> np.ndarray:
    """atoms.py:76-120: converge each distinct element once, place on the diagonal.

    ``orb`` is the molecular orbital shell table with ``shell_atoms``; every atom
    of one element carries the same shells, so the element is the cache key.
    """
    cache: dict[str, np.ndarray] = {}
    blocks = []
    for atom, symbol in enumerate(symbols):
        if symbol not in cache:
            cache[symbol] = spherical_atom(_atom_table(orb, atom), charges_by_symbol[symbol])
        blocks.append(cache[symbol])
    n = sum(b.shape[0] for b in blocks)
    d = np.zeros((n, n))
    start = 0
    for b in blocks:
        w = b.shape[0]
        d[start:start + w, start:start + w] = b
        start += w
    return d


class _Table:
    pass


def _atom_table(orb, atom: int):
    """The shells of one atom, centred at the origin (atoms.py:42-50, 55-64)."""
    sel = np.nonzero(np.asarray(orb.shell_atoms) == atom)[0]
    off = np.asarray(orb.primitive_offsets)
    k = np.asarray(orb.n_contractions)
    coef_off = np.concatenate([[0], np.cumsum(k * np.diff(off))])
    t = _Table()
    t.angular_momenta = np.asarray(orb.angular_momenta)[sel]
    t.centers = np.zeros((len(sel), 3))
    t.primitive_offsets = np.concatenate([[0], np.cumsum(np.diff(off)[sel])]).astype(np.int64)
    t.exponents = np.concatenate([np.asarray(orb.exponents)[off[i]:off[i + 1]] for i in sel])
    t.coefficients = np.concatenate([np.asarray(orb.coefficients)[coef_off[i]:coef_off[i + 1]] for i in sel])
    t.n_contractions = k[sel]
    return t


def spherical_atom(table, z: float) -> np.ndarray:
    """atoms.py:55-73: neutral atom, exact J/K, electrons averaged over both spins."""
    s = overlap(table)
    h = core_hamiltonian(table, np.array([z]), np.zeros((1, 3)))
    jk = ExactJK(eri_exact(table))
    result = solve_rhf(s, h, jk, 0.0, z / 2.0, averaged=True)
    return result.density


# ----------------------------------------------------------------- pipeline
@dataclass
class DfRhfProblem:
    s: np.ndarray
    h: np.ndarray
    b: np.ndarray
    e_nuc: float
    n_alpha: int
    metric: np.ndarray
    three_center: np.ndarray
    dropped: int


def build_problem(orb, aux, charges, positions, e_nuc: float, n_alpha: int) -> DfRhfProblem:
    """hartree_fock.py:88-191 molecular Hamiltonian with a fitted two-body term."""
    s = overlap(orb)
    h = core_hamiltonian(orb, charges, positions)
    m = metric(aux)
    t3 = three_center(aux, orb)
    half, dropped = inverse_square_root(m)
    b = (half @ t3.reshape(t3.shape[0], -1)).reshape(t3.shape)
    return DfRhfProblem(s, h, b, e_nuc, n_alpha, m, t3, dropped)


# ------------------------------------------------------------------ DF-MP2
def df_mp2(b: np.ndarray, mo_energies: np.ndarray, mo_coefficients: np.ndarray, n_occ: int) -> float:
    """hafnium/mp/mp2.py:135-176 for a restricted reference.

    The reference sums ``E2 = 1/4 sum_ijab |<ij||ab>|^2 / (e_i + e_j - e_a - e_b)``
    over spin orbitals with ``(ia|jb) = sum_P B[P,i,a] B[P,j,b]`` in the orbital
    basis (ADR-0030); for a closed shell the spin sums reduce to
    ``E2 = sum_ijab (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b)``
    over spatial orbitals, all electrons correlated.
    """
    order = np.argsort(mo_energies, kind="stable")
    e = mo_energies[order]
    c = mo_coefficients[:, order]
    co, cv = c[:, :n_occ], c[:, n_occ:]
    eo, ev = e[:n_occ], e[n_occ:]
    bov = np.einsum("pmn,mi,na->pia", b, co, cv, optimize=True)  # [aux, occ, vir]
    total = 0.0
    for i in range(n_occ):
        iajb = np.einsum("pa,pjb->jab", bov[:, i, :], bov, optimize=True)  # (ia|jb) for all j
        denom = eo[i] + eo[:, None, None] - ev[None, :, None] - ev[None, None, :]
        total += float(np.sum(iajb * (2.0 * iajb - iajb.transpose(0, 2, 1)) / denom))
    return total


# ------------------------------------------------------------ nuclear gradient
def functions_by_atom(table, positions: np.ndarray) -> np.ndarray:
    """gradient.py:158-168: ``[atom, ao]`` with one where the function sits on the atom.

    The reference reads the atom from each function's label; a molecular shell
    table carries the atom's position as the shell centre, so the atom is the
    one at that centre.
    """
    rows = []
    counts = getattr(table, "n_contractions", None)
    if counts is None:
        counts = table.contraction_counts
    for sh in range(len(table.angular_momenta)):
        dist = np.linalg.norm(np.asarray(positions) - np.asarray(table.centers[sh]), axis=1)
        atom = int(np.argmin(dist))
        if dist[atom] > 1e-10:
            raise ValueError(f"shell {sh} sits on no atom")
        rows += [atom] * (int(counts[sh]) * (2 * int(table.angular_momenta[sh]) + 1))
    out = np.zeros((len(positions), len(rows)))
    out[rows, np.arange(len(rows))] = 1.0
    return out


def _on_centers(derivative, weights, atoms):
    """gradient.py:171-178: 2 sum_{u on K} sum_v d[x,u,v] w[v,u] as [atom, 3]."""
    rows = 2.0 * np.einsum("xuv,vu->xu", derivative, weights)
    return (rows @ atoms.T).T


def _two_electron(metric_d, aux_d, orb_d, effective, metric_weights, atoms, aux_atoms):
    """gradient.py:181-203: gradient of sum_P tr(L_P G_P) + tr(M W) at fixed G and W."""
    symmetric = effective + np.transpose(effective, (0, 2, 1))
    on_auxiliary = np.einsum("xPuv,Puv->xP", aux_d, effective, optimize=True)
    on_auxiliary = on_auxiliary + 2.0 * np.einsum("xPQ,PQ->xP", metric_d, metric_weights)
    on_orbital = np.einsum("xPuv,Puv->xu", orb_d, symmetric, optimize=True)
    return (on_auxiliary @ aux_atoms.T + on_orbital @ atoms.T).T


def nuclear_repulsion_gradient(charges, positions) -> np.ndarray:
    """gradient.py:222-235: -sum_{L != K} Z_K Z_L (R_K - R_L) / |R_K - R_L|^3."""
    pos = np.asarray(positions, dtype=np.float64)
    z = np.asarray(charges, dtype=np.float64)
    sep = pos[:, None, :] - pos[None, :, :]
    dist = np.sqrt(np.sum(sep**2, axis=-1))
    eye = np.eye(len(z)) > 0
    w = np.where(eye, 0.0, z[:, None] * z[None, :] / np.where(eye, 1.0, dist) ** 3)
    return -np.sum(w[:, :, None] * sep, axis=1)


def nuclear_gradient(orb, aux, charges, positions, d_alpha, fock) -> dict:
    """gradient.py:72-149 for a restricted state: the five terms, each [atom, 3].

    ``d_alpha`` and ``fock`` are the converged alpha density and Fock matrix;
    the spin traces are ``total = 2 D`` and ``weighted = 2 D F D``, and the
    exchange pairs of the spin-orbital density reduce to ``T_Q = 2 D L_Q D``.
    """
    o, a = kernel_table(orb), kernel_table(aux)
    z3 = np.zeros((1, 3))
    total = 2.0 * d_alpha
    weighted = 2.0 * d_alpha @ fock @ d_alpha
    atoms = functions_by_atom(orb, positions)
    aux_atoms = functions_by_atom(aux, positions)
    by_center, by_nucleus = kernels.nuclear_attraction_derivative(o, o, z3, charges, positions)
    one_electron = _on_centers(kernels.kinetic_derivative(o, o, z3)[0] + by_center[0], total, atoms) + np.einsum(
        "kxuv,vu->kx", by_nucleus[0], total
    )
    overlap_term = -_on_centers(kernels.overlap_derivative(o, o, z3)[0], weighted, atoms)
    m = metric(aux)
    t3 = three_center(aux, orb)
    metric_d = kernels.coulomb_two_center_derivative(a, a, z3)[0]
    aux_d, orb_d = kernels.coulomb_three_center_derivative(a, o, o, np.zeros((1, 2, 3)))
    aux_d, orb_d = aux_d[0], orb_d[0]
    half, _ = inverse_square_root(m)
    inverse = half @ half
    fitted_charges = np.einsum("Puv,vu->P", t3, total)
    c = inverse @ fitted_charges
    coulomb_term = _two_electron(metric_d, aux_d, orb_d, c[:, None, None] * total[None, :, :],
                                 -0.5 * c[:, None] * c[None, :], atoms, aux_atoms)
    pairs = 2.0 * np.einsum("uv,Pvw,wx->Pux", d_alpha, t3, d_alpha, optimize=True)
    n = total.shape[0]
    exchange_pairs = t3.reshape(-1, n * n) @ np.transpose(pairs, (0, 2, 1)).reshape(-1, n * n).T
    exchange_term = _two_electron(metric_d, aux_d, orb_d, -np.einsum("PQ,Quv->Puv", inverse, pairs, optimize=True),
                                  0.5 * inverse @ exchange_pairs @ inverse, atoms, aux_atoms)
    return {
        "nuclear_repulsion": nuclear_repulsion_gradient(charges, positions),
        "one_electron": one_electron,
        "overlap": overlap_term,
        "coulomb": coulomb_term,
        "exchange": exchange_term,
    }
