"""Atom frames and the rotation of AO blocks between global and local frames.

Every atom gets a right-handed frame from its neighbours: x towards the nearest
atom, y towards the next atom that is not in line with the first (its part
orthogonal to x), z = x cross y. Neighbours at equal distance (to 1e-6 bohr) are
taken in atom order, so the frames depend only on the geometry's internal
coordinates and the atom order. A density block expressed in the frames of its
two atoms, D~_ij = U_i^T D_ij U_j, does not change when the whole molecule is
rotated or translated, which is what the network predicts. U_i rotates the
functions of atom i: 1 for s shells, the frame matrix for p shells (functions
ordered x, y, z) and the induced rotation of the sphere-normalised real solid
harmonics for d shells (hafnium/basis conventions, cartesian.rs:93-110).
"""

from __future__ import annotations

import functools
import math

import numpy as np


def _fact(n: int) -> float:
    return float(math.factorial(n))


def _binom(n: int, k: int) -> float:
    return float(math.comb(n, k)) if 0 <= k <= n else 0.0


def cartesian_components(l: int):
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


@functools.lru_cache(maxsize=None)
def solid_harmonics(l: int) -> np.ndarray:
    """[2l+1][ncart] Cartesian-to-spherical matrix (Helgaker 6.4.47, sphere-normalised)."""
    comps = cartesian_components(l)
    out = np.zeros((2 * l + 1, len(comps)))
    sphere = math.sqrt((2 * l + 1) / (4 * math.pi))
    ms = [1, -1, 0] if l == 1 else list(range(-l, l + 1))
    for row, m in enumerate(ms):
        am = abs(m)
        norm = math.sqrt(2 * _fact(l + am) * _fact(l - am) / (2.0 if m == 0 else 1.0)) / (2 ** am * _fact(l))
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                vmax = (am - 1) // 2 if m < 0 else am // 2
                for vh in range(vmax + 1):
                    two_v = 2 * vh + 1 if m < 0 else 2 * vh
                    if two_v > am:
                        continue
                    sign = 1.0 if (t + vh) % 2 == 0 else -1.0
                    c = sign * 0.25 ** t * _binom(l, t) * _binom(l - t, am + t) * _binom(t, u) * _binom(am, two_v)
                    py = 2 * u + two_v
                    px = 2 * t + am - py
                    pz = l - 2 * t - am
                    out[row, comps.index((px, py, pz))] += sphere * norm * c
    return out


def _monomials(points: np.ndarray, l: int) -> np.ndarray:
    comps = cartesian_components(l)
    return np.stack([points[:, 0] ** a * points[:, 1] ** b * points[:, 2] ** c for a, b, c in comps], axis=1)


def harmonic_rotation(r: np.ndarray, l: int) -> np.ndarray:
    """U with S_m(R^T x) = sum_m' S_m'(x) U[m', m]: the local function m in global terms."""
    if l == 0:
        return np.ones((1, 1))
    t = solid_harmonics(l)
    rng = np.random.default_rng(1234)
    pts = rng.normal(size=(64, 3))
    local = _monomials(pts @ r, l) @ t.T  # S_m(R^T x): rows x, columns m
    glob = _monomials(pts, l) @ t.T  # S_m'(x)
    u, *_ = np.linalg.lstsq(glob, local, rcond=None)
    return u


def atom_frames(positions: np.ndarray):
    """Frame matrices (columns: the local x, y, z axes in global coordinates) of
    every atom, or None when an atom has no two neighbours off one line (fewer
    than three atoms, or a linear molecule)."""
    pos = np.asarray(positions, dtype=np.float64)
    n = len(pos)
    if n < 3:
        return None
    rows = np.arange(n)
    diff = pos[None, :, :] - pos[:, None, :]  # [i, j] = r_j - r_i
    dist = np.linalg.norm(diff, axis=2)
    key = np.round(dist, 6)
    np.fill_diagonal(key, np.inf)  # the atom itself sorts last
    # neighbours nearest first, equal distances (to 1e-6 bohr) in atom order
    order = np.lexsort((np.broadcast_to(rows, (n, n)), key), axis=-1)
    first = order[:, 0]
    x = diff[rows, first] / dist[rows, first][:, None]
    cand = order[:, 1:n - 1]
    v = diff[rows[:, None], cand]
    v = v - np.einsum("ijk,ik->ij", v, x)[:, :, None] * x[:, None, :]
    norm = np.linalg.norm(v, axis=2)
    off_line = norm > 0.1 * dist[rows[:, None], cand]  # more than about 6 degrees off the x axis
    if not np.all(off_line.any(axis=1)):
        return None
    k = off_line.argmax(axis=1)
    y = v[rows, k] / norm[rows, k][:, None]
    return list(np.stack([x, y, np.cross(x, y)], axis=2))


def harmonic_rotations(frames, l: int) -> np.ndarray:
    """``harmonic_rotation`` of many frames at once: [frame, 2l+1, 2l+1]."""
    frames = np.asarray(frames, dtype=np.float64)
    if l == 0:
        return np.ones((len(frames), 1, 1))
    t = solid_harmonics(l)
    rng = np.random.default_rng(1234)
    pts = rng.normal(size=(64, 3))
    glob = _monomials(pts, l) @ t.T
    rotated = np.einsum("pk,fkj->fpj", pts, frames).reshape(-1, 3)  # pts @ r for every frame
    local = (_monomials(rotated, l) @ t.T).reshape(len(frames), 64, -1)
    return np.einsum("mp,fpn->fmn", np.linalg.pinv(glob), local)


def shell_layout(table, atom_index: int):
    """(l, n_contractions) of the shells on one atom of a ShellTable, in order."""
    sel = np.nonzero(np.asarray(table.shell_atoms) == atom_index)[0]
    return [(int(table.angular_momenta[s]), int(table.n_contractions[s])) for s in sel]


def ao_rotation(r: np.ndarray, layout) -> np.ndarray:
    """Block-diagonal U over the shells of ``layout`` (list of (l, n_contractions))."""
    return ao_rotations([r], [layout])[0]


def ao_rotations(frames, layouts):
    """``ao_rotation`` of every atom (frame and shell layout), with the rotation
    of each angular momentum formed for all atoms at once."""
    lmax = max((l for layout in layouts for l, _ in layout), default=0)
    per_l = [harmonic_rotations(frames, l) for l in range(lmax + 1)]
    out = []
    for a, layout in enumerate(layouts):
        blocks = []
        for l, k in layout:
            blocks.extend([per_l[l][a]] * k)
        n = sum(b.shape[0] for b in blocks)
        u = np.zeros((n, n))
        at = 0
        for b in blocks:
            m = b.shape[0]
            u[at:at + m, at:at + m] = b
            at += m
        out.append(u)
    return out
