"""Water frames and the rotation of AO blocks between global and local frames.

Each rigid water (atoms O, H, H) defines a right-handed frame: x along the HOH
bisector, z along the plane normal (H1 - O) x (H2 - O), y = z x x. A density
block expressed in the frames of its two waters, D~_ij = U_i^T D_ij U_j, does not
change when the whole cluster is rotated or translated, which is what the
network predicts. U_i rotates the cc-pVDZ functions of water i: 1 for s shells,
the frame matrix for p shells (functions ordered x, y, z) and the induced 5x5
rotation of the sphere-normalised real solid harmonics for d shells
(hafnium/basis conventions, cartesian.rs:93-110).
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


def water_frame(o: np.ndarray, h1: np.ndarray, h2: np.ndarray) -> np.ndarray:
    """Columns: the local x, y, z axes in global coordinates."""
    x = (h1 - o) + (h2 - o)
    x /= np.linalg.norm(x)
    z = np.cross(h1 - o, h2 - o)
    z /= np.linalg.norm(z)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)


def shell_layout(table, atom_index: int):
    """(l, n_contractions) of the shells on one atom of a ShellTable, in order."""
    sel = np.nonzero(np.asarray(table.shell_atoms) == atom_index)[0]
    return [(int(table.angular_momenta[s]), int(table.n_contractions[s])) for s in sel]


def ao_rotation(r: np.ndarray, layout) -> np.ndarray:
    """Block-diagonal U over the shells of ``layout`` (list of (l, n_contractions))."""
    blocks = []
    for l, k in layout:
        u = harmonic_rotation(r, l)
        blocks.extend([u] * k)
    n = sum(b.shape[0] for b in blocks)
    out = np.zeros((n, n))
    at = 0
    for b in blocks:
        m = b.shape[0]
        out[at:at + m, at:at + m] = b
        at += m
    return out


def cluster_frames(molecule):
    """Per water: origin (O position) and frame matrix; atoms ordered O, H, H."""
    pos = np.asarray(molecule.positions)
    nw = len(molecule.symbols) // 3
    frames = []
    for w in range(nw):
        o, h1, h2 = pos[3 * w], pos[3 * w + 1], pos[3 * w + 2]
        frames.append((o, water_frame(o, h1, h2)))
    return frames
