"""Analytic nuclear gradient of the DF-RHF energy on the device.

``nuclear_gradient(ham, result, molecule)`` restates
``hafnium.properties.nuclear_gradient`` (hafnium/properties/gradient.py:72-149)
for a converged closed-shell state: the same five terms (nuclear repulsion,
one-electron, overlap, Coulomb, exchange), the same effective densities
(``c_P D`` and ``-sum_Q M^-1_PQ T_Q`` with the metric weights ``-c c^T / 2``
and ``M^-1 E M^-1 / 2``), computed by ``hf_nuclear_gradient``: the effective
densities by DMMA GEMMs in the occupied basis, ``Gamma_P = C^T (L^-T B)_P C``,
and every derivative integral contracted with its weight as it is formed.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class NuclearGradient:
    """gradient.py:44-69: each term [atom, 3] in Hartree per Bohr."""

    nuclear_repulsion: np.ndarray
    one_electron: np.ndarray
    overlap: np.ndarray
    coulomb: np.ndarray
    exchange: np.ndarray

    @property
    def total(self) -> np.ndarray:
        return self.nuclear_repulsion + self.one_electron + self.overlap + self.coulomb + self.exchange


def occupied_factor(density: np.ndarray, overlap: np.ndarray, n_occ: int) -> np.ndarray:
    """C [n, n_occ] with C C^T = D for an idempotent closed-shell density D
    (D S D = D): the eigenvectors of S^1/2 D S^1/2 with eigenvalue one, back
    transformed by S^-1/2. For a state given only as its density and Fock
    matrix, as the reference's ScfResult gives it."""
    w, v = np.linalg.eigh(overlap)
    half = (v * np.sqrt(w)) @ v.T
    inv_half = (v / np.sqrt(w)) @ v.T
    occ_w, occ_v = np.linalg.eigh(half @ density @ half)
    keep = np.argsort(occ_w)[::-1][:n_occ]
    return inv_half @ occ_v[:, keep]


def gradient_from_state(two_body, occupied, fock, molecule) -> NuclearGradient:
    """The gradient of the state whose occupied orbitals (torch CUDA tensor or
    NumPy [n, n_occ]) and Fock matrix are given, for the molecule's nuclei."""
    if hasattr(occupied, "data_ptr"):
        d = occupied @ occupied.T
        weighted = 2.0 * d @ fock @ d
    else:
        occupied = np.asarray(occupied, dtype=np.float64)
        d = occupied @ occupied.T
        weighted = 2.0 * d @ np.asarray(fock, dtype=np.float64) @ d
    terms = two_body.context.nuclear_gradient(occupied, weighted, molecule.nuclear_charges, molecule.positions)
    return NuclearGradient(*terms)


def nuclear_gradient(ham, result, molecule) -> NuclearGradient:
    """Gradient of a converged restricted ``result`` (a ScfResult of
    ``hafnium_b200.scf.solve_rhf`` on ``ham``) of ``molecule``."""
    import torch

    if not result.converged:
        raise ValueError("the gradient of an unconverged state is not first order in its error")
    order = torch.argsort(result.mo_energies, stable=True)
    occupied = result.mo_coefficients[:, order[: int(ham.n_alpha)]].contiguous()
    return gradient_from_state(ham.two_body, occupied, result.fock, molecule)
