"""DF-MP2 on the device from the fitted tensor the SCF already holds.

``df_mp2(ham, result)`` restates ``hafnium.mp.df_mp2`` (hafnium/mp/mp2.py:68-176)
for a restricted reference: the second-order energy
E2 = sum_ijab (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b) with
(ia|jb) from the same fitted tensor B as the SCF's J and K, all electrons
correlated, computed by ``hf_mp2_energy`` (DMMA transforms and pair GEMMs).
"""

from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Mp2Result:
    """hafnium/mp/mp2.py:37-65 (energies only; the amplitudes are not kept)."""

    reference_energy: float
    correlation_energy: float

    @property
    def total_energy(self) -> float:
        return self.reference_energy + self.correlation_energy


def df_mp2(ham, reference) -> Mp2Result:
    """Second-order energy of a converged restricted ``reference`` (a ScfResult of
    ``hafnium_b200.scf.solve_rhf`` on ``ham``)."""
    import torch

    order = torch.argsort(reference.mo_energies)
    c = reference.mo_coefficients[:, order].contiguous()
    e = reference.mo_energies[order].contiguous()
    context = ham.two_body.context
    correlation = context.mp2_energy(c, e, int(ham.n_alpha))
    return Mp2Result(float(reference.energy), correlation)
