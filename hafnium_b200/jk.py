"""The drop-in two-electron builder: ``CoulombExchange`` over a device-resident B.

``B200DensityFittedCoulombExchange`` satisfies hafnium's ``CoulombExchange``
protocol (hafnium/scf/coulomb_exchange.py:53-71) with the constructor of
``DensityFittedCoulombExchange.from_molecule`` (coulomb_exchange.py:148-164):

    two_body = B200DensityFittedCoulombExchange.from_molecule(engine, basis, auxiliary, molecule)
    hamiltonian = Hamiltonian.from_molecule(engine, basis, molecule, two_body)
    result = solve_scf(hamiltonian, SymmetrySpec.from_name("RHF"))

``coulomb(D)`` and ``exchange(D)`` take and return ``[n_ao, n_ao]`` float64
arrays: NumPy arrays (the reference's host backend) stay NumPy, and CUDA
tensors stay on the device. The metric, the three-centre integrals, the
Cholesky factorisation and B = L^-1 (P|uv) are built on the GPU by
``libhfjk.so``; the ``engine`` argument is accepted for signature parity and
not used.
"""

from __future__ import annotations

import numpy as np

from hafnium_b200 import _lib
from hafnium_b200.basis import ShellTable
from hafnium_b200.errors import InputError


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


class B200DensityFittedCoulombExchange:
    """J and K from the packed fitted tensor on one B200."""

    def __init__(self, context: _lib.Context, precision: int = _lib.PREC_FP64) -> None:
        self.context = context
        self._n_ao, self._n_aux = context.dims()
        self.precision = precision

    @classmethod
    def from_tables(cls, orbital, auxiliary, *, device: int = 0, precision: int = _lib.PREC_FP64):
        """Build from structure-of-arrays shell tables (``hafnium_b200.basis.ShellTable``
        or the reference's own ``hafnium.integrals.ShellTable``)."""
        context = _lib.Context(device)
        context.upload(orbital, auxiliary)
        context.build()
        return cls(context, precision)

    @classmethod
    def from_molecule(cls, engine, basis, auxiliary, molecule, *, omega: float | None = None, device: int = 0,
                      precision: int = _lib.PREC_FP64):
        """Fit the integrals of ``molecule`` in ``auxiliary`` (coulomb_exchange.py:148-164).

        ``basis``/``auxiliary`` are reference ``BasisSet`` objects (or basis names
        when ``molecule`` is a ``hafnium_b200.molecule.Molecule``). The long-range
        kernel (``omega``) is not built on the device.
        """
        del engine
        if omega is not None:
            raise InputError("the range-separated (omega) kernel is not available on the device")
        if isinstance(basis, str):
            orbital = ShellTable.build(basis, molecule.symbols, molecule.positions)
            aux = ShellTable.build(auxiliary, molecule.symbols, molecule.positions)
        else:
            orbital = ShellTable.from_reference(basis, molecule)
            aux = ShellTable.from_reference(auxiliary, molecule)
        return cls.from_tables(orbital, aux, device=device, precision=precision)

    @property
    def n_ao(self) -> int:
        """Number of atomic orbitals."""
        return self._n_ao

    @property
    def n_aux(self) -> int:
        """Number of auxiliary functions."""
        return self._n_aux

    def _check(self, density) -> None:
        shape = tuple(density.shape)
        if shape != (self._n_ao, self._n_ao):
            raise InputError(f"the density has shape {list(shape)}, the integrals {self._n_ao} atomic orbitals")

    def coulomb(self, density):
        """``J[u, v] = sum_wx (uv|wx) D[w, x]`` (coulomb_exchange.py:176-182)."""
        self._check(density)
        if _is_torch(density) and density.is_cuda:
            import torch

            d = density.to(torch.float64).contiguous()
            out = torch.empty_like(d)
            self.context.coulomb_device(d, out)
            return out
        return self.context.coulomb_host(np.asarray(density, dtype=np.float64))

    def exchange(self, density):
        """``K[u, v] = sum_wx (uw|xv) D[w, x]`` (coulomb_exchange.py:184-190).

        A positive semidefinite density (every density the SCF driver passes) is
        factorised on the device by a pivoted Cholesky; an indefinite one by a
        device eigendecomposition into a signed factor.
        """
        self._check(density)
        on_device = _is_torch(density) and density.is_cuda
        try:
            if on_device:
                import torch

                d = density.to(torch.float64).contiguous()
                out = torch.empty_like(d)
                self.context.exchange_device(d, out, self.precision)
                return out
            return self.context.exchange_host(np.asarray(density, dtype=np.float64), self.precision)
        except InputError as error:
            if "semidefinite" not in str(error):
                raise
        return self._exchange_signed(density, on_device)

    def _exchange_signed(self, density, on_device: bool):
        import torch

        dev = torch.device("cuda", self.context.device)
        d = (density if on_device else torch.as_tensor(np.asarray(density, dtype=np.float64))).to(dev, torch.float64)
        d = 0.5 * (d + d.T)
        w, v = torch.linalg.eigh(d)
        keep = w.abs() > 1e-14 * w.abs().max()
        c = (v[:, keep] * w[keep].abs().sqrt()).contiguous()
        sign = torch.sign(w[keep]).contiguous()
        out = torch.empty_like(d)
        self.context.exchange_factored_device(c, out, sign, self.precision)
        return out if on_device else out.cpu().numpy()

    def orbital_tensor(self, c_bra, c_ket):
        """``B[P, p, q]`` in an orbital basis (hafnium/orbitals/integrals.py:73-157,
        ``transform_df_tensor`` for restricted real orbitals): ``[aux, n_bra, n_ket]``
        from ``C`` blocks ``[n_ao, n_bra]`` and ``[n_ao, n_ket]``. The auxiliary index
        is the Cholesky gauge of this fitting; contractions over it are the
        reference's."""
        return self.context.mo_fitted_tensor(c_bra, c_ket)

    def exchange_factored(self, factor, weights=None, precision: int | None = None):
        """``K`` for ``D = C diag(w) C^T`` with ``C`` of shape ``[n_ao, k]``."""
        prec = self.precision if precision is None else precision
        if _is_torch(factor) and factor.is_cuda:
            import torch

            out = torch.empty((self._n_ao, self._n_ao), dtype=torch.float64, device=factor.device)
            self.context.exchange_factored_device(factor.contiguous(), out, weights, prec)
            return out
        return self.context.exchange_factored_host(np.asarray(factor), weights, prec)

    def context_exchange_bf16(self, density):
        """Split-BF16 K of a positive semidefinite device density."""
        import torch

        d = density.to(torch.float64).contiguous()
        out = torch.empty_like(d)
        self.context.exchange_device(d, out, _lib.PREC_BF16X3)
        return out

    def stats(self) -> dict:
        return self.context.stats()
