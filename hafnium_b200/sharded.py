"""The fitted tensor of one molecule sharded over devices by auxiliary index.

B = L^-1 (P|uv) is split by rows: each rank of a process group holds the rows
[q0, q1) of its shard (``shard_rows``) on its own GPU. J and K are sums over the
auxiliary index (hafnium/scf/coulomb_exchange.py:176-190),

    J = sum_q (B_q . D) B_q,        K = sum_q B_q D B_q,

so every rank builds the partial sums over its rows and one all-reduce of the
n_ao x n_ao result per build completes them (18.9 MB at (H2O)64; NCCL over
NVLink on the GPU path, gloo on the host). The density is the same on every
rank, so the mixed-precision schedule (``MixedExchangeSchedule``) takes the
same decisions on all of them and the collectives stay in step. The metric is
factored in full on every rank (N^3/3 flops, small next to the fit).

``ShardedCoulombExchange`` satisfies the same ``CoulombExchange`` protocol as
``B200DensityFittedCoulombExchange``; ``local`` is any builder with the
protocol's methods whose results are its rows' partial sums (on the GPU a
``B200DensityFittedCoulombExchange`` built with ``rows=shard_rows(...)``).
"""

from __future__ import annotations

import numpy as np

from hafnium_b200.errors import InputError


def shard_rows(n_aux: int, world_size: int, rank: int) -> tuple[int, int]:
    """Rows [q0, q1) of rank ``rank``: contiguous, as equal as possible (the J and
    K builds, repeated every iteration, cost in proportion to the rows)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise InputError(f"rank {rank} is not in a group of {world_size}")
    if n_aux < world_size:
        raise InputError(f"{n_aux} auxiliary functions cannot be split over {world_size} ranks")
    base, extra = divmod(n_aux, world_size)
    q0 = rank * base + min(rank, extra)
    return q0, q0 + base + (1 if rank < extra else 0)


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


class ShardedCoulombExchange:
    """J and K over the shards of a process group (every rank calls every method
    with the same density, in the same order)."""

    def __init__(self, local, group=None, schedule: str = "fp64") -> None:
        self.local = local
        self.group = group
        self.context = getattr(local, "context", None)
        if schedule not in ("fp64", "mixed"):
            raise InputError("the exchange schedule is 'fp64' or 'mixed'")
        if schedule == "mixed":
            from hafnium_b200.jk import MixedExchangeSchedule

            self.schedule = MixedExchangeSchedule(self)
        else:
            self.schedule = None

    @property
    def n_ao(self) -> int:
        return self.local.n_ao

    @property
    def n_aux(self) -> int:
        return self.local.n_aux

    def _sum(self, partial):
        """The sum of every rank's ``partial`` (torch tensors in place, NumPy arrays
        through a host tensor)."""
        import torch
        import torch.distributed as dist

        if _is_torch(partial):
            dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=self.group)
            return partial
        t = torch.from_numpy(np.ascontiguousarray(partial))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t.numpy()

    def coulomb(self, density):
        """``J = sum over all ranks' rows of (B_q . D) B_q``."""
        return self._sum(self.local.coulomb(density))

    def exchange(self, density):
        """``K = sum over all ranks' rows of B_q D B_q``; with the mixed schedule the
        arithmetic of each build follows ``MixedExchangeSchedule``."""
        if self.schedule is not None:
            import torch

            on_device = _is_torch(density) and density.is_cuda
            index = getattr(self.context, "device", None)
            d = density if on_device else torch.as_tensor(np.asarray(density, dtype=np.float64))
            d = d.to(torch.device("cuda", index) if index is not None else d.device, torch.float64).contiguous()
            k = self.schedule.exchange(d)
            return k if on_device else k.cpu().numpy()
        return self._sum(self.local.exchange(density))

    def exchange_factored(self, factor, weights=None, precision=None):
        """``K`` for ``D = C diag(w) C^T``, summed over the ranks."""
        return self._sum(self.local.exchange_factored(factor, weights, precision))
