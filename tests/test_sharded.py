"""The fitted tensor sharded by auxiliary index over two gloo ranks (CPU).

Each rank holds rows [q0, q1) of the oracle's fitted tensor of a water dimer
(cc-pVDZ / def2-universal-jkfit); the partial J and K over its rows, summed by
``ShardedCoulombExchange``'s all-reduce, must equal the oracle's J and K of
the whole tensor (coulomb_exchange.py:176-190). With the mixed schedule both
ranks must take the same arithmetic at every call (the collectives stay in
step) and agree with the unsharded schedule.
"""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from hafnium_b200 import _lib
from hafnium_b200.errors import InputError
from hafnium_b200.sharded import ShardedCoulombExchange, shard_rows


def test_shard_rows_cover_every_row_once():
    for n_aux, world in ((904, 2), (7232, 8), (113, 3), (5, 5)):
        rows = [shard_rows(n_aux, world, r) for r in range(world)]
        assert rows[0][0] == 0 and rows[-1][1] == n_aux
        assert all(rows[r][1] == rows[r + 1][0] for r in range(world - 1))
        sizes = [q1 - q0 for q0, q1 in rows]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(InputError):
        shard_rows(3, 4, 0)
    with pytest.raises(InputError):
        shard_rows(10, 2, 2)


class RowsBuilder:
    """Partial J and K over rows [q0, q1) of a full B[aux, ao, ao] (host torch)."""

    def __init__(self, b: np.ndarray, rows) -> None:
        self.b = torch.as_tensor(b[rows[0]:rows[1]])
        self.n_ao = b.shape[1]
        self.n_aux = b.shape[0]
        self.context = HostContext()

    def coulomb(self, d):
        d = torch.as_tensor(d)
        charges = torch.einsum("quv,uv->q", self.b, d)
        return torch.einsum("q,quv->uv", charges, self.b).numpy()

    def exchange(self, d):
        d = torch.as_tensor(d)
        return torch.einsum("quw,wx,qxv->uv", self.b, d, self.b).numpy()

    def exchange_factored(self, factor, weights=None, precision=None):
        x = torch.einsum("quv,vi->qui", self.b, factor)
        k = torch.einsum("qui,qwi->uw", x, x)
        if precision == _lib.PREC_BF16X3:
            k = k * (1.0 + 1e-5)  # a stand-in for the split-BF16 rounding
        return k


class HostContext:
    device = None

    def density_factor_device(self, d, max_rank):
        w, v = torch.linalg.eigh(0.5 * (d + d.T))
        keep = w > 1e-14 * w.abs().max()
        return (v[:, keep] * w[keep].sqrt()).contiguous()

    def overlap_device(self):
        return self.s


def _problem():
    from hafnium_b200.basis import ShellTable
    from hafnium_b200.molecule import water_cluster
    from oracle import dfrhf

    mol = water_cluster(2, 0)
    orb = ShellTable.build("cc-pvdz", mol.symbols, mol.positions)
    aux = ShellTable.build("def2-universal-jkfit", mol.symbols, mol.positions)
    b = dfrhf.df_tensor(dfrhf.metric(aux), dfrhf.three_center(aux, orb))
    s = dfrhf.overlap(orb)
    return b, s


def _densities(s: np.ndarray, count: int):
    """A converging sequence of PSD densities of rank 10 (S-orthonormal factors)."""
    rng = np.random.default_rng(7)
    n = s.shape[0]
    w, v = np.linalg.eigh(s)
    s_half_inv = (v / np.sqrt(w)) @ v.T
    q0, _ = np.linalg.qr(rng.normal(size=(n, 10)))
    q1, _ = np.linalg.qr(q0 + 0.05 * rng.normal(size=(n, 10)))
    out = []
    for step in range(count):
        t = 0.5 ** step
        q, _ = np.linalg.qr(q1 + t * (q0 - q1))
        c = s_half_inv @ q
        out.append(c @ c.T)
    return out


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    from oracle import dfrhf

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        b, s = _problem()
        rows = shard_rows(b.shape[0], world, rank)
        local = RowsBuilder(b, rows)
        local.context.s = torch.as_tensor(s)
        sharded = ShardedCoulombExchange(local)
        d = _densities(s, 1)[0]
        j_err = float(np.max(np.abs(sharded.coulomb(d) - dfrhf.coulomb(b, d))))
        k_err = float(np.max(np.abs(sharded.exchange(d) - dfrhf.exchange(b, d))))
        mixed_local = RowsBuilder(b, rows)
        mixed_local.context.s = torch.as_tensor(s)
        mixed = ShardedCoulombExchange(mixed_local, schedule="mixed")
        mixed.schedule.anchor_change, mixed.schedule.final_change = 1e-2, 1e-4
        ks = [mixed.exchange(dk) for dk in _densities(s, 20)]
        kinds = [e["precision"] for e in mixed.schedule.log]
        out.put((rank, j_err, k_err, kinds, ks[-1]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_shards_sum_to_the_full_fitted_jk():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29800 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {r: rest for r, *rest in (q.get(timeout=120) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        j_err, k_err, _, _ = results[r]
        assert j_err < 1e-12 and k_err < 1e-12
    # the mixed schedule: the same decisions on both ranks, the same K, and the
    # arithmetic of the unsharded schedule on the whole tensor
    assert results[0][2] == results[1][2]
    np.testing.assert_array_equal(results[0][3], results[1][3])
    kinds = results[0][2]
    assert kinds[0] == "bf16" and "anchor" in kinds and "incremental" in kinds
    b, s = _problem()
    whole = RowsBuilder(b, (0, b.shape[0]))
    whole.context.s = torch.as_tensor(s)
    from hafnium_b200.jk import MixedExchangeSchedule

    reference = MixedExchangeSchedule(whole, anchor_change=1e-2, final_change=1e-4)
    k_last = None
    for dk in _densities(s, 20):
        k_last = reference.exchange(torch.as_tensor(dk))
    assert [e["precision"] for e in reference.log] == kinds
    np.testing.assert_allclose(results[0][3], k_last.numpy(), atol=1e-12, rtol=0)
