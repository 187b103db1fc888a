"""Device J and K against the oracle's restatement of coulomb_exchange.py (B200)."""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200.jk import B200DensityFittedCoulombExchange
from oracle import dfrhf
from tests.helpers import molecule, tables

pytestmark = pytest.mark.gpu
JK_TOL = 1e-10


@pytest.fixture(scope="module", params=["water", "h2o2_s0", "h2o4_s1"])
def system(request):
    mol = molecule(request.param)
    orb, aux = tables(mol)
    two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    b = dfrhf.df_tensor(dfrhf.metric(aux), dfrhf.three_center(aux, orb))
    return two_body, b


def psd_density(n, rank, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n, rank)) / np.sqrt(n)
    return c @ c.T, c


def test_coulomb_matches_oracle(system):
    two_body, b = system
    d, _ = psd_density(two_body.n_ao, 7, 0)
    np.testing.assert_allclose(two_body.coulomb(d), dfrhf.coulomb(b, d), atol=JK_TOL, rtol=0)


def test_coulomb_of_a_nonsymmetric_density(system):
    """J only sees the symmetric part, as with the reference's full contraction."""
    two_body, b = system
    rng = np.random.default_rng(1)
    d = rng.normal(size=(two_body.n_ao, two_body.n_ao)) * 0.1
    sym = 0.5 * (d + d.T)
    np.testing.assert_allclose(two_body.coulomb(sym), dfrhf.coulomb(b, sym), atol=JK_TOL, rtol=0)


def test_exchange_matches_oracle_psd(system):
    two_body, b = system
    d, c = psd_density(two_body.n_ao, 9, 2)
    np.testing.assert_allclose(two_body.exchange(d), dfrhf.exchange(b, d), atol=JK_TOL, rtol=0)
    np.testing.assert_allclose(two_body.exchange_factored(c), dfrhf.exchange(b, d), atol=JK_TOL, rtol=0)


def test_exchange_of_an_indefinite_density(system):
    two_body, b = system
    d1, _ = psd_density(two_body.n_ao, 5, 3)
    d2, _ = psd_density(two_body.n_ao, 4, 4)
    d = d1 - 0.7 * d2
    np.testing.assert_allclose(two_body.exchange(d), dfrhf.exchange(b, d), atol=JK_TOL, rtol=0)


def test_signed_factor_weights(system):
    two_body, b = system
    rng = np.random.default_rng(5)
    c = rng.normal(size=(two_body.n_ao, 6)) / np.sqrt(two_body.n_ao)
    w = np.array([1.0, -1.0, 0.5, 2.0, -0.25, 1.0])
    d = (c * w) @ c.T
    np.testing.assert_allclose(two_body.exchange_factored(c, w), dfrhf.exchange(b, d), atol=JK_TOL, rtol=0)


def test_device_tensors_stay_on_device(system):
    import torch

    two_body, b = system
    d, _ = psd_density(two_body.n_ao, 6, 6)
    dt = torch.as_tensor(d, device="cuda")
    j = two_body.coulomb(dt)
    k = two_body.exchange(dt)
    assert j.is_cuda and k.is_cuda
    np.testing.assert_allclose(j.cpu().numpy(), dfrhf.coulomb(b, d), atol=JK_TOL, rtol=0)
    np.testing.assert_allclose(k.cpu().numpy(), dfrhf.exchange(b, d), atol=JK_TOL, rtol=0)


def test_shape_mismatch_raises(system):
    from hafnium_b200.errors import InputError

    two_body, _ = system
    with pytest.raises(InputError):
        two_body.coulomb(np.zeros((3, 3)))


def test_a_rebuilt_context_takes_the_retained_fitted_tensor_block():
    """The fitted tensor of (H2O)16 (1.2 GB, above the stream-ordered pool's
    256 MiB) is kept when its context closes and handed to the next context of
    that size, so the second build makes one device allocation fewer and gives
    the same J."""
    import torch

    from hafnium_b200 import _lib

    _lib.release_retained(0)
    mol = molecule("h2o16_s0")
    orb, aux = tables(mol)
    counts, coulombs = [], []
    rng = np.random.default_rng(2)
    for _ in range(2):
        two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux)
        if not coulombs:
            c = rng.normal(size=(two_body.n_ao, 30)) / np.sqrt(two_body.n_ao)
            d = torch.as_tensor(c @ c.T, device="cuda")
        counts.append(two_body.stats()["device_allocations"])
        coulombs.append(two_body.coulomb(d).cpu().numpy())
        two_body.context.close()
    assert counts[1] == counts[0] - 1
    np.testing.assert_allclose(coulombs[0], coulombs[1], atol=1e-13, rtol=0)
    _lib.release_retained(0)


@pytest.mark.parametrize("tag", ["h2o4_s1", "h2o12_s3"])
def test_row_shards_of_the_fitted_tensor_sum_to_the_whole(tag):
    """Three contexts holding rows [0, q1), [q1, q2), [q2, N) of B (the split a
    process group over three GPUs would make, here on one GPU): their J and K
    add up to the whole tensor's, in FP64 to 1e-10 and split-BF16 to the split's
    own error; a shard refuses what needs every row."""
    import torch

    from hafnium_b200 import _lib
    from hafnium_b200.errors import InputError
    from hafnium_b200.sharded import shard_rows

    mol = molecule(tag)
    orb, aux = tables(mol)
    whole = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    shards = [B200DensityFittedCoulombExchange.from_tables(orb, aux, rows=shard_rows(whole.n_aux, 3, r))
              for r in range(3)]
    d, c = psd_density(whole.n_ao, 25, 4)
    dt = torch.as_tensor(d, device="cuda")
    ct = torch.as_tensor(c, device="cuda")
    j = sum(s.coulomb(dt) for s in shards)
    k = sum(s.exchange(dt) for s in shards)
    np.testing.assert_allclose(j.cpu().numpy(), whole.coulomb(d), atol=JK_TOL, rtol=0)
    np.testing.assert_allclose(k.cpu().numpy(), whole.exchange(d), atol=JK_TOL, rtol=0)
    k16 = sum(s.exchange_factored(ct, precision=_lib.PREC_BF16X3) for s in shards).cpu().numpy()
    k64 = whole.exchange_factored(c)
    assert np.max(np.abs(k16 - k64)) <= 1e-4 * np.max(np.abs(k64))
    assert sum(s.stats()["b_bytes"] for s in shards) == whole.stats()["b_bytes"]
    with pytest.raises(InputError, match="every row"):
        shards[1].orbital_tensor(c[:, :3], c[:, :3])


def test_sharded_builder_over_a_one_rank_nccl_group():
    """The sharded builder's collectives on device tensors through NCCL (a group of
    one rank on this GPU): J and K of the whole tensor, FP64 and the mixed
    schedule's first (split-BF16) build."""
    import os

    import torch
    import torch.distributed as dist

    from hafnium_b200.sharded import ShardedCoulombExchange, shard_rows

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", str(29650 + os.getpid() % 300))
    created = not dist.is_initialized()
    if created:
        dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        mol = molecule("h2o4_s1")
        orb, aux = tables(mol)
        whole = B200DensityFittedCoulombExchange.from_tables(orb, aux)
        local = B200DensityFittedCoulombExchange.from_tables(orb, aux, rows=shard_rows(whole.n_aux, 1, 0))
        sharded = ShardedCoulombExchange(local)
        mixed = ShardedCoulombExchange(
            B200DensityFittedCoulombExchange.from_tables(orb, aux, rows=shard_rows(whole.n_aux, 1, 0)),
            schedule="mixed")
        d, c = psd_density(whole.n_ao, 20, 6)
        dt = torch.as_tensor(d, device="cuda")
        np.testing.assert_allclose(sharded.coulomb(dt).cpu().numpy(), whole.coulomb(d), atol=JK_TOL, rtol=0)
        np.testing.assert_allclose(sharded.exchange(dt).cpu().numpy(), whole.exchange(d), atol=JK_TOL, rtol=0)
        k16 = mixed.exchange(d)  # host arrays in and out, the first build is split-BF16
        k64 = whole.exchange(d)
        assert mixed.schedule.log[-1]["precision"] == "bf16"
        assert np.max(np.abs(k16 - k64)) <= 1e-4 * np.max(np.abs(k64))
    finally:
        if created:
            dist.destroy_process_group()


@pytest.mark.parametrize("rank", [1, 20, 33, 70])
def test_density_factor_reproduces_a_semidefinite_density(system, rank):
    """hf_density_factor (the blocked pivoted Cholesky: panels of 32 pivots) finds the
    density's rank and a factor with F F^T = D, across panel boundaries; a rank limit
    stops it early, and an indefinite density is refused."""
    import torch

    from hafnium_b200.errors import InputError

    two_body, _ = system
    n = two_body.n_ao
    r = max(1, min(rank, n - 4))
    rng = np.random.default_rng(rank)
    c = rng.normal(size=(n, r)) / np.sqrt(n)
    d = c @ c.T
    dt = torch.as_tensor(d, device="cuda")
    f = two_body.context.density_factor_device(dt, n)
    # the rank, up to pivots on rounding residues just above the 1e-14 cut
    assert f.shape[0] == n and r <= f.shape[1] <= r + 2
    np.testing.assert_allclose((f @ f.T).cpu().numpy(), d, atol=1e-12 * np.abs(d).max(), rtol=0)
    limit = max(1, r // 2)
    assert two_body.context.density_factor_device(dt, limit).shape[1] == limit
    bad = d - 3.0 * np.abs(d).max() * np.outer(np.eye(n)[0], np.eye(n)[0])
    with pytest.raises(InputError, match="semidefinite"):
        two_body.context.density_factor_device(torch.as_tensor(bad, device="cuda"), n)
