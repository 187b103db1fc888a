"""Split-BF16 exchange on tcgen05 against the FP64 exchange (B200).

Three BF16 products (hi*hi + hi*lo + lo*hi) keep about 16 significant bits of
each operand, and the FP32 accumulation over N * n_cols terms adds rounding that
grows with the length of the sum. The bound checked here is 1e-4 of the largest
|K| element; observed errors are 1e-5 to 5.5e-5 of it, the largest for
n = 288 (padded to 384), N = 1356, 300 columns.
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200 import _lib
from hafnium_b200.jk import B200DensityFittedCoulombExchange
from hafnium_b200.molecule import water_cluster
from tests.helpers import molecule, tables

pytestmark = pytest.mark.gpu
REL_TOL = 1e-4


@pytest.fixture(scope="module", params=["water", "h2o4_s1", "h2o8_s2", "h2o12_s3"])
def two_body(request):
    # (H2O)12 has n = 288, padded to 384 = 3 x 128: stage 2's column tiles must then be
    # 128 wide (256-wide tiles would leave the last 128 columns of K out)
    mol = water_cluster(12, 3) if request.param == "h2o12_s3" else molecule(request.param)
    orb, aux = tables(mol)
    return B200DensityFittedCoulombExchange.from_tables(orb, aux)


@pytest.mark.parametrize("ncols", [5, 40, 300])
def test_bf16_factored_exchange_matches_fp64(two_body, ncols):
    rng = np.random.default_rng(ncols)
    c = rng.normal(size=(two_body.n_ao, ncols)) / np.sqrt(two_body.n_ao * ncols)
    ctx = two_body.context
    k64 = ctx.exchange_factored_host(c, None, _lib.PREC_FP64)
    k16 = ctx.exchange_factored_host(c, None, _lib.PREC_BF16X3)
    scale = np.max(np.abs(k64))
    err = np.max(np.abs(k16 - k64))
    print(f"n={two_body.n_ao} ncols={ncols}: max|K16-K64| = {err:.2e}, relative {err / scale:.2e}")
    assert err <= REL_TOL * scale
    np.testing.assert_allclose(k16, k16.T, atol=0, rtol=0)


def test_bf16_exchange_from_a_density(two_body):
    rng = np.random.default_rng(3)
    c = rng.normal(size=(two_body.n_ao, 12)) / np.sqrt(two_body.n_ao)
    d = c @ c.T
    ctx = two_body.context
    k64 = ctx.exchange_host(d, _lib.PREC_FP64)
    k16 = ctx.exchange_host(d, _lib.PREC_BF16X3)
    assert np.max(np.abs(k16 - k64)) <= REL_TOL * np.max(np.abs(k64))


def test_bf16_signed_factor_matches_fp64(two_body):
    """D = C diag(w) C^T with weights of both signs (the incremental builds'
    difference densities): one split-BF16 build against the FP64 one, the error
    relative to the larger of the positive and negative parts."""
    rng = np.random.default_rng(11)
    k = 20
    c = rng.normal(size=(two_body.n_ao, 2 * k)) / np.sqrt(two_body.n_ao * k)
    w = np.concatenate([np.full(k, 1.0), np.full(k, -0.7)])
    ctx = two_body.context
    k64 = ctx.exchange_factored_host(c, w, _lib.PREC_FP64)
    k16 = ctx.exchange_factored_host(c, w, _lib.PREC_BF16X3)
    scale = max(np.max(np.abs(ctx.exchange_factored_host(c[:, :k], None, _lib.PREC_FP64))),
                0.7 * np.max(np.abs(ctx.exchange_factored_host(c[:, k:], None, _lib.PREC_FP64))))
    assert np.max(np.abs(k16 - k64)) <= REL_TOL * scale
    np.testing.assert_allclose(k16, k16.T, atol=0, rtol=0)


def test_bf16_exchange_is_reproducible(two_body):
    """Stage 2 sums its k splits in a fixed order: two builds give the same bits."""
    rng = np.random.default_rng(7)
    c = rng.normal(size=(two_body.n_ao, 50)) / np.sqrt(two_body.n_ao * 50)
    ctx = two_body.context
    first = ctx.exchange_factored_host(c, None, _lib.PREC_BF16X3)
    second = ctx.exchange_factored_host(c, None, _lib.PREC_BF16X3)
    assert np.array_equal(first, second)


def test_a_device_wait_that_runs_out_is_reported_and_the_context_recovers():
    """The pipeline's bounded waits: the stall self-test makes the MMA thread wait
    on a barrier that nothing completes; with a 1 ms limit the wait runs out, the
    kernel ends (copies drained, tensor memory freed) and the build reports
    HF_ERR_TIMEOUT as BackendError. The next build on the same context, at the
    default limit, is correct again."""
    from hafnium_b200.errors import BackendError, InputError

    mol = molecule("h2o4_s1")
    orb, aux = tables(mol)
    two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    ctx = two_body.context
    rng = np.random.default_rng(5)
    c = rng.normal(size=(two_body.n_ao, 20)) / np.sqrt(two_body.n_ao)
    k64 = ctx.exchange_factored_host(c, None, _lib.PREC_FP64)
    ctx.exchange_factored_host(c, None, _lib.PREC_BF16X3)  # the BF16 copy of B exists before the stall
    ctx.set_wait_limit(1e-3, stall_next_build=True)
    with pytest.raises(BackendError, match="wait ran out"):
        ctx.exchange_factored_host(c, None, _lib.PREC_BF16X3)
    ctx.set_wait_limit(2.0)
    for _ in range(2):
        k16 = ctx.exchange_factored_host(c, None, _lib.PREC_BF16X3)
        assert np.max(np.abs(k16 - k64)) <= REL_TOL * np.max(np.abs(k64))
    with pytest.raises(InputError, match="wait limit"):
        ctx.set_wait_limit(1e-9)
