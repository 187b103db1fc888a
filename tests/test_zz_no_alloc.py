"""hf_coulomb_static: the Coulomb build that allocates no device memory (B200).

Callers whose device memory is already fully reserved by their own pool
allocator, or whose loop may not pay for a cudaMalloc's device synchronisation,
call hf_coulomb_static instead of hf_coulomb; its scratch is a static device
array (n_ao <= 1536, n_aux <= 8192). This file is collected last on purpose: it
must pass on its own in a fresh process and after every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

from hafnium_b200 import _lib
from hafnium_b200.errors import InputError
from hafnium_b200.jk import B200DensityFittedCoulombExchange
from tests.helpers import molecule, tables

pytestmark = pytest.mark.gpu
JK_TOL = 1e-10


def test_static_coulomb_matches_the_allocating_entry_point_twice():
    import torch

    mol = molecule("h2o4_s1")
    orb, aux = tables(mol)
    rng = np.random.default_rng(11)
    # a fresh context whose first J build is the static one: that build must not allocate
    fresh = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    n = fresh.n_ao
    c = rng.normal(size=(n, 20)) / np.sqrt(n)
    d = torch.as_tensor(c @ c.T, device="cuda")
    got = torch.full_like(d, float("nan"))
    before = fresh.context.stats()["device_allocations"]
    fresh.context.coulomb_static_device(d, got)
    assert fresh.context.stats()["device_allocations"] == before
    first = got.clone()
    # the allocating entry point on another context gives the expected J
    two_body = B200DensityFittedCoulombExchange.from_tables(orb, aux)
    expected = torch.empty_like(d)
    two_body.context.coulomb_device(d, expected)
    np.testing.assert_allclose(first.cpu().numpy(), expected.cpu().numpy(), atol=JK_TOL, rtol=0)
    for _ in range(2):  # two calls in a row share (and must re-clear) the static scratch
        got = torch.full_like(d, float("nan"))
        two_body.context.coulomb_static_device(d, got)
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), expected.cpu().numpy(), atol=JK_TOL, rtol=0)


def test_static_coulomb_rejects_systems_beyond_its_limit():
    import torch

    from hafnium_b200.molecule import water_cluster

    mol = water_cluster(65, 0)  # 1560 orbital functions > 1536
    orb, aux = tables(mol)
    ctx = _lib.Context(0)
    ctx.upload(orb, aux)  # no fitted tensor needed: the size check comes first
    d = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(InputError, match="n_ao <= 1536"):
        ctx.coulomb_static_device(d, d)
