"""The mixed-precision exchange schedule's host logic (CPU, torch on the host).

The difference factorisation behind the incremental builds and the state
machine behind the protocol's ``exchange(D)``, with a stand-in builder whose
"BF16" builds add a known relative error, so the arithmetic each call chooses
and the accuracy it keeps can be checked without a GPU.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from hafnium_b200 import _lib
from hafnium_b200.jk import MixedExchangeSchedule, difference_factors, polar_rotation


def orthonormal_pair(n=40, o=8, angle=1e-3, seed=0):
    """S-orthonormal C_new, C_old (C^T S C = I) spanning nearby subspaces."""
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n))
    s = a @ a.T / n + np.eye(n)
    w, v = np.linalg.eigh(s)
    s_half_inv = (v / np.sqrt(w)) @ v.T
    q, _ = np.linalg.qr(rng.normal(size=(n, o)))
    k = rng.normal(size=(n, n))
    k = angle * (k - k.T)
    rot = np.linalg.matrix_power(np.eye(n) + k / 16, 16)  # near-orthogonal rotation exp(K)
    rot, _ = np.linalg.qr(rot)
    q2 = rot @ q
    mix = np.linalg.qr(rng.normal(size=(o, o)))[0]  # a different gauge of the same span
    c_new = s_half_inv @ q
    c_old = s_half_inv @ (q2 @ mix)
    return torch.as_tensor(c_new), torch.as_tensor(c_old), torch.as_tensor(s)


@pytest.mark.parametrize("angle", [1e-2, 1e-4, 1e-7])
def test_difference_factors_reproduce_the_difference(angle):
    c_new, c_old, s = orthonormal_pair(angle=angle)
    vp, vm = difference_factors(c_new, c_old, s)
    diff = c_new @ c_new.T - c_old @ c_old.T
    got = vp @ vp.T - vm @ vm.T
    assert float((got - diff).abs().max()) < 1e-14
    # both factors scale like the square root of the difference, not like the densities
    scale = float(diff.abs().max())
    assert float((vp @ vp.T).abs().max()) < 20 * scale
    assert float((vm @ vm.T).abs().max()) < 20 * scale


def test_difference_factors_pad_unequal_ranks():
    c_new, c_old, s = orthonormal_pair(angle=1e-3)
    c_old = c_old[:, :6]
    vp, vm = difference_factors(c_new, c_old, s)
    diff = c_new @ c_new.T - c_old @ c_old.T
    assert float((vp @ vp.T - vm @ vm.T - diff).abs().max()) < 1e-13


def test_polar_rotation_falls_back_for_a_far_rotation():
    rng = np.random.default_rng(1)
    m = torch.as_tensor(rng.normal(size=(6, 6)) * 0.01)  # singular values far below one
    r = polar_rotation(m)
    assert float((r.T @ r - torch.eye(6, dtype=r.dtype)).abs().max()) < 1e-13
    u, _, vh = torch.linalg.svd(m)
    assert float((r - u @ vh).abs().max()) < 1e-10


class FakeContext:
    def __init__(self, s):
        self.s = s

    def overlap_device(self):
        return self.s

    def density_factor_device(self, d, max_rank):
        w, v = torch.linalg.eigh(0.5 * (d + d.T))
        keep = w > 1e-14 * w.abs().max()
        return (v[:, keep] * w[keep].sqrt()).contiguous()


class FakeBuilder:
    """K = sum_P B_P D B_P on the host; "BF16" builds carry a relative error of 1e-5."""

    def __init__(self, b, s):
        self.b = b
        self.context = FakeContext(s)
        self.calls = []

    def exchange_factored(self, factor, precision=_lib.PREC_FP64):
        self.calls.append(precision)
        x = torch.einsum("puv,vi->pui", self.b, factor)
        k = torch.einsum("pui,pwi->uw", x, x)
        if precision == _lib.PREC_BF16X3:
            k = k * (1.0 + 1e-5)
        return k


def test_schedule_phases_and_accuracy():
    """A converging sequence of densities: BF16 builds while the change is large,
    one FP64 anchor, incremental builds, one late FP64 re-anchor; the last builds
    err by far less than the BF16 builds."""
    n, o = 40, 8
    c_new, c_old, s = orthonormal_pair(n, o, angle=3e-2, seed=3)
    rng = np.random.default_rng(4)
    b = torch.as_tensor(rng.normal(size=(30, n, n)))
    b = 0.5 * (b + b.transpose(1, 2))
    builder = FakeBuilder(b, s)
    schedule = MixedExchangeSchedule(builder)
    # densities along a path converging geometrically from c_old's to c_new's span
    exact = FakeBuilder(b, s)
    errors = []
    for step in range(24):
        t = 0.5 ** step
        c = c_new + t * (c_old - c_new)  # not orthonormal, but PSD densities are all the schedule needs
        d = c @ c.T
        k = schedule.exchange(d)
        k_exact = exact.exchange_factored(schedule.two_body.context.density_factor_device(d, n))
        errors.append(float((k - k_exact).abs().max() / k_exact.abs().max()))
    kinds = [entry["precision"] for entry in schedule.log]
    assert kinds[0] == "bf16"
    assert kinds.count("anchor") == 2  # the anchor after the BF16 phase and one late re-anchor
    first_anchor = kinds.index("anchor")
    assert all(k == "bf16" for k in kinds[:first_anchor])
    assert set(kinds[first_anchor:]) == {"anchor", "incremental"}
    assert errors[0] > 5e-6  # a BF16 build
    assert max(errors[first_anchor:]) < 1e-7  # incremental on the first anchor
    assert errors[-1] < 1e-9  # incremental on the late anchor
    # a jump back to a far density restarts the BF16 phase
    schedule.exchange(c_old @ c_old.T)
    assert schedule.log[-1]["precision"] == "bf16"
