"""Oracle: NumPy forward and backward of the learned-guess message-passing network.

TEST INFRASTRUCTURE ONLY: the checker for the gradients of the device training
kernels (hafnium_b200/csrc/mpnn.cu). The network has no counterpart in the
reference (it is the north star's new learned initial guess); this file states
its mathematics independently of the CUDA code:

    h_i^0 = h0[elem_i]                           (learned embedding of atom i's element)
    for each layer l:
        m_ij = silu(W_m^l [h_i ; h_j ; e_ij] + b_m^l) * fcut_ij
        a_i  = sum_j m_ij
        h_i  <- h_i + silu(W_u^l [h_i ; a_i] + b_u^l)
    d_i  = W_d h_i + b_d                          (diagonal block of atom i, upper entries)
    g_ij = silu(W_e [h_i ; h_j ; e_ij] + b_e)
    o_ij = W_o g_ij + b_o                         (the block between atoms i and j)
    loss = sum_i |d_i - t_i|^2 + w_edge sum_ij |o_ij - t_ij|^2

Weights are stored as [in, out]; activations as rows.
"""

from __future__ import annotations

import numpy as np


def silu(x):
    return x / (1.0 + np.exp(-x))


def dsilu(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def forward(params: dict, graph: dict, layers: int):
    """Returns the outputs and the cache the backward pass needs."""
    src, dst = graph["src"], graph["dst"]  # edge (i -> j): i = src (receiver), j = dst
    e, fc = graph["edge"], graph["fcut"]
    h = params["h0"][graph["elem"]]
    cache = []
    for l in range(layers):
        xm = np.concatenate([h[src], h[dst], e], axis=1)
        zm = xm @ params[f"Wm{l}"] + params[f"bm{l}"]
        m = silu(zm) * fc[:, None]
        a = np.zeros_like(h)
        np.add.at(a, src, m)
        xu = np.concatenate([h, a], axis=1)
        zu = xu @ params[f"Wu{l}"] + params[f"bu{l}"]
        cache.append((h, xm, zm, xu, zu))
        h = h + silu(zu)
    d = h @ params["Wd"] + params["bd"]
    xe = np.concatenate([h[src], h[dst], e], axis=1)
    ze = xe @ params["We"] + params["be"]
    g = silu(ze)
    o = g @ params["Wo"] + params["bo"]
    return {"d": d, "o": o, "h": h}, (cache, xe, ze, g)


def loss_and_grad(params: dict, graph: dict, targets: dict, layers: int, w_edge: float = 1.0):
    out, (cache, xe, ze, g) = forward(params, graph, layers)
    src, dst = graph["src"], graph["dst"]
    fc = graph["fcut"]
    rd = out["d"] - targets["d"]
    ro = out["o"] - targets["o"]
    loss = float(np.sum(rd * rd) + w_edge * np.sum(ro * ro))
    grads = {}
    dd = 2.0 * rd
    do = 2.0 * w_edge * ro
    h = out["h"]
    grads["Wd"] = h.T @ dd
    grads["bd"] = dd.sum(0)
    dh = dd @ params["Wd"].T
    grads["Wo"] = g.T @ do
    grads["bo"] = do.sum(0)
    dg = do @ params["Wo"].T
    dze = dg * dsilu(ze)
    grads["We"] = xe.T @ dze
    grads["be"] = dze.sum(0)
    dxe = dze @ params["We"].T
    width = h.shape[1]
    np.add.at(dh, src, dxe[:, :width])
    np.add.at(dh, dst, dxe[:, width:2 * width])
    for l in reversed(range(layers)):
        h_in, xm, zm, xu, zu = cache[l]
        # h_out = h_in + silu(zu)
        dzu = dh * dsilu(zu)
        grads[f"Wu{l}"] = xu.T @ dzu
        grads[f"bu{l}"] = dzu.sum(0)
        dxu = dzu @ params[f"Wu{l}"].T
        dh_in = dh + dxu[:, :width]
        da = dxu[:, width:]
        dm = da[src] * fc[:, None]
        dzm = dm * dsilu(zm)
        grads[f"Wm{l}"] = xm.T @ dzm
        grads[f"bm{l}"] = dzm.sum(0)
        dxm = dzm @ params[f"Wm{l}"].T
        np.add.at(dh_in, src, dxm[:, :width])
        np.add.at(dh_in, dst, dxm[:, width:2 * width])
        dh = dh_in
    grads["h0"] = np.zeros_like(params["h0"])
    np.add.at(grads["h0"], graph["elem"], dh)
    return loss, grads
