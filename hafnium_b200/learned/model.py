"""The learned initial density: a message-passing network over atoms and the
AO shell-pair blocks between them.

Nodes are the atoms of a molecule, edges the ordered atom pairs closer than
``R_CUT``. A node starts from a learned embedding of its element; every edge
carries the geometry of atom j seen from the frame of atom i (j's position, the
relative rotation of the two frames, a radial basis of the distance), so
everything the network sees and predicts is independent of how the molecule
sits in space. Four residual message-passing layers of width 128 feed two
heads: the diagonal block of each atom's density in its own frame (the upper
triangle of the atom's shell-pair blocks, on top of the training set's mean
block for its element) and the block between the two atoms of each edge (all
their shell pairs), both laid out on NA_AO functions per atom (cc-pVDZ: 14 for
B-Ne, 5 for H and He; the unused rows and columns are trained towards zero).
Blocks between atoms further apart than ``R_CUT`` are zero.

Forward, backward and Adam run on the device through the kernels of
include/hfnn.h (FP32). ``predict_density`` turns the blocks into a global
density, which the SCF projects onto the occupied space (the n_occ leading
natural orbitals in the overlap metric) so that it starts from an idempotent
density with the right electron count. For a molecule with an element the
network was not trained on, an atom without a frame (a linear molecule), a basis
other than cc-pVDZ or without trained weights the caller falls back to the
superposition of atomic densities.
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import math
import pathlib

import numpy as np

from hafnium_b200.learned.frames import ao_rotations, atom_frames, shell_layout

R_CUT = 10.0  # bohr, atom-atom
N_RBF = 16
EDGE_FEATURES = 3 + 9 + N_RBF  # position of j in i's frame, R_i^T R_j, RBF of the distance
WIDTH = 128
LAYERS = 4
ELEMENTS = ("H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne")  # embedding rows, Z = 1..10
NA_AO = 14  # functions of one atom, padded (cc-pVDZ: 14 for B-Ne, 5 for H and He)
DIAG = NA_AO * (NA_AO + 1) // 2
OFF = NA_AO * NA_AO
BASIS = "cc-pvdz"
WEIGHTS = pathlib.Path(__file__).resolve().parent / "weights_ccpvdz_atoms.npz"
_IU = np.triu_indices(NA_AO)


def element_index(symbol: str) -> int:
    """Row of the element's embedding (Z - 1), -1 outside H-Ne."""
    name = symbol.capitalize()
    return ELEMENTS.index(name) if name in ELEMENTS else -1


def build_graph(molecule, table=None) -> dict | None:
    """Nodes, edges, edge features, the per-atom AO rotations and function
    ranges (host arrays); None when an atom has no frame or lies outside H-Ne."""
    from hafnium_b200.basis import ShellTable

    elem = np.array([element_index(s) for s in molecule.symbols], dtype=np.int32)
    if len(elem) == 0 or np.any(elem < 0):
        return None
    pos = np.asarray(molecule.positions, dtype=np.float64)
    frames = atom_frames(pos)
    if frames is None:
        return None
    if table is None:
        table = ShellTable.build(BASIS, molecule.symbols, pos)
    n = len(pos)
    rot = np.zeros((n, NA_AO, NA_AO))
    nfun = np.zeros(n, dtype=np.int64)
    for a, u in enumerate(ao_rotations(frames, [shell_layout(table, a) for a in range(n)])):
        if u.shape[0] > NA_AO:
            return None
        nfun[a] = u.shape[0]
        rot[a, : u.shape[0], : u.shape[0]] = u
    offsets = np.concatenate([[0], np.cumsum(nfun)[:-1]])
    fr = np.stack(frames)  # [atom, 3, 3], columns the local axes
    diff = pos[None, :, :] - pos[:, None, :]  # [i, j] = r_j - r_i
    dist = np.linalg.norm(diff, axis=2)
    src, dst = np.nonzero((dist < R_CUT) & ~np.eye(n, dtype=bool))
    d = dist[src, dst]
    rel = np.einsum("eab,ea->eb", fr[src], diff[src, dst]) / R_CUT
    rr = np.einsum("eab,eac->ebc", fr[src], fr[dst]).reshape(-1, 9)
    centers = np.linspace(1.0, R_CUT, N_RBF)
    width = centers[1] - centers[0]
    rbf = np.exp(-(((d[:, None] - centers[None, :]) / width) ** 2))
    return {
        "n_nodes": n,
        "elem": elem,
        "src": src.astype(np.int32),
        "dst": dst.astype(np.int32),
        "edge": np.concatenate([rel, rr, rbf], axis=1).reshape(-1, EDGE_FEATURES),
        "fcut": 0.5 * (np.cos(np.pi * d / R_CUT) + 1.0),
        "rot": rot,
        "nfun": nfun,
        "offsets": offsets,
        "n_ao": int(nfun.sum()),
    }


def _padded_index(graph: dict):
    """(atom, local function) of every global function, in global order."""
    nf = graph["nfun"]
    atom, local = np.nonzero(np.arange(NA_AO)[None, :] < nf[:, None])
    return atom, local


def local_targets(graph: dict, density: np.ndarray, mean_diag: np.ndarray | None = None) -> dict:
    """Blocks of a converged (per-spin) density in the frames of their atoms,
    laid out on NA_AO functions per atom."""
    n = graph["n_nodes"]
    atom, local = _padded_index(graph)
    dp = np.zeros((n, NA_AO, n, NA_AO))
    dp[atom[:, None], local[:, None], atom[None, :], local[None, :]] = density
    rot = graph["rot"]
    dl = np.einsum("iab,iajc,jcd->ibjd", rot, dp, rot, optimize=True)
    idx = np.arange(n)
    d = dl[idx, :, idx, :][:, _IU[0], _IU[1]]
    if mean_diag is not None:
        d = d - mean_diag[graph["elem"]]
    o = dl[graph["src"], :, graph["dst"], :].reshape(-1, OFF)
    return {"d": d, "o": o}


def blocks_to_density(graph: dict, d_blocks: np.ndarray, o_blocks: np.ndarray, mean_diag: np.ndarray) -> np.ndarray:
    """Global per-spin density from local-frame blocks (symmetrised over the two
    edges of an atom pair)."""
    n = graph["n_nodes"]
    dl = np.zeros((n, NA_AO, n, NA_AO))
    diag = np.zeros((n, NA_AO, NA_AO))
    diag[:, _IU[0], _IU[1]] = d_blocks + mean_diag[graph["elem"]]
    diag = diag + np.transpose(np.triu(diag, 1), (0, 2, 1))
    idx = np.arange(n)
    dl[idx, :, idx, :] = diag
    o = o_blocks.reshape(-1, NA_AO, NA_AO)
    np.add.at(dl, (graph["src"], slice(None), graph["dst"], slice(None)), 0.5 * o)
    np.add.at(dl, (graph["dst"], slice(None), graph["src"], slice(None)), 0.5 * np.transpose(o, (0, 2, 1)))
    rot = graph["rot"]
    dp = np.einsum("iab,ibjc,jdc->iajd", rot, dl, rot, optimize=True)
    atom, local = _padded_index(graph)
    return dp[atom[:, None], local[:, None], atom[None, :], local[None, :]]


def init_params(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)

    def dense(i, o, scale=1.0):
        return (rng.normal(size=(i, o)) * scale / math.sqrt(i)).astype(np.float32), np.zeros(o, np.float32)

    p = {"h0": (rng.normal(size=(len(ELEMENTS), WIDTH)) * 0.5).astype(np.float32)}  # one row per element
    for l in range(LAYERS):
        p[f"Wm{l}"], p[f"bm{l}"] = dense(2 * WIDTH + EDGE_FEATURES, WIDTH)
        p[f"Wu{l}"], p[f"bu{l}"] = dense(2 * WIDTH, WIDTH, 0.5)
    p["Wd"], p["bd"] = dense(WIDTH, DIAG, 0.1)
    p["We"], p["be"] = dense(2 * WIDTH + EDGE_FEATURES, WIDTH)
    p["Wo"], p["bo"] = dense(WIDTH, OFF, 0.1)
    return p


def param_names(layers: int = LAYERS):
    names = ["h0"]
    for l in range(layers):
        names += [f"Wm{l}", f"bm{l}", f"Wu{l}", f"bu{l}"]
    return names + ["Wd", "bd", "We", "be", "Wo", "bo"]


class DeviceNet:
    """Parameters on the device and the forward/backward passes over one graph."""

    def __init__(self, params: dict, layers: int = LAYERS, device: int = 0) -> None:
        import torch

        from hafnium_b200 import _lib

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.layers = layers
        self.lib = _lib.load()
        self._bind()
        self.p = {k: torch.as_tensor(np.asarray(v, dtype=np.float32), device=self.dev).contiguous()
                  for k, v in params.items()}
        self.width = int(self.p["h0"].shape[1])

    def _bind(self) -> None:
        L, v, f, i, i64 = self.lib, ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_int64
        L.hfnn_sgemm.argtypes = [i, i, i, v, i, v, i, v, v, i, v]
        L.hfnn_silu.argtypes = [i64, i, v, v, v, i, v]
        L.hfnn_dsilu.argtypes = [i64, i, v, v, v, v, v]
        L.hfnn_gather.argtypes = [i64, i, v, v, v, i, i, v]
        L.hfnn_scatter_add.argtypes = [i64, i, v, i, i, v, v, v, v]
        L.hfnn_colsum.argtypes = [i64, i, v, v, v]
        L.hfnn_sq_loss.argtypes = [i64, v, v, f, v, v, v]
        L.hfnn_adam.argtypes = [i64, v, v, v, v, f, f, f, f, i, v]

    @staticmethod
    def _ptr(t):
        return None if t is None else t.data_ptr()

    def _ok(self, status: int, what: str) -> None:
        if status != 0:
            from hafnium_b200.errors import BackendError

            raise BackendError(f"{what} failed with status {status}")

    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def linear(self, x, w, b, out=None, ta=0, tb=0, accumulate=0):
        """out = op(x) op(w) + b with the shapes hfnn_sgemm takes."""
        m = x.shape[1] if ta else x.shape[0]
        k = x.shape[0] if ta else x.shape[1]
        n = w.shape[0] if tb else w.shape[1]
        if out is None:
            out = self.torch.empty((m, n), dtype=self.torch.float32, device=self.dev)
        self._ok(self.lib.hfnn_sgemm(m, n, k, self._ptr(x), ta, self._ptr(w), tb, self._ptr(b), self._ptr(out),
                                     accumulate, self._stream()), "hfnn_sgemm")
        return out

    def upload_graph(self, graph: dict) -> dict:
        t = self.torch
        return {
            "n": graph["n_nodes"],
            "elem": t.as_tensor(graph["elem"], dtype=t.int32, device=self.dev),
            "src": t.as_tensor(graph["src"], dtype=t.int32, device=self.dev),
            "dst": t.as_tensor(graph["dst"], dtype=t.int32, device=self.dev),
            "edge": t.as_tensor(graph["edge"], dtype=t.float32, device=self.dev).contiguous(),
            "fcut": t.as_tensor(graph["fcut"], dtype=t.float32, device=self.dev).contiguous(),
            "ne": int(len(graph["src"])),
        }

    def _edge_input(self, h, g):
        t, W = self.torch, self.width
        ne = g["ne"]
        x = t.empty((ne, 2 * W + EDGE_FEATURES), dtype=t.float32, device=self.dev)
        s = self._stream()
        ld = 2 * W + EDGE_FEATURES
        self._ok(self.lib.hfnn_gather(ne, W, self._ptr(h), self._ptr(g["src"]), self._ptr(x), ld, 0, s), "gather")
        self._ok(self.lib.hfnn_gather(ne, W, self._ptr(h), self._ptr(g["dst"]), self._ptr(x), ld, W, s), "gather")
        self._ok(self.lib.hfnn_gather(ne, EDGE_FEATURES, self._ptr(g["edge"]), None, self._ptr(x), ld, 2 * W, s),
                 "gather")
        return x

    def forward(self, g):
        t, W, s = self.torch, self.width, self._stream()
        n, ne = g["n"], g["ne"]
        h = t.empty((n, W), dtype=t.float32, device=self.dev)  # each atom's element embedding
        self._ok(self.lib.hfnn_gather(n, W, self._ptr(self.p["h0"]), self._ptr(g["elem"]), self._ptr(h), W, 0, s),
                 "gather")
        cache = []
        for l in range(self.layers):
            xm = self._edge_input(h, g)
            zm = self.linear(xm, self.p[f"Wm{l}"], self.p[f"bm{l}"])
            m = t.empty_like(zm)
            self._ok(self.lib.hfnn_silu(ne, W, self._ptr(zm), self._ptr(g["fcut"]), self._ptr(m), 0, s), "silu")
            a = t.zeros((n, W), dtype=t.float32, device=self.dev)
            self._ok(self.lib.hfnn_scatter_add(ne, W, self._ptr(m), W, 0, self._ptr(g["src"]), None, self._ptr(a), s),
                     "scatter")
            xu = t.cat([h, a], dim=1).contiguous()
            zu = self.linear(xu, self.p[f"Wu{l}"], self.p[f"bu{l}"])
            cache.append((xm, zm, xu, zu))
            h = h.clone()
            self._ok(self.lib.hfnn_silu(n, W, self._ptr(zu), None, self._ptr(h), 1, s), "silu")
        d = self.linear(h, self.p["Wd"], self.p["bd"])
        xe = self._edge_input(h, g)
        ze = self.linear(xe, self.p["We"], self.p["be"])
        ge = t.empty_like(ze)
        self._ok(self.lib.hfnn_silu(ne, W, self._ptr(ze), None, self._ptr(ge), 0, s), "silu")
        o = self.linear(ge, self.p["Wo"], self.p["bo"])
        return {"d": d, "o": o, "h": h}, (cache, xe, ze, ge)

    def loss_and_grad(self, g, targets: dict, w_edge: float = 1.0):
        t, W, s = self.torch, self.width, self._stream()
        n, ne = g["n"], g["ne"]
        out, (cache, xe, ze, ge) = self.forward(g)
        loss = t.zeros(1, dtype=t.float32, device=self.dev)
        dd = t.empty_like(out["d"])
        do = t.empty_like(out["o"])
        self._ok(self.lib.hfnn_sq_loss(dd.numel(), self._ptr(out["d"]), self._ptr(targets["d"]), 1.0, self._ptr(dd),
                                       self._ptr(loss), s), "loss")
        self._ok(self.lib.hfnn_sq_loss(do.numel(), self._ptr(out["o"]), self._ptr(targets["o"]), w_edge,
                                       self._ptr(do), self._ptr(loss), s), "loss")
        grads = {}
        h = out["h"]

        def dense_bwd(x, dz, wname, bname):
            grads[wname] = self.linear(x, dz, None, ta=1)  # x^T dz
            gb = t.empty(dz.shape[1], dtype=t.float32, device=self.dev)
            self._ok(self.lib.hfnn_colsum(dz.shape[0], dz.shape[1], self._ptr(dz), self._ptr(gb), s), "colsum")
            grads[bname] = gb
            return self.linear(dz, self.p[wname], None, tb=1)  # dz W^T

        dh = dense_bwd(h, dd, "Wd", "bd")
        dg = dense_bwd(ge, do, "Wo", "bo")
        dze = t.empty_like(ze)
        self._ok(self.lib.hfnn_dsilu(ne, W, self._ptr(dg), self._ptr(ze), None, self._ptr(dze), s), "dsilu")
        dxe = dense_bwd(xe, dze, "We", "be")
        ld = 2 * W + EDGE_FEATURES
        self._ok(self.lib.hfnn_scatter_add(ne, W, self._ptr(dxe), ld, 0, self._ptr(g["src"]), None, self._ptr(dh), s),
                 "scatter")
        self._ok(self.lib.hfnn_scatter_add(ne, W, self._ptr(dxe), ld, W, self._ptr(g["dst"]), None, self._ptr(dh), s),
                 "scatter")
        for l in reversed(range(self.layers)):
            xm, zm, xu, zu = cache[l]
            dzu = t.empty_like(zu)
            self._ok(self.lib.hfnn_dsilu(n, W, self._ptr(dh), self._ptr(zu), None, self._ptr(dzu), s), "dsilu")
            dxu = dense_bwd(xu, dzu, f"Wu{l}", f"bu{l}")
            dh_in = dh + dxu[:, :W]
            da = dxu[:, W:].contiguous()
            dm = t.empty((ne, W), dtype=t.float32, device=self.dev)
            self._ok(self.lib.hfnn_gather(ne, W, self._ptr(da), self._ptr(g["src"]), self._ptr(dm), W, 0, s),
                     "gather")
            dzm = t.empty_like(zm)
            self._ok(self.lib.hfnn_dsilu(ne, W, self._ptr(dm), self._ptr(zm), self._ptr(g["fcut"]), self._ptr(dzm), s),
                     "dsilu")
            dxm = dense_bwd(xm, dzm, f"Wm{l}", f"bm{l}")
            dh_in = dh_in.contiguous()
            self._ok(self.lib.hfnn_scatter_add(ne, W, self._ptr(dxm), ld, 0, self._ptr(g["src"]), None,
                                               self._ptr(dh_in), s), "scatter")
            self._ok(self.lib.hfnn_scatter_add(ne, W, self._ptr(dxm), ld, W, self._ptr(g["dst"]), None,
                                               self._ptr(dh_in), s), "scatter")
            dh = dh_in
        gh0 = t.zeros_like(self.p["h0"])  # per element: the sum over its atoms
        self._ok(self.lib.hfnn_scatter_add(n, W, self._ptr(dh.contiguous()), W, 0, self._ptr(g["elem"]), None,
                                           self._ptr(gh0), s), "scatter")
        grads["h0"] = gh0
        return loss, grads


class Adam:
    def __init__(self, net: DeviceNet, lr: float = 1e-3) -> None:
        t = net.torch
        self.net, self.lr, self.step = net, lr, 0
        self.m = {k: t.zeros_like(v) for k, v in net.p.items()}
        self.v = {k: t.zeros_like(v) for k, v in net.p.items()}

    def apply(self, grads: dict, scale: float = 1.0) -> None:
        self.step += 1
        net = self.net
        for k, p in net.p.items():
            g = grads[k] * scale if scale != 1.0 else grads[k]
            net._ok(net.lib.hfnn_adam(p.numel(), p.data_ptr(), g.contiguous().data_ptr(), self.m[k].data_ptr(),
                                      self.v[k].data_ptr(), self.lr, 0.9, 0.999, 1e-8, self.step, net._stream()),
                    "adam")


def save_weights(path: pathlib.Path, params: dict, mean_diag: np.ndarray, meta: dict) -> str:
    arrays = {k: np.asarray(v, dtype=np.float32) for k, v in params.items()}
    arrays["mean_diag"] = np.asarray(mean_diag, dtype=np.float64)
    digest = hashlib.sha256()
    for k in sorted(arrays):
        digest.update(k.encode())
        digest.update(np.ascontiguousarray(arrays[k]).tobytes())
    meta = dict(meta, sha256=digest.hexdigest(), version=2, layers=LAYERS, width=WIDTH, r_cut=R_CUT, na_ao=NA_AO)
    np.savez_compressed(path, meta=json.dumps(meta), **arrays)
    return meta["sha256"]


def load_weights(path: pathlib.Path = WEIGHTS):
    """Parameters, the mean diagonal block and the metadata; None when absent or corrupt."""
    if not pathlib.Path(path).exists():
        return None
    with np.load(path) as z:
        meta = json.loads(str(z["meta"]))
        arrays = {k: z[k] for k in z.files if k != "meta"}
    digest = hashlib.sha256()
    for k in sorted(arrays):
        digest.update(k.encode())
        digest.update(np.ascontiguousarray(arrays[k]).tobytes())
    if digest.hexdigest() != meta.get("sha256"):
        return None
    mean_diag = arrays.pop("mean_diag")
    return arrays, mean_diag, meta


def assemble_density(graph: dict, d_blocks, o_blocks, mean_diag: np.ndarray, device):
    """``blocks_to_density`` on the device: the network's blocks (torch tensors)
    to the global per-spin density, FP64, as a torch tensor on ``device``."""
    import torch

    n = graph["n_nodes"]
    f64 = dict(dtype=torch.float64, device=device)
    elem = torch.as_tensor(graph["elem"], dtype=torch.long, device=device)
    iu0 = torch.as_tensor(_IU[0], dtype=torch.long, device=device)
    iu1 = torch.as_tensor(_IU[1], dtype=torch.long, device=device)
    diag = torch.zeros((n, NA_AO, NA_AO), **f64)
    diag[:, iu0, iu1] = d_blocks.to(torch.float64) + torch.as_tensor(mean_diag, **f64)[elem]
    diag = diag + torch.triu(diag, 1).transpose(1, 2)
    # dl[i][j] = the (i, j) block in the frames of atoms i and j
    dl = torch.zeros((n, n, NA_AO, NA_AO), **f64)
    idx = torch.arange(n, device=device)
    dl[idx, idx] = diag
    src = torch.as_tensor(graph["src"], dtype=torch.long, device=device)
    dst = torch.as_tensor(graph["dst"], dtype=torch.long, device=device)
    o = o_blocks.to(torch.float64).reshape(-1, NA_AO, NA_AO)
    dl.index_put_((src, dst), 0.5 * o, accumulate=True)
    dl.index_put_((dst, src), 0.5 * o.transpose(1, 2), accumulate=True)
    rot = torch.as_tensor(graph["rot"], **f64)
    dp = torch.einsum("iab,ijbc,jdc->ijad", rot, dl, rot)
    atom, local = _padded_index(graph)
    atom = torch.as_tensor(atom, dtype=torch.long, device=device)
    local = torch.as_tensor(local, dtype=torch.long, device=device)
    return dp[atom[:, None], atom[None, :], local[:, None], local[None, :]]


def predict_density(molecule, weights=None, device: int = 0, table=None):
    """The network's per-spin density of a molecule in cc-pVDZ (a torch FP64
    tensor on the device), or None (fall back to SAD): no weights, an element
    the network was not trained on, or an atom without a frame."""
    loaded = load_weights() if weights is None else weights
    if loaded is None:
        return None
    params, mean_diag, meta = loaded
    trained = set(meta.get("elements", ()))
    if any(s.capitalize() not in trained for s in molecule.symbols):
        return None
    graph = build_graph(molecule, table)
    if graph is None:
        return None
    net = DeviceNet(params, device=device)
    out, _ = net.forward(net.upload_graph(graph))
    return assemble_density(graph, out["d"], out["o"], mean_diag, net.dev)
