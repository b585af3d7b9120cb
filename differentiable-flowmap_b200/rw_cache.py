"""Trajectory interop with the reference's on-disk format (RW_Cache).

The reference keeps its forward trajectory in ``.npy`` files
(3D/lfm_midpoint_simulator.py:46-165, 2D/vortex/lfm_midpoint_simulator.py:
91-184): every named stream ("u", "s", "phi", "phi_xyz", "F", ...) is cached in
chunks of ``n_steps`` = 100 frames and saved as ``{name}_{first}_{last}.npy``,
an array ``(n_steps, *padded grid, C)`` of float32 holding the whole chunk
buffer (frames past the last written one keep the buffer's older content, as
in the reference).  Single arrays go to ``{name}_{j}.npy`` (write_disk).

Frames are stored in the reference's padded, component-last layouts:

* a MAC field (u, adj_u): ``(n+1)^dim x dim`` with face grid c in
  ``[..., c]`` over its own extent (scalar2vec, 3D/taichi_utils.py:11-20),
* face vector fields (phi_xyz, F): ``(n+1)^dim x dim*dim`` with face grid c's
  dim-vector in ``[..., c*dim:(c+1)*dim]`` (vec2mat, 3D/taichi_utils.py:35-44),
* a cell vector field (phi): ``n^dim x dim``; a scalar (s, adj_s): ``n^dim x 1``.

Here the same layouts are produced from, and unpacked into, this package's
device tensors (a MAC field is a list of face tensors; vector fields are
``(dim, *grid)`` component planes).  ``export_forward`` / ``import_forward``
write and read a simulator's whole forward trajectory in the reference's
directory tree (midpoint/, passive/, flowmap_phi/, flowmap_phi_xyz/ (2D:
flowmap_phi_xy/), flowmap_F/, final/), so a Taichi run can be compared frame
by frame, or its forward pass fed to this package's adjoint.
"""
from __future__ import annotations

import os
import re
from typing import Dict, List, Sequence

import numpy as np
import torch

N_STEPS = 100  # frames per chunk file (RW_Cache.n_steps)

_CHUNK = re.compile(r"^.*?_(\d+)_(\d+)\.\w+$")


def _np(t) -> np.ndarray:
    if isinstance(t, torch.Tensor):
        return t.detach().to(torch.float32).cpu().numpy()
    return np.asarray(t, dtype=np.float32)


# ----------------------------------------------------------------- layouts
def pack_mac(u: Sequence) -> np.ndarray:
    """MAC field -> (n+1)^dim x dim (scalar2vec)."""
    dim = len(u)
    comps = [_np(x) for x in u]
    shape = tuple(comps[0].shape[a] + (0 if a == 0 else 1) for a in range(dim))
    out = np.zeros(shape + (dim,), dtype=np.float32)
    for c, x in enumerate(comps):
        out[tuple(slice(0, s) for s in x.shape) + (c,)] = x
    return out


def unpack_mac(buf: np.ndarray, res: Sequence[int]) -> List[np.ndarray]:
    dim = len(res)
    out = []
    for c in range(dim):
        sl = tuple(slice(0, res[a] + (1 if a == c else 0)) for a in range(dim))
        out.append(np.ascontiguousarray(buf[sl + (c,)]))
    return out


def pack_face_vectors(f: Sequence) -> np.ndarray:
    """Face vector fields (f[c] of shape (dim, *face grid c)) -> (n+1)^dim x dim*dim (vec2mat)."""
    dim = len(f)
    comps = [_np(x) for x in f]
    res = [comps[0].shape[1 + a] - (1 if a == 0 else 0) for a in range(dim)]
    out = np.zeros(tuple(r + 1 for r in res) + (dim * dim,), dtype=np.float32)
    for c, x in enumerate(comps):
        sl = tuple(slice(0, s) for s in x.shape[1:])
        for a in range(dim):
            out[sl + (c * dim + a,)] = x[a]
    return out


def unpack_face_vectors(buf: np.ndarray, res: Sequence[int]) -> List[np.ndarray]:
    dim = len(res)
    out = []
    for c in range(dim):
        sl = tuple(slice(0, res[a] + (1 if a == c else 0)) for a in range(dim))
        out.append(np.ascontiguousarray(np.moveaxis(buf[sl + (slice(c * dim, (c + 1) * dim),)], -1, 0)))
    return out


def pack_cell_vector(v) -> np.ndarray:
    """(dim, *grid) -> n^dim x dim."""
    return np.ascontiguousarray(np.moveaxis(_np(v), 0, -1))


def unpack_cell_vector(buf: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.moveaxis(buf, -1, 0))


def pack_scalar(s) -> np.ndarray:
    return _np(s)[..., None]


def unpack_scalar(buf: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(buf[..., 0])


# ----------------------------------------------------------------- chunks
class RW_Cache:
    """Chunked frame streams with the reference's file naming and contents
    (3D/lfm_midpoint_simulator.py:46-165).  A stream's buffer is allocated on
    first use with the shape of the frames written (component-last, float32)."""

    def __init__(self, n_steps: int = N_STEPS):
        self.n_steps = n_steps
        self.buffer: Dict[str, dict] = {}

    def init(self):
        for b in self.buffer.values():
            b["info"].clear()
            b["file_info"].clear()

    def _stream(self, name, frame_shape):
        b = self.buffer.get(name)
        if b is None or b["buffer"] is None or b["buffer"].shape[1:] != tuple(frame_shape):
            b = {"buffer": np.zeros((self.n_steps,) + tuple(frame_shape), dtype=np.float32), "info": [],
                 "file_info": []}
            self.buffer[name] = b
        return b

    def force_write(self, name: str, dir: str):
        b = self.buffer.get(name)
        if b is not None and b["info"]:
            info = b["info"]
            np.save(os.path.join(dir, f"{name}_{info[0]}_{info[-1]}.npy"), b["buffer"])
            info.clear()

    def write_disk_with_cache(self, frame: np.ndarray, name: str, dir: str, j: int):
        """Append frame j (an already packed array) to stream ``name``; a full
        chunk is saved first (write_disk_with_cache)."""
        b = self._stream(name, frame.shape)
        info = b["info"]
        if len(info) >= self.n_steps:
            np.save(os.path.join(dir, f"{name}_{info[0]}_{info[-1]}.npy"), b["buffer"])
            info.clear()
        b["buffer"][len(info)] = frame
        info.append(int(j))

    def read_disk_with_cache(self, name: str, dir: str, j: int) -> np.ndarray:
        """Frame j of stream ``name``: from the cached chunk or from the chunk
        file whose range holds j (read_disk_with_cache)."""
        b = self.buffer.get(name)
        if b is None:
            b = {"buffer": None, "info": [], "file_info": []}
            self.buffer[name] = b
        if not b["file_info"]:
            for fname in os.listdir(dir):
                m = _CHUNK.match(fname)
                if m and fname.startswith(name + "_"):
                    b["file_info"].append((int(m.group(1)), int(m.group(2)), fname))
            b["file_info"].sort(key=lambda x: x[0])
        info = b["info"]
        if info and info[0] <= j <= info[-1]:
            return b["buffer"][info.index(j)]
        for a, z, fname in b["file_info"]:
            if a <= j <= z:
                data = np.load(os.path.join(dir, fname))
                b["buffer"] = data
                info.clear()
                info.extend(range(a, z + 1))
                return data[info.index(j)]
        raise ValueError(f"Frame {j} not found in any available file.")

    @staticmethod
    def write_disk(data, name: str, dir: str, j: int):
        if isinstance(data, (int, float)):
            arr = np.array([data])
        else:
            arr = _np(data) if isinstance(data, torch.Tensor) else np.asarray(data)
        np.save(os.path.join(dir, f"{name}_{j}.npy"), arr)

    @staticmethod
    def read_disk(name: str, dir: str, j: int) -> np.ndarray:
        path = os.path.join(dir, f"{name}_{j}.npy")
        if not os.path.exists(path):
            raise FileNotFoundError(f"File not found: {path}")
        return np.load(path)


# ------------------------------------------------------- simulator trajectories
DIRS = {"midpoint": "midpoint", "final": "final", "F": "flowmap_F", "phi": "flowmap_phi", "passive": "passive"}


def _dirs(log_dir: str, dim: int) -> Dict[str, str]:
    d = {k: os.path.join(log_dir, v) for k, v in DIRS.items()}
    d["phi_f"] = os.path.join(log_dir, "flowmap_phi_xyz" if dim == 3 else "flowmap_phi_xy")
    for p in d.values():
        os.makedirs(p, exist_ok=True)
    return d


def export_forward(sim, log_dir: str, n_steps: int = N_STEPS) -> Dict[str, str]:
    """Write a finished forward run (``sim`` after its last step_midpoint) in
    the reference's layout: midpoint velocity "u" per step, passive "s" per
    step (the value before the step; when ``sim`` keeps a passive store), per
    reinit interval "phi", the face maps ("phi_xyz" / "phi_xy") and "F", and
    final/{u_x,u_y[,u_z]}_{N}, final_ind_0 = [N], final/s_{N}.  Returns the
    directories used."""
    if sim.store_mid is None:
        raise ValueError("export_forward needs the full trajectory store (recompute=False)")
    dim = sim.dim
    d = _dirs(log_dir, dim)
    cache = RW_Cache(n_steps)
    N = sim.step_num[None] + 1
    for n in range(N):
        cache.write_disk_with_cache(pack_mac([m[n] for m in sim.store_mid]), "u", d["midpoint"], n)
        if sim.store_passive is not None:
            cache.write_disk_with_cache(pack_scalar(sim.store_passive[n]), "s", d["passive"], n)
    n_int = (N - 1) // sim.reinit_every + 1
    fname = "phi_xyz" if dim == 3 else "phi_xy"
    for k in range(n_int):
        cache.write_disk_with_cache(pack_cell_vector(sim.store_phi[k]), "phi", d["phi"], k)
        cache.write_disk_with_cache(pack_face_vectors([f[k] for f in sim.store_phi_f]), fname, d["phi_f"], k)
        cache.write_disk_with_cache(pack_face_vectors([f[k] for f in sim.store_F_f]), "F", d["F"], k)
    for c, nm in enumerate(("u_x", "u_y", "u_z")[:dim]):
        RW_Cache.write_disk(sim.u[c], nm, d["final"], N)
    RW_Cache.write_disk(N, "final_ind", d["final"], 0)
    if sim.cfg.add_passive_scalar:
        RW_Cache.write_disk(sim.passive, "s", d["final"], N)
        cache.force_write("s", d["passive"])
    cache.force_write("u", d["midpoint"])
    cache.force_write(fname, d["phi_f"])
    cache.force_write("phi", d["phi"])
    cache.force_write("F", d["F"])
    return d


def import_forward(sim, log_dir: str) -> int:
    """Load a forward trajectory written by the reference (or by export_forward)
    into ``sim``'s stores and final state, so that init_gradient and the
    adjoint steps can run without this package's forward pass.  Returns the
    final step index N.  The reference writes the maps only at reinit steps,
    so its runs end on a whole interval; export_forward also writes the map of
    a final partial interval, which this reader accepts.  The passive scalar
    per step is read when ``sim`` keeps a passive store."""
    if sim.store_mid is None:
        raise ValueError("import_forward needs the full trajectory store (recompute=False)")
    dim, res = sim.dim, sim.grid.shape
    d = _dirs(log_dir, dim)
    cache = RW_Cache()
    N = int(RW_Cache.read_disk("final_ind", d["final"], 0)[0])
    if N > sim.total_steps:
        raise ValueError(f"trajectory of {N} steps exceeds total_steps={sim.total_steps}")
    dev = sim.device

    def put(dst, arr):  # a BF16 store rounds to nearest even, as fm_convert does
        dst.copy_(torch.from_numpy(np.ascontiguousarray(arr)).to(dev))

    for n in range(N):
        comps = unpack_mac(cache.read_disk_with_cache("u", d["midpoint"], n), res)
        for c in range(dim):
            put(sim.store_mid[c][n], comps[c])
        if sim.store_passive is not None:
            put(sim.store_passive[n], unpack_scalar(cache.read_disk_with_cache("s", d["passive"], n)))
    fname = "phi_xyz" if dim == 3 else "phi_xy"
    n_int = (N - 1) // sim.reinit_every + 1
    for k in range(n_int):
        put(sim.store_phi[k], unpack_cell_vector(cache.read_disk_with_cache("phi", d["phi"], k)))
        pf = unpack_face_vectors(cache.read_disk_with_cache(fname, d["phi_f"], k), res)
        Ff = unpack_face_vectors(cache.read_disk_with_cache("F", d["F"], k), res)
        for c in range(dim):
            put(sim.store_phi_f[c][k], pf[c])
            put(sim.store_F_f[c][k], Ff[c])
    for c, nm in enumerate(("u_x", "u_y", "u_z")[:dim]):
        put(sim.u[c], RW_Cache.read_disk(nm, d["final"], N))
    if sim.cfg.add_passive_scalar:
        s = RW_Cache.read_disk("s", d["final"], N)
        put(sim.passive, s)
        if sim.store_passive is not None:
            put(sim.store_passive[N], s)
    sim.step_num[None] = N - 1
    return N
