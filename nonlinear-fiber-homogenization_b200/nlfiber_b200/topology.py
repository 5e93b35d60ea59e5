"""Binary cells on the GPU: periodic connected components and floating-piece removal (nlfiber/topology.py:8-63
periodic_label, spanning, remove_floating), the binarization steps of DensityMap.binary after the smoothing and
the periodic upsampling (nlfiber/density.py:96-149), in libnlf.so (nlf_topo_*, nlf_upsample_sym).

Binary arrays are NumPy bool arrays (or CUDA bool / uint8 tensors) in C order; results are NumPy arrays as the
reference returns them. Components are found by union-find on the device; the reference pads the cell by one
periodic layer and merges scipy's labels across it. The components are the same; their numbering follows each
component's first voxel in C order.
"""
import ctypes
import threading

import numpy as np

from ._lib import check, lib, ptr

_local = threading.local()


class PeriodicCells:
    """Device workspace for binary cells of side n (n^3 voxels, n^2 for d = 2). Not shared between threads."""

    def __init__(self, d, n):
        if d not in (2, 3):
            raise ValueError("d must be 2 or 3")
        self.d, self.n = int(d), int(n)
        self.shape = (self.n,) * self.d
        h = ctypes.c_void_p()
        check(lib.nlf_topo_create(ctypes.byref(h), self.d, self.n))
        self._h = h
        self._lib = lib
        self.stream = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and getattr(self, "_lib", None) is not None:
            self._lib.nlf_topo_destroy(h)
            self._h = None

    def _bytes(self, b, writable=False):
        """(buffer, NumPy array or None): a uint8 view of b usable by the library."""
        if hasattr(b, "data_ptr") and not isinstance(b, np.ndarray):
            import torch
            if tuple(b.shape) != self.shape or b.device.type != "cuda":
                raise ValueError(f"b must be a CUDA tensor of shape {self.shape}")
            t = b.contiguous()
            if t.dtype == torch.bool:
                t = t.view(torch.uint8)
            if t.dtype != torch.uint8:
                raise TypeError("b must be bool or uint8")
            return t, None
        a = np.ascontiguousarray(np.asarray(b, dtype=bool))
        if a.shape != self.shape:
            raise ValueError(f"b must have shape {self.shape}, got {a.shape}")
        if writable and not a.flags["WRITEABLE"]:
            a = a.copy()
        return a.view(np.uint8), a

    def label(self, b, faces=False):
        """nlfiber/topology.py:8-43: (labels (int64, 1..n, 0 for void), n). faces: face connectivity."""
        buf, _ = self._bytes(b)
        lab = np.empty(self.shape, dtype=np.int32)
        nc = ctypes.c_int()
        check(lib.nlf_topo_label(self._h, ptr(buf), 1 if faces else 0, lab.ctypes.data, ctypes.byref(nc),
                                 self.stream))
        return lab.astype(np.int64), int(nc.value)

    def remove_floating(self, b, counts=False):
        """nlfiber/topology.py:57-63: the spanning components of b (a new array; CUDA tensors are updated in
        place and returned). counts: also (components, spanning components)."""
        is_dev = hasattr(b, "data_ptr") and not isinstance(b, np.ndarray)
        if is_dev:
            buf, out = self._bytes(b)
            if buf.data_ptr() != b.data_ptr():
                raise ValueError("CUDA tensors must be contiguous (updated in place)")
        else:
            a = np.array(b, dtype=bool, copy=True, order="C")
            if a.shape != self.shape:
                raise ValueError(f"b must have shape {self.shape}, got {a.shape}")
            buf, out = a.view(np.uint8), a
        nc, ns = ctypes.c_int(), ctypes.c_int()
        check(lib.nlf_topo_remove_floating(self._h, ptr(buf), ctypes.byref(nc), ctypes.byref(ns), None,
                                           self.stream))
        res = b if is_dev else out
        return (res, int(nc.value), int(ns.value)) if counts else res

    def select(self, u, rank, mask=None):
        """The rank-th smallest value (0-based) of u over the voxels where mask is set (all when None)."""
        u = _f64(u, self.shape)
        mb = None if mask is None else self._bytes(mask)[0]
        out = ctypes.c_double()
        check(lib.nlf_topo_select(self._h, ptr(u), ptr(mb), int(rank), ctypes.byref(out), self.stream))
        return float(out.value)

    def binary(self, u, v, remove_floating=True, out=None):
        """nlfiber/density.py:105-122 on the smoothed field u: b = u > quantile(u, 1 - v), then floating pieces
        removed and the solid grown back towards v. Returns a NumPy bool array, or fills the CUDA tensor `out`."""
        u = _f64(u, self.shape)
        if out is None:
            b = np.empty(self.shape, dtype=bool)
            buf = b.view(np.uint8)
        else:
            buf, b = self._bytes(out)[0], out
        it = ctypes.c_int()
        check(lib.nlf_topo_binary(self._h, ptr(u), float(v), 1 if remove_floating else 0, ptr(buf),
                                  ctypes.byref(it), self.stream))
        self.last_rounds = int(it.value)
        return b


def _f64(u, shape):
    if hasattr(u, "data_ptr") and not isinstance(u, np.ndarray):
        import torch
        if u.dtype != torch.float64 or tuple(u.shape) != shape:
            raise ValueError(f"u must be a float64 tensor of shape {shape}")
        return u.contiguous()
    u = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
    if u.shape != shape:
        raise ValueError(f"u must have shape {shape}, got {u.shape}")
    return u


def cells(d, n):
    """The calling thread's workspace for side n (kept for reuse)."""
    c = getattr(_local, "cells", None)
    if c is None:
        c = _local.cells = {}
    key = (int(d), int(n))
    if key not in c:
        c[key] = PeriodicCells(d, n)
    return c[key]


def _structure_faces(b, connectivity):
    if connectivity is None:
        return False
    st = np.asarray(connectivity, dtype=bool)
    d = np.ndim(b)
    if st.shape != (3,) * d:
        raise ValueError("connectivity must be a 3^d structure")
    if st.all():
        return False
    g = np.indices((3,) * d) - 1
    faces = np.abs(g).sum(axis=0) <= 1
    if np.array_equal(st, faces):
        return True
    raise ValueError("connectivity: the full 3^d neighbourhood or the faces (generate_binary_structure(d, 1))")


def periodic_label(b, connectivity=None):
    """nlfiber/topology.py:8-43: connected components of a periodic binary array, (labels, n). connectivity:
    None (26 / 8 neighbours) or the face structure ndimage.generate_binary_structure(d, 1)."""
    b = np.asarray(b, dtype=bool) if not hasattr(b, "data_ptr") else b
    return cells(np.ndim(b) if isinstance(b, np.ndarray) else b.dim(), b.shape[0]).label(
        b, faces=_structure_faces(b, connectivity))


def remove_floating(b):
    """nlfiber/topology.py:57-63: keep only the spanning solid components."""
    d = np.ndim(b) if isinstance(b, np.ndarray) or not hasattr(b, "dim") else b.dim()
    return cells(d, b.shape[0]).remove_floating(b)


def upsample_sym(u, f):
    """exact_symmetrize(upsample_periodic(u, f)) (nlfiber/density.py:104,133-149): u of side n (CUDA float64
    tensor or NumPy) -> CUDA float64 tensor of side 2 (m / 2), m = round(n f)."""
    import torch
    d = u.dim() if hasattr(u, "dim") else np.ndim(u)
    n = u.shape[0]
    m = int(round(n * f))
    s = 2 * (m // 2)
    src = u.contiguous() if hasattr(u, "data_ptr") else np.ascontiguousarray(np.asarray(u, dtype=np.float64))
    out = torch.empty((s,) * d, dtype=torch.float64, device="cuda")
    check(lib.nlf_upsample_sym(d, n, m, ptr(src), ptr(out), None))
    return out
