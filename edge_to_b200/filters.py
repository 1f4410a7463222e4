"""Cone density filter on structured grids, drop-in for CuStructuredFilter2D/3D
(geom/_filters.py:164-254).

The stencil is built exactly as the reference does (offsets within ceil(r_min), weights
(r_min - |o*scale|)/r_min kept where positive and normalised to sum 1); the filter and its
exact transpose run in libedge_b200.so with boundary renormalisation.
"""
import ctypes

import numpy as np
import torch

from . import _lib


class _TransposeView:
    def __init__(self, original):
        self._original = original

    def __matmul__(self, rhs):
        return self._original._rmatvec(rhs)

    def dot(self, rhs):
        return self._original._rmatvec(rhs)

    @property
    def T(self):
        return self._original


class FilterKernel:
    def __init__(self):
        self.weights = None
        self.offsets = None
        self.shape = None
        self.matvec = self.dot

    def dot(self, rho):
        if isinstance(rho, type(self.weights)):
            if rho.ndim == 1:
                if rho.shape[0] == self.shape[1]:
                    return self._matvec(rho)
                raise ValueError("Input vector size does not match the filter kernel size.")
            raise NotImplementedError("Only vector inputs are supported.")
        raise ValueError(f"Input must be a {type(self.weights)} array vector.")

    def __matmul__(self, rhs):
        return self.dot(rhs)

    @property
    def T(self):
        return _TransposeView(self)


def cone_stencil(dim, h, r_min):
    """Offsets (n, dim) and normalised weights of the cone filter (geom/_filters.py:175-195)."""
    scales = np.asarray(h, dtype=np.float64)
    scales = scales / scales.min()
    n = int(np.ceil(r_min))
    rng = np.arange(-n, n + 1, dtype=np.int32)
    grids = np.meshgrid(*([rng] * dim), indexing="ij")
    offsets = np.vstack([g.ravel() for g in grids]).T.astype(np.int32)
    dist = np.linalg.norm(offsets * scales[None], axis=1)
    w = (r_min - dist) / r_min
    keep = w > 0
    offsets, w = offsets[keep], w[keep]
    return offsets, w / w.sum()


class _CuStructuredFilter(FilterKernel):
    def _setup(self, mesh, r_min, dim, h):
        self.r_min = r_min
        self.dtype = mesh.dtype
        self.nel = [int(v) for v in mesh.nel]
        n = int(np.prod(self.nel))
        self.shape = (n, n)
        offs, w = cone_stencil(dim, h, r_min)
        self.offsets = torch.as_tensor(offs, device="cuda")
        self.weights = torch.as_tensor(w, dtype=torch.float64, device="cuda")
        off3 = np.zeros((offs.shape[0], 3), dtype=np.int32)
        off3[:, :dim] = offs
        hnd = ctypes.c_void_p()
        _lib.call("edge_filter_create", dim, _lib.int_array(self.nel + [1] * (3 - dim)), int(offs.shape[0]),
                  off3.ravel().ctypes.data_as(_lib.c_int_p), np.ascontiguousarray(w).ctypes.data_as(_lib.c_double_p),
                  ctypes.byref(hnd))
        self._h = hnd
        self._norm = None

    @property
    def handle(self):
        return self._h

    @property
    def normalizer(self):
        """N_e = sum of the in-bounds tap weights (get_filter_weights_{2D,3D}); informational."""
        if self._norm is None:
            self._norm = self._compute_norm()
        return self._norm

    def _compute_norm(self):
        nel = np.array(self.nel)
        offs = self.offsets.cpu().numpy()
        w = self.weights.cpu().numpy()
        idx = np.stack(np.meshgrid(*[np.arange(n) for n in nel], indexing="ij"), -1).reshape(-1, len(nel))
        N = np.zeros(idx.shape[0])
        for o, wk in zip(offs, w):
            nb = idx + o[None]
            N += wk * np.all((nb >= 0) & (nb < nel[None]), axis=1)
        return torch.as_tensor(N, device="cuda")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().edge_filter_destroy(h)
            except Exception:
                pass
            self._h = None

    def _prep(self, v):
        if isinstance(v, np.ndarray):
            v = torch.from_numpy(v)
        return v.to(device="cuda", dtype=torch.float64).contiguous()

    def _matvec(self, rho):
        x = self._prep(rho)
        out = torch.empty_like(x)
        _lib.call("edge_filter_apply", self._h, _lib.ptr(x), _lib.ptr(out), _lib.stream_ptr())
        return out

    def _rmatvec(self, rho):
        x = self._prep(rho)
        out = torch.empty_like(x)
        _lib.call("edge_filter_apply_T", self._h, _lib.ptr(x), _lib.ptr(out), _lib.stream_ptr())
        return out


class CuStructuredFilter3D(_CuStructuredFilter):
    def __init__(self, mesh, r_min):
        super().__init__()
        self.nelx, self.nely, self.nelz = int(mesh.nel[0]), int(mesh.nel[1]), int(mesh.nel[2])
        self._setup(mesh, r_min, 3, [mesh.dx, mesh.dy, mesh.dz])


class CuStructuredFilter2D(_CuStructuredFilter):
    def __init__(self, mesh, r_min):
        super().__init__()
        self.nelx, self.nely = int(mesh.nel[0]), int(mesh.nel[1])
        self._setup(mesh, r_min, 2, [mesh.dx, mesh.dy])


StructuredFilter2D = CuStructuredFilter2D
StructuredFilter3D = CuStructuredFilter3D


class CuGeneralFilter(FilterKernel):
    """Cone density filter of an unstructured mesh, drop-in for CuGeneralFilter
    (geom/_filters.py:278-298 with filter_kernel_{2D,3D}_general, core/_filter.py:126-182):
    for every element the element centroids within r_min (a KD-tree ball query, closed
    ball), weights (r_min - d) / r_min normalised to sum 1 per row.  The matrix is built on
    the host once; H and H^T are applied on the device (edge_csr_apply, a transpose stored
    beside H so both products are gathers in a fixed order)."""

    def __init__(self, mesh, r_min):
        super().__init__()
        from scipy.spatial import cKDTree
        self.dtype = mesh.dtype
        self.nd = int(np.asarray(mesh.nodes).shape[1])
        cent = np.asarray(mesh.centeroids, dtype=np.float64)
        n = cent.shape[0]
        tree = cKDTree(cent)
        rows = tree.query_ball_point(cent, r_min)
        indptr = np.zeros(n + 1, dtype=np.int64)
        idx, val = [], []
        for i, nb in enumerate(rows):
            nb = np.asarray(sorted(nb), dtype=np.int64)
            w = (r_min - np.linalg.norm(cent[nb] - cent[i], axis=-1)) / r_min
            idx.append(nb)
            val.append(w / w.sum())
            indptr[i + 1] = indptr[i] + nb.size
        self._indptr = indptr
        self._indices = np.ascontiguousarray(np.concatenate(idx).astype(np.int32))
        self._data = np.ascontiguousarray(np.concatenate(val))
        self.shape = (n, n)
        self.weights = torch.as_tensor(self._data, device="cuda")
        h = ctypes.c_void_p()
        _lib.call("edge_csr_create", n, indptr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                  self._indices.ctypes.data_as(_lib.c_int_p), self._data.ctypes.data_as(_lib.c_double_p),
                  ctypes.byref(h))
        self._h = h

    @property
    def kernel(self):
        """H as a torch sparse CSR matrix on the device (the reference keeps a cupy CSR)."""
        return torch.sparse_csr_tensor(torch.as_tensor(self._indptr), torch.as_tensor(self._indices.astype(np.int64)),
                                       torch.as_tensor(self._data), size=self.shape).to("cuda")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().edge_csr_destroy(h)
            except Exception:
                pass
            self._h = None

    def _apply(self, rho, transpose):
        if isinstance(rho, np.ndarray):
            rho = torch.from_numpy(rho)
        x = rho.to(device="cuda", dtype=torch.float64).contiguous().reshape(-1)
        out = torch.empty_like(x)
        _lib.call("edge_csr_apply", self._h, _lib.ptr(x), _lib.ptr(out), 1 if transpose else 0, _lib.stream_ptr())
        return out.reshape(rho.shape)

    def _matvec(self, rho):
        return self._apply(rho, False)

    def _rmatvec(self, rho):
        return self._apply(rho, True)


GeneralFilter = CuGeneralFilter
