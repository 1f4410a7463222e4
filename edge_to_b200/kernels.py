"""Matrix-free structured stiffness kernel K(rho), drop-in for StructuredStiffnessKernel
(kernels/_cuda.py:62-302) on CuStructuredMesh2D/3D.

Vectors are torch CUDA tensors in the reference layout (FP64, v[node*dof + c]); the
operator itself runs in libedge_b200.so (hand-written sm_100a kernels).  As in the
reference, ``dot`` returns a buffer that the next call overwrites
(kernels/_cuda.py:175-204), and constrained DOFs act as identity rows/columns.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def _as_dev_f64(x, name="array"):
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(x)
    if not isinstance(x, torch.Tensor):
        raise NotImplementedError("Only torch tensors (or numpy arrays) are supported as vectors.")
    if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous():
        x = x.to(device="cuda", dtype=torch.float64).contiguous()
    return x


class StiffnessKernel:
    def __init__(self):
        self.has_rho = False
        self.rho = None
        self.shape = None
        self.matvec = self.dot
        self.rmatvec = self.dot

    def __matmul__(self, rhs):
        return self.dot(rhs)


class CuStructuredStiffnessKernel(StiffnessKernel):
    def __init__(self, mesh):
        super().__init__()
        self.mesh = mesh
        self.dof = mesh.dof
        self.K_single = mesh.K_single
        self.dtype = mesh.dtype
        self.elements_size = mesh.elements_size
        self.n_nodes = mesh.n_nodes
        self.n_elements = mesh.n_elements
        self.dim = len(mesh.nel)
        self.shape = (self.n_nodes * self.dof, self.n_nodes * self.dof)
        self.constraints = torch.zeros(self.n_nodes * self.dof, dtype=torch.bool, device="cuda")
        self.has_con = False
        self.mat_vec = None
        self.diag = None
        self.dk = None
        h = ctypes.c_void_p()
        nel = _lib.int_array(list(mesh.nel) + [1] * (3 - self.dim))
        K0 = np.ascontiguousarray(np.asarray(mesh.K_single, dtype=np.float64))
        _lib.call("edge_problem_create", self.dim, nel, K0.ctypes.data_as(_lib.c_double_p), _lib.EDGE_FP64,
                  ctypes.byref(h))
        self._h = h
        self._bind_stream()

    # --------------------------------------------------------------- plumbing
    @property
    def handle(self):
        return self._h

    def _bind_stream(self):
        _lib.call("edge_set_stream", self._h, _lib.stream_ptr())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().edge_problem_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def uses_transform(self):
        return bool(_lib.lib().edge_uses_transform(self._h))

    # --------------------------------------------------------------- reference API
    def set_rho(self, rho):
        rho = _as_dev_f64(rho)
        if rho.numel() != self.n_elements:
            raise ValueError("rho size does not match the number of elements.")
        self.rho = rho
        self._bind_stream()
        _lib.call("edge_set_rho", self._h, _lib.ptr(rho))
        self.has_rho = True

    def _push_constraints(self):
        self._bind_stream()
        c = self.constraints.to(torch.uint8).contiguous()
        _lib.call("edge_set_constraints", self._h, _lib.ptr(c))
        torch.cuda.current_stream().synchronize()

    def set_constraints(self, constraints):
        self.constraints[:] = False
        idx = torch.as_tensor(np.asarray(constraints, dtype=np.int64) if not isinstance(constraints, torch.Tensor)
                              else constraints, device="cuda").long()
        if idx.numel():
            self.constraints[idx] = True
        self.has_con = True
        self._push_constraints()

    def add_constraints(self, constraints):
        idx = torch.as_tensor(np.asarray(constraints, dtype=np.int64) if not isinstance(constraints, torch.Tensor)
                              else constraints, device="cuda").long()
        if idx.numel():
            self.constraints[idx] = True
        self.has_con = True
        self._push_constraints()

    def reset(self):
        self.has_rho = False
        self.rho = None
        self.constraints[:] = False
        self.has_con = False
        self._push_constraints()
        self.mat_vec = None
        self.diag = None
        self.dk = None

    def _matvec(self, rho, vec):
        if rho is not self.rho:
            self.set_rho(rho)
        return self.dot(vec)

    def _rmatvec(self, rho, vec):
        return self._matvec(rho, vec)

    def dot(self, rhs):
        if not self.has_rho:
            raise ValueError("Rho has not been set. dot works only after setting rho.")
        if not isinstance(rhs, (torch.Tensor, np.ndarray)):
            raise NotImplementedError("Only torch tensors as vectors are supported.")
        if rhs.shape[0] != self.n_nodes * self.dof:
            raise ValueError("Shape of the input vector does not match the number of nodes and dof.")
        u = _as_dev_f64(rhs)
        if self.mat_vec is None:
            self.mat_vec = torch.empty(self.shape[0], dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_matvec", self._h, _lib.ptr(u), _lib.ptr(self.mat_vec))
        return self.mat_vec

    def dot_dense(self, rhs):
        """The same product through the dense node-centric kernel (cross-check path)."""
        u = _as_dev_f64(rhs)
        out = torch.empty(self.shape[0], dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_matvec_dense", self._h, _lib.ptr(u), _lib.ptr(out))
        return out

    def diagonal(self, rho=None):
        if rho is None and not self.has_rho:
            raise ValueError("Rho has not been set. diagonal works only after setting rho or if rho is provided.")
        if rho is not None:
            self.set_rho(rho)
        if self.diag is None:
            self.diag = torch.empty(self.shape[0], dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_diagonal", self._h, _lib.ptr(self.diag))
        return self.diag

    def process_grad(self, U):
        U = _as_dev_f64(U)
        if self.dk is None:
            self.dk = torch.empty(self.n_elements, dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_process_grad", self._h, _lib.ptr(U), _lib.ptr(self.dk))
        return self.dk

    def fea_integrals(self, w, U, B, D):
        """Per-element strain = B u_e, stress = D strain and strain energy 1/2 w_e u_e^T K0 u_e
        (the structured path of TopOpt/_solver.py:80-137); B, D: the mesh's B_single, D_single.
        Returns (strain [n_el, nb], stress [n_el, nb], strain_energy [n_el]) on the device."""
        w = _as_dev_f64(w)
        U = _as_dev_f64(U)
        Bt = torch.as_tensor(np.ascontiguousarray(np.asarray(B, dtype=np.float64)), device="cuda")
        Dt = torch.as_tensor(np.ascontiguousarray(np.asarray(D, dtype=np.float64)), device="cuda")
        nb = Bt.shape[0]
        if Bt.shape[1] != self.elements_size * self.dof or Dt.shape != (nb, nb):
            raise ValueError("B must be nb x (element nodes * dof) and D nb x nb")
        if w.numel() != self.n_elements or U.numel() != self.shape[0]:
            raise ValueError("weights / displacement size does not match the mesh")
        strain = torch.empty((self.n_elements, nb), dtype=torch.float64, device="cuda")
        stress = torch.empty_like(strain)
        energy = torch.empty(self.n_elements, dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_fea_integrals", self._h, _lib.ptr(U), _lib.ptr(w), _lib.ptr(Bt), _lib.ptr(Dt), int(nb),
                  _lib.ptr(strain), _lib.ptr(stress), _lib.ptr(energy))
        return strain, stress, energy

    # --------------------------------------------------------------- beyond the reference
    def set_springs(self, dofs, stiffness):
        """Grounded point springs K_ii += k on DOF indices ``dofs`` (the compliant-mechanism
        input/output springs); every product and PCG solve includes them.  ``dofs=[]``
        removes them.  The reference has no springs (its only objective is compliance)."""
        d = np.ascontiguousarray(np.asarray(dofs, dtype=np.int64).reshape(-1))
        k = np.broadcast_to(np.asarray(stiffness, dtype=np.float64), d.shape).copy()
        self._bind_stream()
        _lib.call("edge_set_springs", self._h, int(d.size), d.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                  k.ctypes.data_as(_lib.c_double_p))
        self.springs = (d, k)

    def process_grad_adjoint(self, U, V):
        """dk_e = -v_e^T K0 u_e: the element sensitivity dJ/dE_e of a linear objective
        J = l.u whose adjoint solution K v = l is V (for compliance V = U and this equals
        process_grad)."""
        U = _as_dev_f64(U)
        V = _as_dev_f64(V)
        out = torch.empty(self.n_elements, dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_process_grad_adjoint", self._h, _lib.ptr(U), _lib.ptr(V), _lib.ptr(out))
        return out


StructuredStiffnessKernel = CuStructuredStiffnessKernel


class _CuGeneralKernel(StiffnessKernel):
    """Matrix-free stiffness operator of an unstructured mesh (CuGeneralMesh): the reference's
    UniformStiffnessKernel / GeneralStiffnessKernel (kernels/_cuda.py:305-815).  The element
    matrices come from the mesh (``Ks`` stacked when uniform, ``K_flat``/``K_ptr`` otherwise);
    the product, diagonal and sensitivities run in libedge_b200.so (edge_gen_*), FP64."""

    def __init__(self, mesh):
        super().__init__()
        self.mesh = mesh
        self.nodes, self.elements = mesh.nodes, mesh.elements
        self.dof = int(mesh.dof)
        self.dtype = mesh.dtype
        self.n_nodes = int(mesh.nodes.shape[0])
        self.n_elements = int(mesh.n_elements)
        self.shape = (self.n_nodes * self.dof, self.n_nodes * self.dof)
        self.constraints = torch.zeros(self.n_nodes * self.dof, dtype=torch.bool, device="cuda")
        self.has_con = False
        sizes = np.asarray(mesh.element_sizes, dtype=np.int64)
        if mesh.is_uniform:
            Ks = np.asarray(mesh.Ks, dtype=np.float64)
            K_flat = np.ascontiguousarray(Ks.reshape(-1))
            nk2 = Ks.shape[1] * Ks.shape[2]
            K_ptr = np.arange(self.n_elements + 1, dtype=np.int64) * nk2
        else:
            K_flat = np.ascontiguousarray(np.asarray(mesh.K_flat, dtype=np.float64))
            K_ptr = np.asarray(mesh.K_ptr, dtype=np.int64)
        self._K_flat, self._K_ptr, self._sizes = K_flat, K_ptr, sizes
        self.elements_flat = np.ascontiguousarray(np.asarray(mesh.elements_flat, dtype=np.int32))
        self.elements_ptr = np.ascontiguousarray(np.asarray(mesh.elements_ptr, dtype=np.int32))
        h = ctypes.c_void_p()
        _lib.call("edge_gen_create", self.dof, self.n_nodes, self.n_elements,
                  self.elements_ptr.ctypes.data_as(_lib.c_int_p), self.elements_flat.ctypes.data_as(_lib.c_int_p),
                  K_flat.ctypes.data_as(_lib.c_double_p), K_ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                  ctypes.byref(h))
        self._h = h
        self.mat_vec = None
        self.diag = None
        self.dk = None

    @property
    def handle(self):
        return self._h

    def _bind_stream(self):
        _lib.call("edge_gen_set_stream", self._h, _lib.stream_ptr())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().edge_gen_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_rho(self, rho):
        rho = _as_dev_f64(rho).reshape(-1)
        if rho.numel() != self.n_elements:
            raise ValueError("rho size does not match the number of elements.")
        self.rho = rho
        self._bind_stream()
        _lib.call("edge_gen_set_rho", self._h, _lib.ptr(rho))
        self.has_rho = True

    def _push_constraints(self):
        self._bind_stream()
        c = self.constraints.to(torch.uint8).contiguous()
        _lib.call("edge_gen_set_constraints", self._h, _lib.ptr(c))
        torch.cuda.current_stream().synchronize()

    def set_constraints(self, constraints):
        self.constraints[:] = False
        idx = torch.as_tensor(np.asarray(constraints, dtype=np.int64) if not isinstance(constraints, torch.Tensor)
                              else constraints, device="cuda").long()
        if idx.numel():
            self.constraints[idx] = True
        self.has_con = True
        self._push_constraints()

    def add_constraints(self, constraints):
        idx = torch.as_tensor(np.asarray(constraints, dtype=np.int64) if not isinstance(constraints, torch.Tensor)
                              else constraints, device="cuda").long()
        if idx.numel():
            self.constraints[idx] = True
        self.has_con = True
        self._push_constraints()

    def _matvec(self, rho, vec):
        if rho is not self.rho:
            self.set_rho(rho)
        v = _as_dev_f64(vec)
        if self.mat_vec is None:
            self.mat_vec = torch.empty(self.shape[0], dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_gen_matvec", self._h, _lib.ptr(v), _lib.ptr(self.mat_vec))
        return self.mat_vec

    def _rmatvec(self, rho, vec):
        return self._matvec(rho, vec)

    def dot(self, rhs):
        if not self.has_rho:
            raise ValueError("Rho has not been set. dot works only after setting rho.")
        if not isinstance(rhs, (torch.Tensor, np.ndarray)):
            raise NotImplementedError("Only torch tensors (or numpy arrays) are supported.")
        if rhs.shape[0] != self.shape[0]:
            raise ValueError("Shape of the input vector does not match the number of nodes and dof.")
        return self._matvec(self.rho, rhs)

    def diagonal(self, rho=None):
        if rho is None and not self.has_rho:
            raise ValueError("Rho has not been set. diagonal works only after setting rho or if rho is provided.")
        if rho is not None:
            self.set_rho(rho)
        if self.diag is None:
            self.diag = torch.empty(self.shape[0], dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_gen_diagonal", self._h, _lib.ptr(self.diag))
        return self.diag

    def process_grad(self, U):
        U = _as_dev_f64(U)
        if self.dk is None:
            self.dk = torch.empty(self.n_elements, dtype=torch.float64, device="cuda")
        self._bind_stream()
        _lib.call("edge_gen_process_grad", self._h, _lib.ptr(U), _lib.ptr(self.dk))
        return self.dk

    def construct(self, rho):
        """K(rho) with constrained rows/columns -> identity as a torch sparse CSR matrix on the
        device (the reference's construct, kernels/_cuda.py:407-420), assembled on the host
        from the element matrices."""
        r = _as_dev_f64(rho).reshape(-1).cpu().numpy()
        dof = self.dof
        rows, cols, vals = [], [], []
        ptr, flat = self.elements_ptr, self.elements_flat
        for e in range(self.n_elements):
            nodes = flat[ptr[e]:ptr[e + 1]].astype(np.int64)
            d = (nodes[:, None] * dof + np.arange(dof)[None, :]).reshape(-1)
            Ke = self._K_flat[self._K_ptr[e]:self._K_ptr[e + 1]].reshape(d.size, d.size)
            rows.append(np.repeat(d, d.size))
            cols.append(np.tile(d, d.size))
            vals.append(r[e] * Ke.reshape(-1))
        rows, cols, vals = map(np.concatenate, (rows, cols, vals))
        cons = self.constraints.cpu().numpy()
        keep = ~(cons[rows] | cons[cols])
        ci = np.nonzero(cons)[0]
        rows = np.concatenate([rows[keep], ci])
        cols = np.concatenate([cols[keep], ci])
        vals = np.concatenate([vals[keep], np.ones(ci.size)])
        n = self.shape[0]
        order = np.lexsort((cols, rows))
        rows, cols, vals = rows[order], cols[order], vals[order]
        key = rows * n + cols
        uniq, start = np.unique(key, return_index=True)
        summed = np.add.reduceat(vals, start)
        r_u, c_u = uniq // n, uniq % n
        indptr = np.zeros(n + 1, dtype=np.int64)
        np.add.at(indptr, r_u + 1, 1)
        indptr = np.cumsum(indptr)
        return torch.sparse_csr_tensor(torch.as_tensor(indptr), torch.as_tensor(c_u), torch.as_tensor(summed),
                                       size=(n, n), dtype=torch.float64).to("cuda")


class CuUniformStiffnessKernel(_CuGeneralKernel):
    """Unstructured mesh of one element kind (kernels/_cuda.py:305-552)."""

    def __init__(self, mesh):
        if not mesh.is_uniform:
            raise ValueError("Mesh is not uniform, you should use GeneralStiffnessKernel instead.")
        super().__init__(mesh)


class CuGeneralStiffnessKernel(_CuGeneralKernel):
    """Unstructured mesh of mixed element kinds (kernels/_cuda.py:554-815)."""

    def __init__(self, mesh):
        if mesh.is_uniform:
            raise ValueError("Mesh is uniform, you should use UniformStiffnessKernel instead.")
        super().__init__(mesh)
