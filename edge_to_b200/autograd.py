"""Differentiable SIMP objectives with a hand-written adjoint.

``SIMPObjective(kernel, solver, filter_kernel, material, f)`` is a callable mapping a
density tensor rho to a scalar J through a ``torch.autograd.Function``:

    forward   rho_f = H rho;  E = clip(rho_f^p, void, 1);  K(E) u = f;  J = l.u
    backward  dJ/dE_e   = -v_e^T K0 u_e   with K(E) v = l
              dJ/drho_f = dJ/dE * p clip(rho_f, void, 1)^(p-1)
              dJ/drho   = H^T dJ/drho_f

For compliance (``objective="compliance"``, l = f) the adjoint state is v = u, so the
backward needs no second solve and reproduces the reference's sensitivity chain
(TopOpt/_cuda.py:282-302 with SingleMaterial.grad, MaterialModels.py:68-71).  For a
compliant mechanism (``objective="displacement"``, l = the weights of the output DOFs,
usually with grounded springs from ``kernel.set_springs``) the backward runs a second
GMG-PCG solve for v.  The reference offers only compliance.

Between forward and backward only u is kept; the element energies are recomputed from it
(and from v) in the backward by edge_process_grad / edge_process_grad_adjoint.  Each
solve is warm-started from this objective's own previous u (or v); the solver's
``last_x0`` is left at the last solution it produced.
"""
import torch

from .kernels import _as_dev_f64


class _SIMPFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, obj):
        J, u = obj._forward(rho.detach())
        ctx.obj = obj
        ctx.save_for_backward(rho.detach(), u)
        return J

    @staticmethod
    def backward(ctx, gJ):
        rho, u = ctx.saved_tensors
        g = ctx.obj._gradient(rho, u)
        return gJ * g, None


class SIMPObjective:
    """J(rho) = l . u(rho) for a structured problem of this package.

    kernel, solver, filter_kernel, material: CuStructuredStiffnessKernel, CuMultiGrid,
    CuStructuredFilter2D/3D and SingleMaterial objects (with BCs set on the kernel).
    f: load vector; objective: "compliance" (l = f) or "displacement" (l from out_dofs and
    out_weights, default weight 1).  tol overrides the solver tolerance for these solves.
    """

    def __init__(self, kernel, solver, filter_kernel, material, f, objective="compliance", out_dofs=None,
                 out_weights=None, iteration=0, tol=None):
        self.kernel, self.solver, self.filter, self.material = kernel, solver, filter_kernel, material
        self.f = _as_dev_f64(f)
        self.iteration = iteration
        self.tol = tol
        if objective == "compliance":
            self.l = None
        elif objective == "displacement":
            if out_dofs is None:
                raise ValueError("objective='displacement' needs out_dofs")
            idx = torch.as_tensor(out_dofs, dtype=torch.long, device="cuda").reshape(-1)
            w = torch.ones(idx.numel(), dtype=torch.float64, device="cuda") if out_weights is None else \
                torch.as_tensor(out_weights, dtype=torch.float64, device="cuda").reshape(-1)
            self.l = torch.zeros_like(self.f)
            self.l.index_add_(0, idx, w)
        else:
            raise ValueError("objective must be 'compliance' or 'displacement'")
        self.objective = objective
        self._u_last = None
        self._v_last = None
        self.last = {}

    def __call__(self, rho):
        return _SIMPFunction.apply(rho, self)

    def _set_design(self, rho):
        rho_f = self.filter._matvec(rho)
        E = self.material(rho_f, self.iteration)
        self.kernel.set_rho(E)
        return rho_f

    def _solve(self, rhs, x0):
        """One GMG-PCG solve warm-started from x0 (a private copy), at self.tol if given."""
        tol_old = self.solver.tol
        if self.tol is not None:
            self.solver.tol = self.tol
        self.solver.last_x0 = None if x0 is None else x0.clone()
        try:
            x, res = self.solver.solve(rhs, use_last=x0 is not None)
        finally:
            self.solver.tol = tol_old
        return x.clone(), res

    def _forward(self, rho):
        self._set_design(_as_dev_f64(rho))
        u, res = self._solve(self.f, self._u_last)
        self._u_last = u
        l = self.f if self.l is None else self.l
        J = torch.dot(l, u)
        self.last = {"residual": res, "pcg_iters": self.solver.last_iters}
        return J, u

    def _gradient(self, rho, u):
        rho_f = self._set_design(_as_dev_f64(rho))
        if self.l is None:
            dk = self.kernel.process_grad(u).clone()
        else:
            v, res = self._solve(self.l, self._v_last)
            self._v_last = v
            self.last.update(adjoint_residual=res, adjoint_pcg_iters=self.solver.last_iters)
            dk = self.kernel.process_grad_adjoint(u, v)
        dE = self.material.grad(rho_f, self.iteration)
        return self.filter._rmatvec(dk * dE)
