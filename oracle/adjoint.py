"""Objective values and adjoint gradients of the SIMP chain, FP64 (oracle; test infrastructure).

The chain rho -> rho_f = H rho -> E = clip(rho_f^p, void, 1) -> K(E) u = f -> J = l.u is the
reference's solve_and_process (TopOpt/_cuda.py:282-302, CPU TopOpt/_solver.py:313-334) with
SingleMaterial (MaterialModels.py:47-73).  For compliance (l = f) the gradient is the
reference's dr.  The compliant-mechanism objective (l = unit vector at the output DOF, with
grounded springs on the input and output DOFs) has no counterpart in the reference; its
gradient here is the textbook adjoint dJ/dE_e = -v_e^T K0 u_e with K v = l, and it is
checked against central finite differences (parity unpinned against the reference).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import ops


def stiffness(grid, K0, E, cons, springs=None):
    """K(E) with identity rows/columns on constrained DOFs, plus grounded springs on the
    unconstrained spring DOFs (springs = (dofs, k))."""
    K = ops.assemble(grid, K0, E, cons)
    if springs is not None and len(springs[0]):
        d = np.zeros(grid.n_dof)
        mask = np.zeros(grid.n_dof, dtype=bool)
        if cons is not None and len(cons):
            mask[np.asarray(cons)] = True
        dofs, k = np.asarray(springs[0]), np.broadcast_to(np.asarray(springs[1], dtype=float), np.shape(springs[0]))
        for i, ki in zip(dofs, k):
            if not mask[i]:
                d[i] += ki
        K = (K + sp.diags(d)).tocsr()
    return K


class Objective:
    """J(rho) = l.u and its gradient for one structured problem (FP64, direct solves)."""

    def __init__(self, grid, K0, H, f, cons, penalty=3.0, void=1e-9, l=None, springs=None):
        self.grid, self.K0, self.H = grid, K0, H
        self.f = np.asarray(f, dtype=float)
        self.cons = np.asarray(cons if cons is not None else [], dtype=np.int64)
        self.penalty, self.void = penalty, void
        self.l = self.f if l is None else np.asarray(l, dtype=float)
        self.springs = springs

    def _state(self, rho):
        rho_f = ops.filter_apply(self.H, rho)
        E = np.clip(rho_f ** self.penalty, self.void, 1.0)
        K = stiffness(self.grid, self.K0, E, self.cons, self.springs)
        return rho_f, E, K

    def value(self, rho):
        _, _, K = self._state(rho)
        u = spla.spsolve(K.tocsc(), self.f)
        return float(self.l @ u)

    def gradient(self, rho):
        rho_f, E, K = self._state(rho)
        lu = spla.splu(K.tocsc())
        u = lu.solve(self.f)
        v = u if self.l is self.f else lu.solve(self.l)
        dm = self.grid.dof_map()
        dk = -np.einsum("ea,ab,eb->e", v[dm], self.K0, u[dm])
        dE = self.penalty * np.clip(rho_f, self.void, 1.0) ** (self.penalty - 1)
        return ops.filter_apply_T(self.H, dk * dE), float(self.l @ u)


def central_differences(fun, rho, idx, h=1e-4):
    """(J(rho + h e_i) - J(rho - h e_i)) / 2h for i in idx."""
    out = np.empty(len(idx))
    for n, i in enumerate(idx):
        rp = rho.copy()
        rp[i] += h
        rm = rho.copy()
        rm[i] -= h
        out[n] = (fun(rp) - fun(rm)) / (2 * h)
    return out


def inverter_problem(nelx, nely):
    """Compliant-mechanism inverter on nelx x nely Q4 elements: unit force in +x at the
    left-mid node (input), objective the x displacement of the right-mid node (output),
    grounded springs on both, the left edge's top and bottom nelx//40+1 nodes clamped.
    Returns (grid-free description): f, l, cons, springs as DOF arrays."""
    nx, ny = nelx + 1, nely + 1
    node = lambda i, j: j * nx + i          # noqa: E731  (2-D numbering, core/_geom.py:20-25)
    jm = nely // 2
    n_in, n_out = node(0, jm), node(nelx, jm)
    f = np.zeros(2 * nx * ny)
    f[2 * n_in] = 1.0
    l = np.zeros(2 * nx * ny)
    l[2 * n_out] = 1.0
    m = max(1, nely // 40 + 1)
    clamp = [node(0, j) for j in range(m)] + [node(0, nely - j) for j in range(m)]
    cons = np.array(sorted({2 * c + d for c in clamp for d in range(2)}), dtype=np.int64)
    springs = (np.array([2 * n_in, 2 * n_out], dtype=np.int64), np.array([0.1, 0.1]))
    return f, l, cons, springs
