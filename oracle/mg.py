"""Geometric-multigrid-preconditioned CG, FP64 (oracle; test infrastructure).

Restates ``MultiGrid`` (solvers/_multigrid.py:11-230, GPU twin
solvers/_multigrid_cuda.py:15-242):

* levels: A_0 = K(E) with BCs; A_{l+1} = R A_l R^T (Galerkin), D_l = 1/diag(A_l);
  the coarsest level is solved exactly (SuperLU, solvers/_multigrid.py:108-121).
* V-cycle (solvers/_multigrid.py:123-176): n_smooth damped-Jacobi sweeps with
  omega*1.06^level, residual, restriction, recursion from zero, prolongation, n_smooth
  sweeps on the correction against the restricted-level residual, x += e.  The
  reference's 'W' default never triggers its second visit (it tests cycle == 'w').
* PCG (solvers/_multigrid.py:178-230): warm start from the last solution, relative
  residual ||r||/||f|| < tol, omega = min + (d/2) exp((-clip(R, tol, 0.1) + tol) * 500).

variant="gpu" follows the CuPy solver: omega reset to min_omega at every solve
(solvers/_multigrid_cuda.py:210) and the GPU restriction table.  variant="cpu" follows
the NumPy/Numba solver: omega carried over between solves and the 2-D CPU restriction.
"""
import numpy as np
import scipy.sparse.linalg as spla

from . import ops
from .grid import Grid


class MultiGridOracle:
    def __init__(self, grid: Grid, maxiter=1000, tol=1e-5, n_smooth=3, omega=0.5, n_level=3,
                 cycle="W", w_level=1, min_omega=0.4, variant="gpu"):
        self.grid = grid
        self.maxiter = maxiter
        self.tol = tol
        self.n_smooth = n_smooth
        self.omega = omega
        self.max_omega = omega
        self.min_omega = max(omega / 2, min_omega)
        self.d_omega = self.max_omega - self.min_omega
        self.n_level = n_level
        self.cycle = cycle
        self.w_level = [w_level] if isinstance(w_level, int) else list(w_level)
        self.variant = variant
        self.last_x0 = None
        self.pcg_iters = []

    def setup(self, A0):
        self.levels = [(A0, 1.0 / ops.diagonal(A0))]
        self.grids = [self.grid]
        self.R = []
        self.P = []
        g = self.grid
        A = A0
        for _ in range(self.n_level):
            self.R.append(ops.restriction_matrix(g, self.variant))
            self.P.append(ops.prolongation_matrix(g))
            A = ops.galerkin(A, g)
            g = g.coarse()
            self.grids.append(g)
            self.levels.append((A, 1.0 / A.diagonal()))
        self.coarse = spla.splu(self.levels[-1][0].tocsc())

    def _smooth(self, x, b, A, Dinv, n):
        for _ in range(n):
            x += self.omega * Dinv * (b - A @ x)
        return x

    def vcycle(self, x, b, level):
        if level == self.n_level:
            return self.coarse.solve(b)
        A, Dinv = self.levels[level]
        self.omega = self.omega * (1.06) ** level
        x = self._smooth(x, b, A, Dinv, self.n_smooth)
        self.omega = self.omega / (1.06) ** level
        r = b - A @ x
        rc = self.R[level] @ r
        e = self.vcycle(rc * 0.0, rc, level + 1)
        e = self.P[level] @ e
        self.omega = self.omega * (1.06) ** level
        e = self._smooth(e, r, A, Dinv, self.n_smooth)
        self.omega = self.omega / (1.06) ** level
        x += e
        if self.cycle == "w" and level in self.w_level:
            r = b - A @ x
            rc = self.R[level] @ r
            e = self.vcycle(rc * 0.0, rc, level + 1)
            e = self.P[level] @ e
            self.omega = self.omega * (1.06) ** level
            e = self._smooth(e, r, A, Dinv, self.n_smooth)
            self.omega = self.omega / (1.06) ** level
            x += e
        return x

    def solve(self, A0, rhs, use_last=True):
        """Returns (x, relative residual); never raises on non-convergence."""
        if use_last and self.last_x0 is not None:
            x = self.last_x0
        else:
            x = np.zeros_like(rhs)
        self.setup(A0)
        if self.variant == "gpu":
            self.omega = self.min_omega
        r = rhs - A0 @ x
        z = self.vcycle(np.zeros_like(r), r, 0)
        p = z.copy()
        rho_old = float(r @ z)
        norm_b = float(np.sqrt(rhs @ rhs))
        it = 0
        norm_r = float(np.sqrt(r @ r))
        for it in range(self.maxiter):
            q = A0 @ p
            alpha = rho_old / float(p @ q)
            x += alpha * p
            r -= alpha * q
            norm_r = float(np.sqrt(r @ r))
            R = norm_r / norm_b
            if R < self.tol:
                break
            self.omega = self.min_omega + self.d_omega / 2 * np.exp((-np.clip(R, self.tol, 1e-1) + self.tol) * 500)
            z = self.vcycle(np.zeros_like(r), r, 0)
            rho_new = float(r @ z)
            beta = rho_new / rho_old
            p = z + beta * p
            rho_old = rho_new
        self.pcg_iters.append(it + 1)
        self.last_x0 = x
        return x, norm_r / norm_b
