"""SIMP minimum-compliance loop with the OC update, FP64 (oracle; test infrastructure).

Restates TopOpt.optimize / solve_and_process / update_design (TopOpt/_solver.py:271-417,
GPU twin TopOpt/_cuda.py:242-382) with SingleMaterial (MaterialModels.py:31-99):

  rho_f = H rho;  E = clip(rho_f^p, void, 1);  solve K(E) U = f;  c = f.U
  dk = -u_e^T K0 u_e;  dr = H^T (p clip(rho_f, void, 1)^(p-1) dk)
  OC: bisection of lambda in [1e-9, 1e9] until (l2-l1)/(l2+l1) <= 1e-4 on
      rho_new = max(0, max(xL, min(1, min(xU, ocP/lambda)))),
      ocP = max(1e-12, rho sqrt(max(-dr/A, 0))), volume test sum(rho_new A)/V <= vf,
      returning the rho of the last lambda tried (TopOpt/_solver.py:271-311).
"""
import numpy as np

from . import ops
from .elements import element_measure, hex8_stiffness, q4_stiffness
from .grid import Grid
from .mg import MultiGridOracle


def oc_update(rho, dr, A, vol, vf, move):
    rho = rho.reshape(-1)
    xU = np.clip(rho + move, 0.0, 1.0)
    xL = np.clip(rho - move, 0.0, 1.0)
    ocP = rho * np.nan_to_num(np.sqrt(np.maximum(-dr.reshape(-1) / A, 0)), nan=0)
    if np.abs(ocP).sum() == 0:
        ocP = np.ones_like(ocP) * 1e-3
    ocP = np.maximum(1e-12, ocP)
    l1, l2 = 1e-9, 1e9
    lmid = 0.5 * (l1 + l2)
    rho_new = np.maximum(0, np.maximum(xL, np.minimum(1.0, np.minimum(xU, ocP / lmid))))
    steps = 0
    while (l2 - l1) / (l2 + l1) > 1e-4:
        lmid = 0.5 * (l1 + l2)
        rho_new = np.maximum(0, np.maximum(xL, np.minimum(1.0, np.minimum(xU, ocP / lmid))))
        V = (rho_new * A).sum()
        if V / vol <= vf:
            l2 = lmid
        else:
            l1 = lmid
        steps += 1
    return rho_new, lmid, steps


class SIMPOracle:
    """One structured SIMP problem on the CPU, mirroring the reference call order."""

    def __init__(self, nel, h=None, E0=1.0, nu=0.3, void=1e-9, penalty=3.0, vf=0.5, rmin=1.5,
                 move=0.2, mg_kwargs=None, K0=None):
        self.grid = Grid(nel, h)
        g = self.grid
        if K0 is None:
            K0 = q4_stiffness(*g.h, E=E0, nu=nu) if g.dim == 2 else hex8_stiffness(*g.h, E=E0, nu=nu)
        self.K0 = K0
        self.A = element_measure(g.h)
        self.vol = self.A * g.n_el
        self.void, self.penalty, self.vf, self.move = void, penalty, vf, move
        self.H, self.N = ops.filter_matrix(g, rmin)
        self.solver = MultiGridOracle(g, **(mg_kwargs or {}))
        self.f = np.zeros(g.n_dof)
        self.cons = np.zeros(0, dtype=np.int64)

    def add_bc_nodal(self, node_ids, mask):
        node_ids = np.asarray(node_ids)
        mask = np.asarray(mask, dtype=bool)
        if mask.shape[0] == 1:
            mask = np.repeat(mask, node_ids.shape[0], axis=0)
        new = [node_ids[mask[:, d]] * self.grid.dof + d for d in range(self.grid.dof)]
        self.cons = np.unique(np.concatenate([self.cons] + new))

    def add_force_nodal(self, node_ids, F):
        node_ids = np.asarray(node_ids)
        F = np.asarray(F, dtype=np.float64)
        for d in range(self.grid.dof):
            self.f[node_ids * self.grid.dof + d] = F[0, d] if F.shape[0] == 1 else F[:, d]

    def material(self, rho_f):
        return np.clip(rho_f ** self.penalty, self.void, 1.0)

    def material_grad(self, rho_f):
        return self.penalty * np.clip(rho_f, self.void, 1.0) ** (self.penalty - 1)

    def solve_and_process(self, rho):
        rho_f = ops.filter_apply(self.H, rho)
        E = self.material(rho_f)
        K = ops.assemble(self.grid, self.K0, E, self.cons)
        U, res = self.solver.solve(K, self.f, use_last=True)
        comp = float(self.f @ U)
        dk = ops.dk(self.grid, self.K0, U)
        dr = self.material_grad(rho_f) * dk
        dr = ops.filter_apply_T(self.H, dr)
        return comp, dr, res, U

    def optimize(self, rho0, n_iter):
        rho = np.full(self.grid.n_el, float(rho0)) if np.isscalar(rho0) else np.array(rho0, dtype=float)
        comp, dr, res, U = self.solve_and_process(rho)
        hist = {"comp": [], "change": [], "residual": [], "rho": [], "lambda": [], "oc_steps": [],
                "comp0": comp}
        for _ in range(n_iter):
            rho_old = rho.copy()
            comp_old = comp
            rho, lam, steps = oc_update(rho, dr, self.A, self.vol, self.vf, self.move)
            comp, dr, res, U = self.solve_and_process(rho)
            hist["comp"].append(comp)
            hist["change"].append(float(np.sqrt(np.square(rho - rho_old).mean())))
            hist["residual"].append(res)
            hist["rho"].append(rho.copy())
            hist["lambda"].append(lam)
            hist["oc_steps"].append(steps)
            del comp_old
        self.U = U
        return rho, hist


def oc_update_sets(rho, dr, A, vol, law, move):
    """OC of TopOpt/_solver.py:271-311 on an (n_el, n_sets) design, one bisection
    multiplier per column, each stopping at (l2 - l1) / (l2 + l1) <= 1e-4; ocP and the
    constraint test from the multi-material law (MaterialModels.py:207-228)."""
    n = rho.shape[1]
    A = np.asarray(A, dtype=np.float64).reshape(-1)
    xU = np.clip(rho + move, 0.0, 1.0)
    xL = np.clip(rho - move, 0.0, 1.0)
    ocP = np.maximum(1e-12, law.ocp(dr, A, rho))
    l1 = 1e-9 * np.ones(n)
    l2 = 1e9 * np.ones(n)
    lmid = 0.5 * (l1 + l2)
    rho_new = np.maximum(0, np.maximum(xL, np.minimum(1.0, np.minimum(xU, ocP / lmid))))
    while np.any((l2 - l1) / (l2 + l1) > 1e-4):
        lmid = 0.5 * (l1 + l2)
        rho_new = np.maximum(0, np.maximum(xL, np.minimum(1.0, np.minimum(xU, ocP / lmid))))
        valid = law.con(rho_new, A, vol)
        l2[valid] = lmid[valid]
        l1[~valid] = lmid[~valid]
    return rho_new


class MultiMaterialSIMPOracle(SIMPOracle):
    """SIMP with a multi-material law (oracle.material.MultiMaterialLaw) on an (n_el, n_sets)
    design: every column filtered, E from the law, one exact sparse solve, dr = dE/drho_f dk
    per column filtered back, OC per column (oc_update_sets)."""

    def __init__(self, nel, law, **kw):
        super().__init__(nel, void=law.void, penalty=law.penalty, **kw)
        self.law = law

    def solve_and_process(self, rho):
        import scipy.sparse.linalg as spla
        n = self.law.n
        rho_f = np.stack([ops.filter_apply(self.H, rho[:, m]) for m in range(n)], axis=1)
        E = self.law.forward(rho_f)
        K = ops.assemble(self.grid, self.K0, E, self.cons)
        U = spla.spsolve(K.tocsc(), self.f)
        comp = float(self.f @ U)
        dk = ops.dk(self.grid, self.K0, U)
        dr = self.law.backward(rho_f) * dk.reshape(-1, 1)
        dr = np.stack([ops.filter_apply_T(self.H, dr[:, m]) for m in range(n)], axis=1)
        return comp, dr, 0.0, U

    def optimize(self, rho0, n_iter):
        rho = np.array(rho0, dtype=float).reshape(self.grid.n_el, self.law.n)
        comp, dr, _, U = self.solve_and_process(rho)
        hist = {"comp": [], "rho": [], "comp0": comp}
        for _ in range(n_iter):
            rho = oc_update_sets(rho, dr, np.array([self.A]), self.vol, self.law, self.move)
            comp, dr, _, U = self.solve_and_process(rho)
            hist["comp"].append(comp)
            hist["rho"].append(rho.copy())
        self.U = U
        return rho, hist


def mbb_problem(nelx=120, nely=40, law=None, **kw):
    """2-D MBB half-beam: left edge u_x = 0, bottom-right node u_y = 0, F = (0,-1) at top-left
    (with a multi-material law: MultiMaterialSIMPOracle)."""
    p = SIMPOracle((nelx, nely), **kw) if law is None else MultiMaterialSIMPOracle((nelx, nely), law, **kw)
    g = p.grid
    left = np.array([g.node_id(0, j) for j in range(nely + 1)])
    p.add_bc_nodal(left, [[True, False]])
    p.add_bc_nodal(np.array([g.node_id(nelx, 0)]), [[False, True]])
    p.add_force_nodal(np.array([g.node_id(0, nely)]), [[0.0, -1.0]])
    return p


def cantilever_problem(nelx, nely, nelz, **kw):
    """3-D cantilever: x=0 face clamped, total load (0,-1,0) spread over the nodes at x=L, y=0."""
    p = SIMPOracle((nelx, nely, nelz), **kw)
    g = p.grid
    face = np.array([g.node_id(0, j, k) for j in range(nely + 1) for k in range(nelz + 1)])
    p.add_bc_nodal(face, [[True, True, True]])
    edge = np.array([g.node_id(nelx, 0, k) for k in range(nelz + 1)])
    p.add_force_nodal(edge, [[0.0, -1.0 / edge.shape[0], 0.0]])
    return p
