"""SIMP minimum-compliance optimiser, drop-in for CuTopOpt (TopOpt/_cuda.py:17-382).

Same constructor, BC/load API, ``optimize`` loop, history and termination test.  When
the objects handed in are this package's (CuStructuredStiffnessKernel, CuMultiGrid,
CuStructuredFilter2D/3D, SingleMaterial) one SIMP analysis runs as a single library call
(edge_simp_solve_and_process: filter + SIMP law + GMG-PCG + compliance + sensitivity +
filter transpose) and the OC bisection runs on the GPU (edge_oc_update); ``iterate`` (used by
``optimize``) runs a whole SIMP iteration, OC update and analysis, as one CUDA graph launch
(edge_simp_iteration).  Other duck-typed objects go through the reference's object-by-object
call order.

Differences from the reference, on purpose: ``rho_init`` works (the reference raises
UnboundLocalError, TopOpt/_cuda.py:322), and arrays are torch CUDA tensors instead of cupy.
"""
import ctypes
import logging

import numpy as np
import torch
from scipy.spatial import KDTree
from tqdm.auto import trange

from . import _lib
from .filters import _CuStructuredFilter
from .kernels import CuStructuredStiffnessKernel, _as_dev_f64
from .material import PenalizedMultiMaterial, SingleMaterial
from .solvers import CuMultiGrid

logger = logging.getLogger(__name__)


def _to_np(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


class CuTopOpt:
    def __init__(self, mesh, material_model, kernel, solver, filter_kernel=None, max_iter=500, move=0.2, ch_tol=1e-4,
                 fun_tol=1e-6, reuse_sol=True, solve_min_tol=np.inf, min_tol_patience=10, abandon_patience=10,
                 verbose=True):
        self.mesh = mesh
        self.material_model = material_model
        self.kernel = kernel
        self.solver = solver
        self.filter_kernel = filter_kernel
        self.max_iter = max_iter
        self.move = move
        self.ch_tol = ch_tol
        self.fun_tol = fun_tol
        self.solve_min_tol = solve_min_tol
        self.min_tol_patience = min_tol_patience
        self.abandon_patience = abandon_patience
        self.reuse_sol = reuse_sol
        self.verbose = verbose
        self.dtype = mesh.dtype
        if verbose:
            logger.setLevel(logging.INFO)
        self.f = torch.zeros(kernel.shape[0], dtype=torch.float64, device="cuda")
        self.KDTree = None
        self._U = None
        self.last_stats = {}

    # ----------------------------------------------------------------- fast-path detection
    @property
    def fused(self):
        return (isinstance(self.kernel, CuStructuredStiffnessKernel) and isinstance(self.solver, CuMultiGrid)
                and isinstance(self.filter_kernel, _CuStructuredFilter) and isinstance(self.material_model, SingleMaterial)
                and self.solver.kernel is self.kernel and not self.solver.padded)

    # ----------------------------------------------------------------- BCs and loads (TopOpt/_cuda.py:131-240)
    def reset_BC(self):
        self.kernel.set_constraints([])
        self.kernel.has_cons = False

    def reset_F(self):
        self.f[:] = 0

    def _tree(self):
        if self.KDTree is None:
            self.KDTree = KDTree(_to_np(self.mesh.nodes))
        return self.KDTree

    def add_BCs(self, positions, BCs):
        _, idx = self._tree().query(_to_np(positions))
        self.add_BC_nodal(np.asarray(idx), BCs)

    def add_Forces(self, positions, Fs):
        _, idx = self._tree().query(_to_np(positions))
        self.add_F_nodal(np.asarray(idx), Fs)

    def add_BC_nodal(self, node_ids, BCs):
        node_ids = _to_np(node_ids).astype(np.int64)
        BCs = _to_np(BCs).astype(bool)
        if BCs.shape[0] != node_ids.shape[0] and BCs.shape[0] > 1:
            raise ValueError("BCs shape does not match positions shape and is not broadcastable.")
        dof = self.mesh.dof
        cons = []
        for i in range(dof):
            if BCs.shape[0] == 1:
                if BCs[0, i]:
                    cons.append(node_ids * dof + i)
            else:
                cons.append(node_ids[BCs[:, i]] * dof + i)
        if cons:
            self.kernel.add_constraints(np.concatenate(cons))

    def add_F_nodal(self, node_ids, Fs):
        node_ids = _to_np(node_ids).astype(np.int64)
        Fs = _to_np(Fs).astype(np.float64)
        if Fs.shape[0] != node_ids.shape[0] and Fs.shape[0] > 1:
            raise ValueError("Fs shape does not match positions shape and is not broadcastable.")
        dof = self.mesh.dof
        f = self.f.cpu().numpy()
        ids = node_ids.reshape(-1) if Fs.shape[0] == 1 else node_ids.reshape(node_ids.shape[0], -1)[:, 0]
        for i in range(dof):
            f[ids * dof + i] = Fs[0, i] if Fs.shape[0] == 1 else Fs[:, i]
        self.f.copy_(torch.from_numpy(f))

    # ----------------------------------------------------------------- OC (TopOpt/_cuda.py:242-280)
    @property
    def n_sets(self):
        """Design columns per element (1, or the number of materials of a multi-material law)."""
        return int(self.material_model.base_properties()["n_sets"])

    def update_design(self, rho, df):
        if self.n_sets > 1:
            return self._update_design_generic(_as_dev_f64(rho), _as_dev_f64(df))
        rho = _as_dev_f64(rho).reshape(-1)
        df = _as_dev_f64(df).reshape(-1)
        if isinstance(self.material_model, SingleMaterial) and isinstance(self.kernel, CuStructuredStiffnessKernel):
            out = torch.empty_like(rho)
            lam, steps, sq = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
            A = float(np.asarray(self.mesh.As).reshape(-1)[0])
            self.kernel._bind_stream()
            _lib.call("edge_oc_update", self.kernel.handle, _lib.ptr(rho), _lib.ptr(df), A, float(self.mesh.volume),
                      float(self.material_model.volume_fraction), float(self.move), _lib.ptr(out), ctypes.byref(lam),
                      ctypes.byref(steps), ctypes.byref(sq))
            self.last_stats.update(oc_lambda=lam.value, oc_steps=steps.value, oc_sqchange=sq.value)
            return out
        return self._update_design_generic(rho, df)

    def _update_design_generic(self, rho, df):
        """OC with one bisection multiplier per design column (TopOpt/_cuda.py:242-280): all
        columns are bisected together until every column satisfies (l2 - l1) / (l2 + l1) <= 1e-4
        (the reference's np.any test, TopOpt/_cuda.py:270), so a column that has converged keeps
        bisecting while another has not; on the material model's ocP and constraint test.
        Multi-material designs are (n_el, n_sets)."""
        size = self.n_sets
        rho = rho.reshape(-1, size)
        df = df.reshape(-1, size)
        As = torch.as_tensor(np.asarray(self.mesh.As), dtype=torch.float64, device="cuda")
        ocP = self.material_model.ocP(df, As, rho)
        ocP = torch.clamp(ocP, min=1e-12)
        mm = self.material_model
        if isinstance(mm, PenalizedMultiMaterial) and 1 <= size <= 8:
            # the bisection as one launch (edge_oc_update_multi): no host read per step
            rho_c = rho.contiguous()
            ocp_c = ocP.reshape(-1, size).contiguous()
            A = As.reshape(-1).contiguous()
            out = torch.empty_like(rho_c)
            if mm.rho_mat is None:
                mass = _lib.double_array(np.asarray(mm.mass, dtype=np.float64).reshape(-1)[:size].tolist())
                rm = None
            else:
                mass = _lib.double_array([float(mm.mass)])
                rm = _lib.double_array(np.asarray(mm.rho_mat, dtype=np.float64).reshape(-1).tolist())
            _lib.call("edge_oc_update_multi", rho_c.shape[0], size, _lib.ptr(rho_c), _lib.ptr(ocp_c), _lib.ptr(A),
                      1 if A.numel() == rho_c.shape[0] else 0, float(self.move), float(self.mesh.volume), mass, rm,
                      _lib.ptr(out), _lib.stream_ptr())
            return out.reshape(-1) if size == 1 else out
        return self._bisect_torch(rho, ocP, As)

    def _bisect_torch(self, rho, ocP, As):
        """The bisection of _update_design_generic in torch operations, for material models other
        than PenalizedMultiMaterial (their constraint test is theirs to define); one host read
        per step, as the reference's loop."""
        size = self.n_sets
        xU = torch.clamp(rho + self.move, 0.0, 1.0)
        xL = torch.clamp(rho - self.move, 0.0, 1.0)
        l1 = 1e-9 * torch.ones(size, dtype=torch.float64, device="cuda")
        l2 = 1e9 * torch.ones(size, dtype=torch.float64, device="cuda")
        lmid = 0.5 * (l1 + l2)
        rho_new = torch.clamp(torch.maximum(xL, torch.minimum(torch.ones_like(xU), torch.minimum(xU, ocP / lmid))), min=0)
        while bool(torch.any((l2 - l1) / (l2 + l1) > 1e-4)):
            lmid = 0.5 * (l1 + l2)
            rho_new = torch.clamp(torch.maximum(xL, torch.minimum(torch.ones_like(xU), torch.minimum(xU, ocP / lmid))),
                                  min=0)
            valids = self.material_model.evaluate_constraint(rho_new, As, float(self.mesh.volume))
            l2 = torch.where(valids, lmid, l2)
            l1 = torch.where(~valids, lmid, l1)
        return rho_new.reshape(-1) if size == 1 else rho_new

    # ----------------------------------------------------------------- analysis (TopOpt/_cuda.py:282-302)
    def FEA_integrals(self, rho):
        """Strain, stress, strain energy and von Mises stress per element for the design rho
        (TopOpt/_cuda.py:78-129): E = the material's 'plain' value (rho clipped to [void, 1]),
        one solve of K(E) u = f warm-started from the last solution, then the element
        integrals on the device (edge_fea_integrals).  Returns torch tensors on the device."""
        rho_ = self.material_model(_as_dev_f64(rho).reshape(-1), 1e6, plain=True)
        self.kernel.set_rho(rho_)
        U, residual = self.solver.solve(self.f, use_last=True)
        if residual > 1e-5:
            logger.warning(f"Solver residual is above 1e-5 ({residual:.4e}). Consider higher iterations (rerun "
                           f"this function and more iteration from prior solve will be applied).")
        strain, stress, strain_energy = self.kernel.fea_integrals(rho_, U, self.mesh.B_single, self.mesh.D_single)
        s = stress
        if self.mesh.nodes.shape[1] == 2:
            von_mises = torch.sqrt(s[:, 0] ** 2 + s[:, 1] ** 2 - s[:, 0] * s[:, 1] + 3 * s[:, 2] ** 2)
        else:
            von_mises = torch.sqrt(0.5 * ((s[:, 0] - s[:, 1]) ** 2 + (s[:, 1] - s[:, 2]) ** 2 + (s[:, 2] - s[:, 0]) ** 2
                                          + 6 * (s[:, 3] ** 2 + s[:, 4] ** 2 + s[:, 5] ** 2)))
        return strain, stress, strain_energy, von_mises

    def solve_and_process(self, rho, iteration):
        if self.n_sets > 1:
            return self._solve_and_process_sets(_as_dev_f64(rho), iteration)
        rho = _as_dev_f64(rho).reshape(-1)
        if self.fused:
            return self._solve_and_process_fused(rho, iteration)
        rho_ = self.filter_kernel.dot(rho)
        rho__ = self.material_model(rho_, iteration)
        self.kernel.set_rho(rho__)
        U, residual = self.solver.solve(self.f, use_last=self.reuse_sol)
        compliance = torch.dot(self.f, U)
        df = self.kernel.process_grad(U)
        dr = self.material_model.grad(rho_, iteration) * df
        dr = dr.reshape(dr.shape[0], -1)
        for i in range(dr.shape[1]):
            dr[:, i] = self.filter_kernel._rmatvec(dr[:, i].contiguous())
        return compliance, dr, residual

    def _solve_and_process_sets(self, rho, iteration):
        """solve_and_process for an (n_el, n_sets) design (the reference's call order,
        TopOpt/_cuda.py:282-302): each column filtered, the material law maps the filtered
        columns to one E per element, one solve, dr = dE/drho_f * dk per column, each column
        filtered back with the transpose."""
        n = self.n_sets
        rho = rho.reshape(-1, n)
        rho_ = torch.stack([self.filter_kernel.dot(rho[:, m].contiguous()) for m in range(n)], dim=1)
        E = self.material_model(rho_, iteration)
        self.kernel.set_rho(_as_dev_f64(E).reshape(-1))
        U, residual = self.solver.solve(self.f, use_last=self.reuse_sol)
        compliance = torch.dot(self.f, U)
        df = self.kernel.process_grad(U).reshape(-1, 1)
        dr = _as_dev_f64(self.material_model.grad(rho_, iteration)).reshape(-1, n) * df
        for m in range(n):
            dr[:, m] = self.filter_kernel._rmatvec(dr[:, m].contiguous())
        self._U = U
        return compliance, dr, residual

    def _solve_and_process_fused(self, rho, iteration):
        sv = self.solver
        sv._configure()
        tune_sweeps_now = sv.tune_sweeps and sv.sweeps is None and self.reuse_sol and sv.last_x0 is not None
        if (sv.autotune and sv.tuned is None) or tune_sweeps_now:
            # the autotuners need a density on the kernel: use this iteration's SIMP field
            rho_f = self.filter_kernel.dot(rho)
            self.kernel.set_rho(self.material_model(rho_f, iteration))
            sv.tune()
            if tune_sweeps_now:  # warm-started from the previous solution, like the solves after it
                sv.tune_sweep_counts(self.f, sv.last_x0)
        pen = float(self.material_model.current_penalty(iteration))
        use_last = self.reuse_sol and sv.last_x0 is not None
        if sv.last_x0 is None or not use_last:
            sv.last_x0 = torch.zeros_like(self.f)
        U = sv.last_x0
        dr = torch.empty(self.kernel.n_elements, dtype=torch.float64, device="cuda")
        rho_f = torch.empty_like(dr)
        c, res, its = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self.kernel._bind_stream()
        keep = sv.keep_start(U) if use_last else None
        for attempt in range(2):
            _lib.call("edge_simp_solve_and_process", self.kernel.handle, self.filter_kernel.handle, _lib.ptr(rho),
                      pen, float(self.material_model.void), _lib.ptr(self.f), _lib.ptr(U), 1 if use_last else 0,
                      float(sv.tol), int(sv.maxiter), ctypes.byref(c), _lib.ptr(dr), _lib.ptr(rho_f),
                      ctypes.byref(res), ctypes.byref(its))
            # the fixed smoother weight did not converge: once more with the reference's schedule
            if attempt or res.value < sv.tol or not sv.use_omega_schedule():
                break
            if keep is not None:
                U.copy_(keep)
        self.kernel.has_rho = True
        sv.last_iters = its.value
        self._U = U
        self.last_stats.update(sv.stats())
        self.last_stats.update(pcg_iters=its.value, residual=res.value)
        return torch.tensor(c.value, dtype=torch.float64), dr.reshape(-1, 1), res.value

    def iterate(self, rho, df, iteration):
        """One SIMP iteration: ``update_design(rho, df)`` followed by
        ``solve_and_process(rho_new, iteration)``, returning (rho_new, compliance, dr, residual).
        With this package's objects (and once the solver's autotuners have run, on the first
        analyses) the two run as one CUDA graph launch with one host read
        (edge_simp_iteration: the OC bisection loop is a device-side conditional node);
        otherwise as the two calls."""
        sv = self.solver
        ready = (self.fused and self.n_sets == 1 and self.reuse_sol and sv.graph and sv.last_x0 is not None
                 and (not sv.autotune or sv.tuned is not None) and (not sv.tune_sweeps or sv.sweeps is not None))
        if not ready:
            rho_new = self.update_design(rho, df)
            comp, dr, res = self.solve_and_process(rho_new, iteration)
            return rho_new, comp, dr, res
        sv._configure()
        rho = _as_dev_f64(rho).reshape(-1)
        df = _as_dev_f64(df).reshape(-1)
        rho_new = torch.empty_like(rho)
        dr = torch.empty_like(rho)
        rho_f = torch.empty_like(rho)
        U = sv.last_x0
        c, res, its = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        lam, steps, sq = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
        A = float(np.asarray(self.mesh.As).reshape(-1)[0])
        pen = float(self.material_model.current_penalty(iteration))
        self.kernel._bind_stream()
        keep = sv.keep_start(U)
        for attempt in range(2):
            _lib.call("edge_simp_iteration", self.kernel.handle, self.filter_kernel.handle, _lib.ptr(rho),
                      _lib.ptr(df), A, float(self.mesh.volume), float(self.material_model.volume_fraction),
                      float(self.move), pen, float(self.material_model.void), _lib.ptr(self.f), _lib.ptr(U), 1,
                      float(sv.tol), int(sv.maxiter), _lib.ptr(rho_new), _lib.ptr(dr), _lib.ptr(rho_f),
                      ctypes.byref(c), ctypes.byref(res), ctypes.byref(its), ctypes.byref(lam), ctypes.byref(steps),
                      ctypes.byref(sq))
            # the fixed smoother weight did not converge: once more with the reference's schedule
            if attempt or res.value < sv.tol or not sv.use_omega_schedule():
                break
            if keep is not None:
                U.copy_(keep)
        self.kernel.has_rho = True
        sv.last_iters = its.value
        self._U = U
        self.last_stats.update(sv.stats())
        self.last_stats.update(pcg_iters=its.value, residual=res.value, oc_lambda=lam.value, oc_steps=steps.value,
                               oc_sqchange=sq.value, graph_iteration=True)
        return rho_new, torch.tensor(c.value, dtype=torch.float64), dr.reshape(-1, 1), res.value

    # ----------------------------------------------------------------- loop (TopOpt/_cuda.py:304-382)
    def optimize(self, save_comp_history=False, save_change_history=False, save_rho_history=False, rho_init=None,
                 callback=None):
        flag = False
        n = self.n_sets
        if rho_init is None:
            rho = self.material_model.init_desvars(self.kernel.n_elements)
        elif n > 1:  # a multi-material start design is taken as given, clipped to [0, 1]
            rho = torch.clamp(_as_dev_f64(rho_init), 0.0, 1.0)
        else:
            rho = self.material_model(_as_dev_f64(rho_init).reshape(-1), 0, plain=True)
        rho = _as_dev_f64(rho).reshape(-1) if n == 1 else _as_dev_f64(rho).reshape(-1, n)
        comp, df, res = self.solve_and_process(rho, 0)
        prog = trange(self.max_iter, disable=logger.getEffectiveLevel() > logging.INFO)
        comp_history, change_history, rho_history = [], [], []
        for i in prog:
            rho_old = rho.clone()
            comp_old = float(comp)
            rho, comp, df, res = self.iterate(rho, df, i)
            change = float(torch.sqrt(torch.square(rho - rho_old).mean()))
            compf = float(comp)
            change_f = abs(compf - comp_old) / compf
            if save_change_history:
                change_history.append(change)
            if save_rho_history:
                rho_history.append(rho.cpu().numpy())
            if save_comp_history:
                comp_history.append(compf)
            if callback is not None:
                callback(i, rho, compf, change, res)
            prog.set_postfix_str(
                f"Compliance: {compf:.4e}, Change: {change:.4e}, Function Change: {change_f:.4e}, Residual: {res:.4e}")
            if change < self.ch_tol and change_f < self.fun_tol and self.material_model.is_terminal(i):
                flag = True
                break
        hist = {}
        if save_comp_history:
            hist["comp_history"] = comp_history
        if save_change_history:
            hist["change_history"] = change_history
        if save_rho_history:
            hist["rho_history"] = rho_history
        return rho, flag, hist


TopOpt = CuTopOpt
