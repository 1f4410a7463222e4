"""Geometric-multigrid-preconditioned CG, drop-in for CuMultiGrid
(solvers/_multigrid_cuda.py:15-242) on the structured stiffness kernel of this package.

Same constructor keywords and the same algorithm: Galerkin hierarchy rebuilt on every
solve, damped-Jacobi V-cycle with omega*1.06^level, exact coarsest solve, PCG with warm
start from the last solution and the residual-driven omega schedule; omega is reset to
min_omega at the start of each solve as the GPU reference does.  The coarsest level is
factorised by a dense FP64 Cholesky on the GPU (exact, like the reference's splu), so
coarse_solver only selects between equivalent exact solves.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .kernels import CuStructuredStiffnessKernel, _CuGeneralKernel, _as_dev_f64


class Solver:
    def __call__(self, *args, **kwargs):
        return self.solve(*args, **kwargs)

    def solve(self, *args, **kwargs):
        pass

    def reset(self):
        pass


class _PaddedGrid:
    """Embedding of a structured problem whose element counts are not all divisible by
    2**n_level into the next grid that is: the real grid keeps its numbering in the lower
    corner, padding elements have zero stiffness and every node that touches only padding
    elements is constrained (identity rows, zero load).  The padded system restricted to the
    real DOFs is the original one, and its solution is zero on the padding, so a solve on the
    padded grid answers the original problem while the multigrid coarsens cleanly.  (The
    reference's multigrid has no such handling: on odd extents its prolongation is not the
    restriction's transpose and PCG stalls.)"""

    def __init__(self, kernel, n_level):
        from .mesh import CuStructuredMesh2D, CuStructuredMesh3D
        mesh = kernel.mesh
        m = 2 ** n_level
        nel = [int(v) for v in mesh.nel]
        pad = [(v + m - 1) // m * m for v in nel]
        h = [float(L) / n for L, n in zip(mesh.dim, nel)]
        elem = (mesh.K_single, mesh.D_single, mesh.B_single, float(mesh.A_single[0]))
        stiff = lambda x0: elem  # noqa: E731  (the real mesh's element, so K0 is identical)
        if len(nel) == 2:
            pm = CuStructuredMesh2D(pad[0], pad[1], pad[0] * h[0], pad[1] * h[1], stiffness=stiff)
        else:
            pm = CuStructuredMesh3D(pad[0], pad[1], pad[2], pad[0] * h[0], pad[1] * h[1], pad[2] * h[2],
                                    stiffness=stiff)
        self.nel, self.pad = nel, pad
        self.kernel = CuStructuredStiffnessKernel(pm)
        dof = kernel.dof
        if len(nel) == 2:
            i, j = np.meshgrid(np.arange(nel[0]), np.arange(nel[1]), indexing="ij")
            el = (i * pad[1] + j).ravel()                                    # e = i*nely + j
            jn, in_ = np.meshgrid(np.arange(nel[1] + 1), np.arange(nel[0] + 1), indexing="ij")
            nodes = (jn * (pad[0] + 1) + in_).ravel()                        # n = j*(nelx+1) + i
            pj, pi = np.meshgrid(np.arange(pad[1] + 1), np.arange(pad[0] + 1), indexing="ij")
            outside = ((pi > nel[0]) | (pj > nel[1])).ravel()
        else:
            i, j, k = np.meshgrid(np.arange(nel[0]), np.arange(nel[1]), np.arange(nel[2]), indexing="ij")
            el = (i * pad[1] * pad[2] + j * pad[2] + k).ravel()             # e = i*ny*nz + j*nz + k
            jn, in_, kn = np.meshgrid(np.arange(nel[1] + 1), np.arange(nel[0] + 1), np.arange(nel[2] + 1),
                                      indexing="ij")
            nodes = (jn * (pad[0] + 1) * (pad[2] + 1) + in_ * (pad[2] + 1) + kn).ravel()  # n = j*nx*nz + i*nz + k
            pj, pi, pk = np.meshgrid(np.arange(pad[1] + 1), np.arange(pad[0] + 1), np.arange(pad[2] + 1),
                                     indexing="ij")
            outside = ((pi > nel[0]) | (pj > nel[1]) | (pk > nel[2])).ravel()
        self.el_map = torch.as_tensor(el, device="cuda")
        self.dof_map = torch.as_tensor((nodes[:, None] * dof + np.arange(dof)[None, :]).ravel(), device="cuda")
        self.pad_dofs = torch.as_tensor(
            (np.nonzero(outside)[0][:, None] * dof + np.arange(dof)[None, :]).ravel(), device="cuda")
        self._cons_key = None
        self._springs_key = None

    def sync(self, kernel):
        """Copy the real kernel's density, constraints and springs onto the padded kernel."""
        self.set_rho(kernel)
        self.sync_bcs(kernel)

    def set_rho(self, kernel):
        """The real kernel's density onto the padded grid (padding elements zero), on the device
        (edge_set_rho_embedded)."""
        kp = self.kernel
        rho = _as_dev_f64(kernel.rho).reshape(-1).contiguous()
        kp._bind_stream()
        _lib.call("edge_set_rho_embedded", kp.handle, _lib.ptr(rho), _lib.int_array(self.nel))
        kp.rho = None  # the padded grid's E lives in the library only
        kp.has_rho = True

    def sync_bcs(self, kernel):
        """The real kernel's constraints (every padding-only node constrained as well) and springs
        onto the padded kernel, when they changed."""
        kp = self.kernel
        key = (kernel.constraints.data_ptr(), int(kernel.constraints.sum().item()), kernel.has_con)
        if key != self._cons_key:
            c = torch.zeros(kp.shape[0], dtype=torch.bool, device="cuda")
            c[self.dof_map] = kernel.constraints
            c[self.pad_dofs] = True
            kp.set_constraints(torch.nonzero(c).reshape(-1))
            self._cons_key = key
        springs = getattr(kernel, "springs", None)
        skey = None if springs is None else (tuple(springs[0].tolist()), tuple(springs[1].tolist()))
        if skey != self._springs_key:
            if springs is None:
                kp.set_springs([], [])
            else:
                kp.set_springs(self.dof_map[torch.as_tensor(springs[0], device="cuda")].cpu().numpy(), springs[1])
            self._springs_key = skey

    def embed(self, v):
        out = torch.zeros(self.kernel.shape[0], dtype=torch.float64, device="cuda")
        out[self.dof_map] = _as_dev_f64(v).reshape(-1)
        return out

    def extract(self, v):
        return v[self.dof_map]


def pick_sweep_pattern(runs, retime, margin, fallback=None):
    """Choice of the sweep autotuner among converged runs [ms, pattern, pcg_iters].

    The fastest pattern and the cheapest one (fewest sweeps) are timed again with
    ``retime(pattern) -> (ms, converged, iters)`` and decided on the sum of both timings.  A
    pattern with more sweeps must beat the cheapest by ``margin`` (best < margin * cheapest):
    the iterations that extra sweeps save shrink as the SIMP design sharpens (at 12.8M DOF:
    17 % fewer PCG iterations in the first timed SIMP step, 5 % in the fifth), so near-ties on
    the early tuning solve go to fewer sweeps.  When no contender converges again on its
    retime, returns ``(0.0, fallback, 0)`` (the reference's sweeps), as when nothing converged
    at all.  Returns (ms summed, pattern, iters)."""
    runs = sorted(([float(r[0]), list(r[1]), r[2]] for r in runs), key=lambda r: r[0])
    cheap = min(runs, key=lambda r: (sum(r[1]), r[1]))
    contenders = [runs[0]] if runs[0] is cheap else [runs[0], cheap]
    for r in contenders:
        ms, ok, _ = retime(r[1])
        r[0] = r[0] + ms if ok else float("inf")
    best = contenders[0]
    if len(contenders) == 2 and not best[0] < margin * cheap[0]:
        best = cheap
    if best[0] == float("inf") and fallback is not None:
        return (0.0, list(fallback), 0)
    return tuple(best)


class CuMultiGrid(Solver):
    OMEGA_CARRY = False

    def __init__(self, mesh, kernel, maxiter=1000, tol=1e-5, n_smooth=3, omega=0.5, n_level=3, cycle="W",
                 w_level=1, coarse_solver="splu", matrix_free=False, low_level_tol=1e-8, low_level_maxiter=5000,
                 min_omega=0.4, omega_boost=1.06, precision="fp64", autotune=True, graph=True, tune_sweeps=None,
                 omega_carry=None, mixed_omega="auto"):
        if not isinstance(kernel, CuStructuredStiffnessKernel):
            raise TypeError("CuMultiGrid needs the package's CuStructuredStiffnessKernel")
        # smoother weight across solves: reset to min_omega every solve (the GPU solver,
        # solvers/_multigrid_cuda.py:210) or carried over from the last solve (the CPU solver,
        # solvers/_multigrid.py:178-225; the MultiGrid class below)
        self.omega_carry = self.OMEGA_CARRY if omega_carry is None else bool(omega_carry)
        # the mixed-precision preconditioner's smoother weight.  The reference's schedule moves
        # between min_omega and (min_omega + omega) / 2 with the residual
        # (solvers/_multigrid_cuda.py:227); "max" holds it fixed at omega, the schedule's upper
        # bound, and a number holds it there; None keeps the schedule; "auto" (the default)
        # starts on the schedule and lets the sweep autotuner time the weight fixed at omega
        # against it on its tuning solve, keeping the faster.  A solve that does not converge
        # with a fixed weight runs again from the same start on the schedule, which is kept from
        # then on.  Coarser levels scale the weight by omega_boost**level either way, and the
        # FP64 path always keeps the schedule.
        if not (mixed_omega is None or mixed_omega in ("auto", "max")
                or (isinstance(mixed_omega, (int, float)) and mixed_omega > 0)):
            raise ValueError("mixed_omega must be None, 'auto', 'max' or a positive number")
        self.mixed_omega = mixed_omega
        self._omega_mode = "fixed" if mixed_omega not in (None, "auto") else "schedule"
        self._omega_failed = False
        self._x_keep = None
        self.kernel = kernel
        self.mesh = mesh
        self.last_x0 = None
        self.tol = tol
        self.maxiter = maxiter
        self.n_smooth = n_smooth
        self.omega = omega
        self.max_omega = omega
        self.min_omega = max(omega / 2, min_omega)
        self.d_omega = self.max_omega - self.min_omega
        self.omega_boost = omega_boost
        self.n_level = n_level
        self.cycle = cycle
        self.w_level = [w_level] if isinstance(w_level, int) else list(w_level)
        self.matrix_free = matrix_free
        self.dof = mesh.dof
        self.coarse_solver = coarse_solver
        self.low_level_tol = low_level_tol
        self.low_level_maxiter = low_level_maxiter
        self.precision = precision
        if coarse_solver in ("splu", "spsolve") and matrix_free:
            raise ValueError("Matrix free is not supported with splu solver use cg instead.")
        if coarse_solver not in ("cg", "gmres", "splu", "spsolve"):
            raise ValueError("Coarse solver not recognized.")
        if matrix_free:
            raise NotImplementedError("Matrix free is not implemented yet.")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.last_iters = 0
        self._configured = None
        self.autotune = autotune
        self.tuned = None
        # graph=True: each solve (hierarchy set-up + the whole PCG loop) is one CUDA graph
        # launch with device-side loop control; False: host-driven loop, same launches
        self.graph = graph
        # tune_sweeps (default: on for precision="mixed", off for "fp64", which keeps the
        # reference's n_smooth on every level): per-level smoothing sweeps chosen by timing
        # whole solves of the first system; the converged solution meets the same tolerance
        self.tune_sweeps = (precision == "mixed") if tune_sweeps is None else bool(tune_sweeps)
        self.sweeps = None
        # element counts not divisible by 2**n_level: solve on a padded grid (_PaddedGrid)
        self._pad = None
        self._inner = None
        if any(int(v) % (2 ** n_level) for v in mesh.nel):
            self._pad = _PaddedGrid(kernel, n_level)
            self._inner = CuMultiGrid(self._pad.kernel.mesh, self._pad.kernel, maxiter=maxiter, tol=tol,
                                      n_smooth=n_smooth, omega=omega, n_level=n_level, cycle=cycle, w_level=w_level,
                                      min_omega=min_omega, omega_boost=omega_boost, precision=precision,
                                      autotune=autotune, graph=graph, tune_sweeps=tune_sweeps,
                                      omega_carry=self.omega_carry, mixed_omega=mixed_omega)

    def reset(self):
        self.last_x0 = None
        if self._inner is not None:
            self._inner.reset()

    def _omega_value(self):
        """The weight a fixed mode would hold (None: this solver only runs the schedule)."""
        if self.precision != "mixed" or self.mixed_omega is None:
            return None
        return float(self.max_omega) if self.mixed_omega in ("auto", "max") else float(self.mixed_omega)

    @property
    def fixed_omega(self):
        """The smoother weight the mixed path holds fixed now, or None (the reference's schedule)."""
        return self._omega_value() if self._omega_mode == "fixed" else None

    def _set_omega_mode(self, mode):
        self._omega_mode = mode
        if self._inner is not None:
            self._inner._set_omega_mode(mode)
        self._configure()

    def use_omega_schedule(self):
        """Move the mixed path from a fixed smoother weight to the reference's schedule for good
        (after a solve the fixed weight did not converge); returns False when it already runs
        the schedule."""
        if self.fixed_omega is None:
            return False
        self._omega_failed = True
        self._set_omega_mode("schedule")
        return True

    def keep_start(self, x):
        """Copy of a warm start, for the rerun of a solve that the fixed weight did not converge."""
        if self.fixed_omega is None:
            return None
        if self._x_keep is None or self._x_keep.shape != x.shape:
            self._x_keep = torch.empty_like(x)
        self._x_keep.copy_(x)
        return self._x_keep

    def _configure(self):
        fixed = self.fixed_omega
        key = (self.n_level, self.n_smooth, self.max_omega, self.min_omega, self.cycle, tuple(self.w_level),
               self.precision, bool(self.graph), fixed)
        if self._configured == key:
            return
        w = _lib.int_array(self.w_level) if self.w_level else None
        prec = _lib.EDGE_FP64 if self.precision == "fp64" else _lib.EDGE_MIXED
        om, om_min = float(self.max_omega), float(self.min_omega)
        if fixed is not None:
            om = om_min = fixed
        _lib.call("edge_mg_config", self.kernel.handle, int(self.n_level), int(self.n_smooth), om, om_min,
                  1 if self.cycle == "w" else 0, w, len(self.w_level), prec)
        _lib.call("edge_set_graph", self.kernel.handle, 1 if self.graph else 0)
        if self._configured is None:
            _lib.call("edge_mg_set_omega_carry", self.kernel.handle, 1 if self.omega_carry else 0)
        self._configured = key

    def tune(self):
        """Pick the fine-operator tile (warps, TMA stages, y-chunking) by timing each on the
        current density (the project's autotuner); runs once, on the first solve."""
        if self.tuned is not None or not self.autotune or not self.kernel.has_rho:
            return self.tuned
        ms, v, b = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        prec = _lib.EDGE_FP64 if self.precision == "fp64" else _lib.EDGE_MIXED
        self.kernel._bind_stream()
        _lib.call("edge_autotune_fine", self.kernel.handle, prec, 5, ctypes.byref(ms), ctypes.byref(v),
                  ctypes.byref(b))
        kv, kb = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        _lib.call("edge_fine_kind_tiles", self.kernel.handle, kv, kb)
        self.tuned = {"variant": v.value, "blocks_per_sm": b.value, "ms": ms.value,
                      "per_kind": [[int(kv[i]), int(kb[i])] for i in range(3)]}
        return self.tuned

    SWEEP_CANDIDATES = ("1", "1,2", "2", "1,3", "n")
    SWEEP_MARGIN = 0.95  # a pattern with more sweeps than the cheapest must be 5 % faster

    def tune_sweep_counts(self, f, x0=None):
        """Pick per-level smoothing sweeps (fine level first) by timing one solve of K x = f for
        each candidate pattern ("1,2": one sweep on the fine level, two on every coarser
        level; "n": n_smooth everywhere, the reference's V-cycle), every candidate starting
        from x0, and keep the fastest that converges.  Runs once, on the first warm-started
        solve (x0 = the previous solution, as in every later SIMP iteration; solves before it
        use n_smooth); needs the density set.  (Timing solves to tol / 100 instead was tried:
        at 12.8M DOF it overstated what extra sweeps save in the SIMP loop, 25 % fewer PCG
        iterations there against 12 % in the loop, and picked the slower pattern.)"""
        if self.sweeps is not None or not self.tune_sweeps or not self.kernel.has_rho or x0 is None:
            return self.sweeps
        f = _as_dev_f64(f)
        x0 = _as_dev_f64(x0).clone()
        stream = torch.cuda.current_stream()
        x = torch.empty_like(f)
        res, its = ctypes.c_double(), ctypes.c_int()
        self.kernel._bind_stream()
        tol = float(self.tol)

        def timed_solve(pattern):
            _lib.call("edge_mg_set_sweeps", self.kernel.handle, _lib.int_array(pattern), len(pattern))
            x.copy_(x0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.call("edge_mg_solve", self.kernel.handle, _lib.ptr(f), _lib.ptr(x), 1, tol,
                      int(self.maxiter), ctypes.byref(res), ctypes.byref(its))
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1), res.value < tol, its.value

        runs = []
        for cand in self.SWEEP_CANDIDATES:
            if cand == "n":
                pattern = [self.n_smooth] * self.n_level
            else:
                v = [int(t) for t in cand.split(",")]
                pattern = [v[0]] + [v[-1]] * (self.n_level - 1)
            ms, ok, it = timed_solve(pattern)
            if ok:
                runs.append([ms, pattern, it])
        candidates = [{"per_level": r[1], "ms": round(r[0], 3), "pcg_iters": r[2]} for r in runs]
        if not runs:  # nothing converged within maxiter: keep the reference's sweeps
            best = (0.0, [self.n_smooth] * self.n_level, 0)
        else:
            best = pick_sweep_pattern(runs, timed_solve, self.SWEEP_MARGIN, fallback=[self.n_smooth] * self.n_level)
        found = bool(runs) and best[0] > 0.0
        best_ms = best[0] / 2 if found else None
        omega = None
        if self._omega_value() is not None and not self._omega_failed:
            # the chosen pattern once more with the other smoother weight (fixed at omega, or the
            # reference's schedule): keep the faster of the two that converged
            mode = self._omega_mode
            other = "schedule" if mode == "fixed" else "fixed"
            self._set_omega_mode(other)
            ms_o, ok_o, it_o = timed_solve(best[1])
            switch = ok_o and (not found or ms_o < best_ms)
            omega = {"fixed": self._omega_value(), mode + "_ms": round(best_ms, 3) if found else None,
                     other + "_ms": round(ms_o, 3) if ok_o else None, "chosen": other if switch else mode}
            if switch:
                best, best_ms = (ms_o, best[1], it_o), ms_o
            else:
                self._set_omega_mode(mode)
        _lib.call("edge_mg_set_sweeps", self.kernel.handle, _lib.int_array(best[1]), len(best[1]))
        self.sweeps = {"per_level": best[1], "solve_ms": best_ms or 0.0, "pcg_iters": best[2],
                       "tune_tol": tol, "candidates": candidates, "omega": omega}
        return self.sweeps

    @property
    def padded(self):
        """True when this solver works on a padded copy of the grid (odd extents)."""
        return self._pad is not None

    def _run_solve(self, f, x, warm):
        """One solve of K x = f (x: the warm start when warm, overwritten with the solution), on
        this solver's problem or, when padded, on the padded problem through the embedding
        (edge_mg_solve_embedded: the load, warm start and solution stay in the real grid's
        layout); a fixed smoother weight that does not converge is retried on the schedule.
        Returns (residual, iterations)."""
        res, its = ctypes.c_double(), ctypes.c_int()
        target = self._inner if self._pad is not None else self
        target.kernel._bind_stream()
        keep = target.keep_start(x) if warm else None

        def go():
            if self._pad is not None:
                _lib.call("edge_mg_solve_embedded", target.kernel.handle, _lib.int_array(self._pad.nel), _lib.ptr(f),
                          _lib.ptr(x), warm, float(self.tol), int(self.maxiter), ctypes.byref(res), ctypes.byref(its))
            else:
                _lib.call("edge_mg_solve", self.kernel.handle, _lib.ptr(f), _lib.ptr(x), warm, float(self.tol),
                          int(self.maxiter), ctypes.byref(res), ctypes.byref(its))

        go()
        if not res.value < self.tol and self.use_omega_schedule():
            # the fixed smoother weight did not converge: the same solve with the schedule
            if keep is not None:
                x.copy_(keep)
            go()
        return res.value, its.value

    def _solve_padded(self, rhs, use_last):
        inner, pad = self._inner, self._pad
        inner.tol, inner.maxiter = self.tol, self.maxiter
        pad.sync_bcs(self.kernel)
        pad.set_rho(self.kernel)
        inner._configure()
        inner.tune()
        f = _as_dev_f64(rhs)
        warm = 1 if (use_last and self.last_x0 is not None) else 0
        if warm and inner.sweeps is None and inner.tune_sweeps:
            # the sweep autotuner times whole solves on the padded grid (once)
            inner.tune_sweep_counts(pad.embed(f), pad.embed(self.last_x0))
        self._omega_mode, self._omega_failed = inner._omega_mode, inner._omega_failed  # the tuner's choice
        x = self.last_x0 if warm else torch.zeros_like(f)
        res, its = self._run_solve(f, x, warm)
        self.last_x0 = x
        self.last_iters = inner.last_iters = its
        self.tuned, self.sweeps = inner.tuned, inner.sweeps
        return x, res

    def solve(self, rhs, rho=None, use_last=True):
        if not (self.kernel.has_rho or rho is not None):
            raise ValueError("Solver requires a density vector to be passed or set on the kernel.")
        if rho is not None:
            self.kernel.set_rho(rho)
        if self._pad is not None:
            return self._solve_padded(rhs, use_last)
        self._configure()
        self.tune()
        if use_last and self.last_x0 is not None:
            self.tune_sweep_counts(rhs, self.last_x0)
        f = _as_dev_f64(rhs)
        if use_last and self.last_x0 is not None:
            x = self.last_x0
            warm = 1
        else:
            x = torch.zeros_like(f)
            warm = 0
        res, its = self._run_solve(f, x, warm)
        self.last_x0 = x
        self.last_iters = its
        return x, res

    def stats(self):
        if self._inner is not None:
            return self._inner.stats()
        a, b = ctypes.c_double(), ctypes.c_double()
        i, t = ctypes.c_int(), ctypes.c_int()
        _lib.call("edge_last_solve_stats", self.kernel.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(i),
                  ctypes.byref(t))
        return {"setup_ms": a.value, "solve_ms": b.value, "pcg_iters": i.value, "true_residuals": t.value}


class MultiGrid(CuMultiGrid):
    """The reference's CPU multigrid solver (solvers/_multigrid.py:11-230) on the GPU: the same
    algorithm as CuMultiGrid except for the smoother weight, which the CPU solver starts at
    ``omega`` and never resets between solves (CuMultiGrid resets it to ``min_omega`` at
    every solve, as the CuPy solver does), so its PCG iterates are those of the CPU solver.
    In 3-D the two reference solvers' transfers are the same; in 2-D the CPU restriction
    differs from the GPU one (core/_mgm.py:159-160) and this class keeps the GPU one."""
    OMEGA_CARRY = True


class CuCG(Solver):
    """Conjugate gradients without a preconditioner on the matrix-free stiffness operator:
    the reference's CG solver (solvers/_gpu.py:11-58, cupyx cg with M = None; the returned
    residual is recomputed as ||f - K x|| / ||f||).  Works on any grid extent (the multigrid
    needs element counts divisible by 2**n_level) and on unstructured meshes
    (CuUniformStiffnessKernel / CuGeneralStiffnessKernel, the reference's pairing of general
    meshes with CG; there it runs as a host loop with one state read per iteration).  The iteration runs on the device as one
    CUDA graph launch.  matrix_free=False in the reference assembles K first; the product
    and hence the iterates are the same, so here it only records the choice."""

    def __init__(self, kernel, maxiter=1000, tol=1e-5, matrix_free=None):
        if not isinstance(kernel, (CuStructuredStiffnessKernel, _CuGeneralKernel)):
            raise TypeError("CuCG needs one of the package's stiffness kernels")
        self.kernel = kernel
        self.last_x0 = None
        self.tol = tol
        self.maxiter = maxiter
        self.matrix_free = True if matrix_free is None else bool(matrix_free)
        self.last_iters = 0

    def reset(self):
        self.last_x0 = None

    def solve(self, rhs, rho=None, use_last=True):
        if not (self.kernel.has_rho or rho is not None):
            raise ValueError("Solver requires a density vector to be passed or set on the kernel.")
        if rho is not None:
            self.kernel.set_rho(rho)
        f = _as_dev_f64(rhs)
        if use_last and self.last_x0 is not None:
            x = self.last_x0.clone()
            warm = 1
        else:
            x = torch.zeros_like(f)
            warm = 0
        res, its = ctypes.c_double(), ctypes.c_int()
        self.kernel._bind_stream()
        fn = "edge_gen_cg_solve" if isinstance(self.kernel, _CuGeneralKernel) else "edge_cg_solve"
        _lib.call(fn, self.kernel.handle, _lib.ptr(f), _lib.ptr(x), warm, float(self.tol),
                  int(self.maxiter), ctypes.byref(res), ctypes.byref(its))
        if use_last:  # the reference keeps the warm start only on this branch
            self.last_x0 = x
        self.last_iters = its.value
        return x, res.value


CG = CuCG
