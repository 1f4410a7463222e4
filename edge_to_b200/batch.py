"""Many independent 2-D SIMP problems of uneven size at once.

The batching configuration of this project: randomized minimum-compliance problems on
structured Q4 grids, each drawn from its own seed,

  nelx ~ U{64..512}, nely ~ U{32..256}, volume fraction ~ U[0.2, 0.6], r_min ~ U[1.5, 3.0],
  1-2 clamped boundary segments, each 10-50 % of the length of a random edge (both DOFs fixed),
  1-4 unit point loads with a uniformly random direction at random unclamped boundary nodes,
  E0 = 1, Emin (void) = 1e-9, nu = 0.3, penalty 3, move 0.2,

solved with the package's drop-in objects (CuStructuredMesh2D, CuStructuredStiffnessKernel,
CuStructuredFilter2D, SingleMaterial, CuMultiGrid, CuTopOpt).  Extents that the multigrid
cannot coarsen n_level times are handled by CuMultiGrid's padded grid; every solve is one
CUDA graph launch.  Problems are spread over host threads, each with its own CUDA stream
and its own problems, so that the solves of different problems overlap on the GPU (the
library releases the GIL inside every call).  The reference has no batch driver; its
randomizer module (randomizer/ConfigSolve.py) is the intent this follows.
"""
import threading

import numpy as np
import torch

# edges: 0 x = 0, 1 x = nelx, 2 y = 0, 3 y = nely
_EDGES = 4


def random_spec(index, seed=0, nelx_range=(64, 512), nely_range=(32, 256)):
    """The problem of the batch with this index (numpy default_rng(seed + index))."""
    rng = np.random.default_rng(seed + index)
    nelx = int(rng.integers(nelx_range[0], nelx_range[1] + 1))
    nely = int(rng.integers(nely_range[0], nely_range[1] + 1))
    vf = float(rng.uniform(0.2, 0.6))
    rmin = float(rng.uniform(1.5, 3.0))
    segments = []
    for _ in range(int(rng.integers(1, 3))):
        edge = int(rng.integers(0, _EDGES))
        length_el = nely if edge < 2 else nelx
        n = max(1, int(round(float(rng.uniform(0.1, 0.5)) * length_el)))
        start = int(rng.integers(0, length_el - n + 1))
        segments.append((edge, start, n))
    clamped = _segment_nodes(nelx, nely, segments)
    boundary = np.setdiff1d(_boundary_nodes(nelx, nely), clamped)
    n_load = int(rng.integers(1, 5))
    load_nodes = rng.choice(boundary, size=n_load, replace=False)
    ang = rng.uniform(0.0, 2.0 * np.pi, size=n_load)
    forces = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    return {"index": index, "nelx": nelx, "nely": nely, "vf": vf, "rmin": rmin, "segments": segments,
            "clamped_nodes": clamped, "load_nodes": np.asarray(load_nodes, dtype=np.int64), "forces": forces}


def shard_specs(n, rank, seed=0):
    """The n problems of one rank when the batch runs on several GPUs: problem indices
    rank * n .. rank * n + n - 1, so every rank has its own seeded problems (rank 0's are the
    single-GPU batch) and no two ranks share one."""
    return [random_spec(rank * n + i, seed) for i in range(n)]


def _node(nelx, i, j):
    return j * (nelx + 1) + i  # reference 2-D node numbering (core/_geom.py:20-25)


def _edge_node(nelx, nely, edge, t):
    if edge == 0:
        return _node(nelx, 0, t)
    if edge == 1:
        return _node(nelx, nelx, t)
    if edge == 2:
        return _node(nelx, t, 0)
    return _node(nelx, t, nely)


def _segment_nodes(nelx, nely, segments):
    ids = [_edge_node(nelx, nely, e, t) for e, start, n in segments for t in range(start, start + n + 1)]
    return np.unique(np.asarray(ids, dtype=np.int64))


def _boundary_nodes(nelx, nely):
    ids = [_edge_node(nelx, nely, e, t) for e in range(_EDGES)
           for t in range((nely if e < 2 else nelx) + 1)]
    return np.unique(np.asarray(ids, dtype=np.int64))


def n_level_for(nelx, nely, max_level=4):
    """Multigrid depth: coarsen while the shorter side keeps >= 2 coarse elements."""
    lv = 1
    while lv < max_level and min(nelx, nely) >> (lv + 1) >= 2:
        lv += 1
    return lv


def build(spec, precision="mixed", tol=1e-6, maxiter=1000, max_level=4):
    """CuTopOpt of one problem (and its initial design rho = vf)."""
    from . import (CuMultiGrid, CuStructuredFilter2D, CuStructuredMesh2D, CuStructuredStiffnessKernel, CuTopOpt,
                   SingleMaterial, auto_stiffness)
    nelx, nely = spec["nelx"], spec["nely"]
    mesh = CuStructuredMesh2D(nelx, nely, float(nelx), float(nely), stiffness=lambda x: auto_stiffness(x, 1.0, 0.3))
    mat = SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=spec["vf"])
    kernel = CuStructuredStiffnessKernel(mesh)
    filt = CuStructuredFilter2D(mesh, spec["rmin"])
    solver = CuMultiGrid(mesh, kernel, tol=tol, n_level=n_level_for(nelx, nely, max_level), maxiter=maxiter,
                         precision=precision)
    opt = CuTopOpt(mesh, mat, kernel, solver, filt, max_iter=1, move=0.2, ch_tol=0, fun_tol=0, verbose=False)
    opt.add_BC_nodal(spec["clamped_nodes"], np.array([[True, True]]))
    opt.add_F_nodal(spec["load_nodes"], spec["forces"])
    rho = torch.full((mesh.n_elements,), spec["vf"], dtype=torch.float64, device="cuda")
    return opt, rho


class BatchAnalysis:
    """The analyses of many problems with all their solves in one persistent launch
    (edge_batch_solve_and_process): ``solve_and_process(rhos, iteration)`` is the batched form
    of CuTopOpt.solve_and_process for a list of CuTopOpt objects on 2-D structured grids with
    CuMultiGrid solvers (V-cycle) and one SingleMaterial law.  A problem whose solver runs on a
    padded grid contributes that grid's problem (its constraints set once here); the filter,
    law and sensitivities stay on the real grid.  The FP64 Krylov recurrence of the batched
    solve is preconditioned by each solver's V-cycle in its precision."""

    def __init__(self, opts, threads=512, sweeps=None, team=1, split_dof=0):
        import ctypes
        from . import CuMultiGrid, SingleMaterial, _lib
        self.opts = list(opts)
        probs, filts, nelx, nely = [], [], [], []
        for opt in self.opts:
            sv = opt.solver
            if not isinstance(sv, CuMultiGrid) or not isinstance(opt.material_model, SingleMaterial):
                raise TypeError("BatchAnalysis needs CuMultiGrid solvers and SingleMaterial laws")
            if sv.padded:
                if not opt.kernel.has_rho:  # the padded grid's constraints are copied with a density
                    opt.kernel.set_rho(torch.full((opt.mesh.n_elements,), float(opt.material_model.void),
                                                  dtype=torch.float64, device="cuda"))
                sv._pad.sync(opt.kernel)
                inner = sv._inner
                inner.tol, inner.maxiter = sv.tol, sv.maxiter
                inner._configure()
                h = inner.kernel.handle
            else:
                sv._configure()
                h = opt.kernel.handle
            if sweeps is not None:  # (fine level, coarser levels) smoothing sweeps per V-cycle
                pat = [int(sweeps[0])] + [int(sweeps[-1])] * (int(sv.n_level) - 1)
                _lib.call("edge_mg_set_sweeps", h, _lib.int_array(pat), len(pat))
            probs.append(h)
            filts.append(opt.filter_kernel.handle)
            nelx.append(int(opt.mesh.nel[0]))
            nely.append(int(opt.mesh.nel[1]))
        n = len(self.opts)
        laws = {(float(o.material_model.void), float(o.material_model.current_penalty(0))) for o in self.opts}
        if len(laws) != 1:
            raise ValueError("every problem of a batch needs the same void stiffness and penalty")
        self._probs = (ctypes.c_void_p * n)(*probs)
        self._filts = (ctypes.c_void_p * n)(*filts)
        h = ctypes.c_void_p()
        _lib.call("edge_batch_create", n, self._probs, self._filts, _lib.int_array(nelx), _lib.int_array(nely),
                  ctypes.byref(h))
        self.handle = h
        _lib.call("edge_batch_set_threads", self.handle, int(threads), int(team))
        _lib.call("edge_batch_set_split", self.handle, int(split_dof), 1024)
        self.U = [torch.zeros_like(o.f) for o in self.opts]
        self.warm = False
        self.last_iters = [0] * n

    def close(self):
        from . import _lib
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.call("edge_batch_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def problem_times(self):
        """(start_ms, end_ms) of every problem's solve in the last solve launch."""
        import ctypes
        from . import _lib
        n = len(self.opts)
        a, b = (ctypes.c_double * n)(), (ctypes.c_double * n)()
        _lib.call("edge_batch_last_problem_times", self.handle, a, b)
        return list(a), list(b)

    def update_design(self, rhos, drs):
        """The OC updates of every problem in one launch (edge_batch_oc_update): the batched
        form of CuTopOpt.update_design; returns the new designs."""
        import ctypes
        from . import _lib
        n = len(self.opts)
        rhos = [r.reshape(-1).to(dtype=torch.float64).contiguous() for r in rhos]
        drs = [d.reshape(-1).to(dtype=torch.float64).contiguous() for d in drs]
        new = [torch.empty_like(r) for r in rhos]
        P = lambda ts: (ctypes.c_void_p * n)(*[t.data_ptr() for t in ts])  # noqa: E731
        moves = {float(o.move) for o in self.opts}
        if len(moves) != 1:
            raise ValueError("every problem of a batch needs the same move limit")
        A = _lib.double_array([float(np.asarray(o.mesh.As).reshape(-1)[0]) for o in self.opts])
        vol = _lib.double_array([float(o.mesh.volume) for o in self.opts])
        vf = _lib.double_array([float(o.material_model.volume_fraction) for o in self.opts])
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.call("edge_batch_oc_update", self.handle, P(rhos), P(drs), A, vol, vf, moves.pop(), P(new), None, None,
                  stream)
        return new

    def solve_and_process(self, rhos, iteration):
        """(compliances, drs, residuals) of the designs rhos (one per problem, on the device)."""
        import ctypes
        from . import _lib
        n = len(self.opts)
        rhos = [r.reshape(-1).to(dtype=torch.float64).contiguous() for r in rhos]
        drs = [torch.empty_like(r) for r in rhos]
        mm = self.opts[0].material_model
        pen = float(mm.current_penalty(iteration))
        P = lambda ts: (ctypes.c_void_p * n)(*[t.data_ptr() for t in ts])  # noqa: E731
        comp = (ctypes.c_double * n)()
        res = (ctypes.c_double * n)()
        its = (ctypes.c_int * n)()
        fs = [o.f for o in self.opts]
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        sv = self.opts[0].solver
        _lib.call("edge_batch_solve_and_process", self.handle, P(rhos), pen, float(mm.void), P(fs), P(self.U),
                  1 if self.warm else 0, float(sv.tol), int(sv.maxiter), comp, P(drs), res, its, stream)
        self.warm = all(o.reuse_sol for o in self.opts)
        self.last_iters = list(its)
        t = [ctypes.c_double() for _ in range(3)]
        _lib.call("edge_batch_last_times", self.handle, *[ctypes.byref(v) for v in t])
        self.last_times = {"setup_ms": t[0].value, "solve_ms": t[1].value, "post_ms": t[2].value}
        for o, u, it in zip(self.opts, self.U, its):
            o._U = u
            o.solver.last_x0 = u
            o.solver.last_iters = int(it)
        return list(comp), [d.reshape(-1, 1) for d in drs], list(res)


class BatchSIMP:
    """SIMP iterations of many problems, spread over `n_threads` host threads with one CUDA
    stream each.  ``step(n)`` runs n iterations of every problem and returns the device time
    (ms) from the first launch to the last completion, measured with CUDA events."""

    def __init__(self, specs, precision="mixed", tol=1e-6, maxiter=1000, n_threads=8, persistent=False,
                 max_level=4, block_threads=512, sweeps=None, team=1, split_dof=0):
        self.specs = list(specs)
        self.persistent = bool(persistent)
        self.n_threads = 1 if self.persistent else max(1, min(n_threads, len(self.specs)))
        self.streams = [torch.cuda.Stream() for _ in range(self.n_threads)]
        self.items = []
        for k, spec in enumerate(self.specs):
            with torch.cuda.stream(self.streams[k % self.n_threads]):
                opt, rho = build(spec, precision, tol, maxiter, max_level)
            self.items.append({"opt": opt, "rho": rho, "dr": None, "it": 0, "comp": [], "pcg": []})
        torch.cuda.synchronize()
        # persistent: every analysis's solves in one launch and every OC update in one launch
        # (BatchAnalysis), all on one stream; phase_ms sums the device time of the analyses'
        # phases (per-problem preparation, the solve launch, post-processing)
        self.batch = None
        self.phase_ms = {}
        if self.persistent:
            with torch.cuda.stream(self.streams[0]):
                self.batch = BatchAnalysis([it["opt"] for it in self.items], threads=block_threads, sweeps=sweeps,
                                           team=team, split_dof=split_dof)
            torch.cuda.synchronize()

    def _run_persistent(self, n_iter):
        items = self.items
        with torch.cuda.stream(self.streams[0]):
            for _ in range(n_iter):
                first = items[0]["dr"] is None
                if not first:
                    rhos = self.batch.update_design([item["rho"] for item in items], [item["dr"] for item in items])
                    for item, r in zip(items, rhos):
                        item["rho"] = r
                comps, drs, _ = self.batch.solve_and_process([item["rho"] for item in items], items[0]["it"])
                for k, v in self.batch.last_times.items():
                    self.phase_ms[k] = self.phase_ms.get(k, 0.0) + v
                for item, c, d, it in zip(items, comps, drs, self.batch.last_iters):
                    item["dr"] = d
                    if not first:
                        item["it"] += 1
                    item["comp"].append(float(c))
                    item["pcg"].append(int(it))
            self._end[0].record(self.streams[0])

    def _run(self, t, n_iter, err):
        try:
            with torch.cuda.stream(self.streams[t]):
                for item in self.items[t::self.n_threads]:
                    opt = item["opt"]
                    for _ in range(n_iter):
                        if item["dr"] is None:
                            c, item["dr"], _ = opt.solve_and_process(item["rho"], item["it"])
                        else:
                            item["rho"] = opt.update_design(item["rho"], item["dr"])
                            c, item["dr"], _ = opt.solve_and_process(item["rho"], item["it"])
                            item["it"] += 1
                        item["comp"].append(float(c))
                        item["pcg"].append(opt.last_stats.get("pcg_iters", opt.solver.last_iters))
                self._end[t].record(self.streams[t])
        except BaseException as e:  # noqa: BLE001 - reported in step()
            err.append(e)

    def step(self, n_iter):
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record(torch.cuda.current_stream())
        for s in self.streams:
            s.wait_event(start)
        self._end = [torch.cuda.Event(enable_timing=True) for _ in range(self.n_threads)]
        if self.persistent:
            self._run_persistent(n_iter)
            torch.cuda.synchronize()
            return start.elapsed_time(self._end[0])
        err = []
        threads = [threading.Thread(target=self._run, args=(t, n_iter, err)) for t in range(self.n_threads)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        if err:
            raise err[0]
        torch.cuda.synchronize()
        return max(start.elapsed_time(e) for e in self._end)
