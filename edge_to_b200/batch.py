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


def build(spec, precision="mixed", tol=1e-6, maxiter=1000):
    """CuTopOpt of one problem (and its initial design rho = vf)."""
    from . import (CuMultiGrid, CuStructuredFilter2D, CuStructuredMesh2D, CuStructuredStiffnessKernel, CuTopOpt,
                   SingleMaterial, auto_stiffness)
    nelx, nely = spec["nelx"], spec["nely"]
    mesh = CuStructuredMesh2D(nelx, nely, float(nelx), float(nely), stiffness=lambda x: auto_stiffness(x, 1.0, 0.3))
    mat = SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=spec["vf"])
    kernel = CuStructuredStiffnessKernel(mesh)
    filt = CuStructuredFilter2D(mesh, spec["rmin"])
    solver = CuMultiGrid(mesh, kernel, tol=tol, n_level=n_level_for(nelx, nely), maxiter=maxiter,
                         precision=precision)
    opt = CuTopOpt(mesh, mat, kernel, solver, filt, max_iter=1, move=0.2, ch_tol=0, fun_tol=0, verbose=False)
    opt.add_BC_nodal(spec["clamped_nodes"], np.array([[True, True]]))
    opt.add_F_nodal(spec["load_nodes"], spec["forces"])
    rho = torch.full((mesh.n_elements,), spec["vf"], dtype=torch.float64, device="cuda")
    return opt, rho


class BatchSIMP:
    """SIMP iterations of many problems, spread over `n_threads` host threads with one CUDA
    stream each.  ``step(n)`` runs n iterations of every problem and returns the device time
    (ms) from the first launch to the last completion, measured with CUDA events."""

    def __init__(self, specs, precision="mixed", tol=1e-6, maxiter=1000, n_threads=8):
        self.specs = list(specs)
        self.n_threads = max(1, min(n_threads, len(self.specs)))
        self.streams = [torch.cuda.Stream() for _ in range(self.n_threads)]
        self.items = []
        for k, spec in enumerate(self.specs):
            with torch.cuda.stream(self.streams[k % self.n_threads]):
                opt, rho = build(spec, precision, tol, maxiter)
            self.items.append({"opt": opt, "rho": rho, "dr": None, "it": 0, "comp": [], "pcg": []})
        torch.cuda.synchronize()

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
