"""The reference's CPU SIMP iteration on a structured hex8 grid, multi-threaded (oracle; test
infrastructure).  This is the timed CPU baseline of bench.py, never the product path.

It restates, for the 3-D cantilever of the benchmark, the reference's CPU code path one
SIMP iteration takes (TopOpt/_solver.py:271-335 with StructuredStiffnessKernel,
StructuredFilter3D, MultiGrid and SingleMaterial):

  filter         rho_f = H rho, the cone stencil with per-element normalisation
                 (core/_filter.py:6-124; stencil from oracle.ops.filter_stencil)
  material       E = clip(rho_f^p, void, 1)                   (MaterialModels.py:47-73)
  fine operator  node-basis matrix-free K(E) u with BC rows / columns -> identity, one
                 parallel task per node over the node's elements found through the sorted
                 element-node list (mat_vec_node_basis_parallel_wcon, core/_ops.py:330-368)
  diagonal       the same node loop for diag(K(E)), 1 on constrained DOFs (core/_ops.py:45-76)
  multigrid      set-up: level 1 = R A_0 R^T assembled straight from K0, E and the BC mask
                 (get_restricted_3d_l0_nnz_based, core/_mgm.py:739-828), 27 neighbours x 3
                 components per row; coarser levels R A R^T on CSR matrices
                 (get_restricted_l1p, core/_mgm.py:1259-1294); SuperLU on the coarsest level
                 (solvers/_multigrid.py:108-121).  V-cycle (solvers/_multigrid.py:123-176):
                 n_smooth damped-Jacobi sweeps (each a full product, also from x = 0) with
                 omega * 1.06^level, residual, restriction, recursion, prolongation,
                 n_smooth sweeps on the correction; the coarse levels' products are scipy
                 CSR products (single-threaded, as in the reference).  Transfers: full
                 weighting {1, 1/2, 1/4, 1/8} / boundary totals (restriction_matvec_3d,
                 prolongation_matvec_3d, core/_mgm.py:10-92, 176-245).
  PCG            solvers/_multigrid.py:178-229: warm start, omega schedule carried across
                 solves (the CPU solver never resets it), stop at ||r|| / ||f|| < tol.
  sensitivity    dk_e = -u_e^T K0 u_e (process_dk, core/_ops.py:5-13), dr = H^T(p clip^(p-1) dk)
  OC             oracle.topopt.oc_update (TopOpt/_solver.py:271-311)

All kernels are Numba-parallel over the host's threads except where the reference itself
uses scipy.  The numbering is the reference's (core/_geom.py:43-57).
"""
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
from numba import njit, prange

from . import ops
from .elements import HEX8_CORNERS, element_measure, hex8_stiffness
from .grid import Grid
from .topopt import oc_update

_W1 = np.array([1.0, 0.5, 0.25, 0.125])
_WB = np.array([8.0, 6.0, 4.5, 3.375])  # full-weighting totals by number of boundary axes


# ----------------------------------------------------------------------------- structure
def element_nodes(nel):
    """elements_flat of the reference: the 8 corner nodes of every element, element order
    e = i*nely*nelz + j*nelz + k, corner order HEX8_CORNERS (core/_geom.py:43-57)."""
    nelx, nely, nelz = nel
    nx, nz = nelx + 1, nelz + 1
    i, j, k = np.meshgrid(np.arange(nelx), np.arange(nely), np.arange(nelz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    out = np.empty((i.size, 8), dtype=np.int32)
    for a, (di, dj, dk) in enumerate(HEX8_CORNERS):
        out[:, a] = (j + dj) * nx * nz + (i + di) * nz + (k + dk)
    return out.reshape(-1)


def node_adjacency(elements_flat, n_nodes):
    """Stable sort of the element-node list and each node's range in it (the reference's
    sorter / node_ids); position p of the list is corner p % 8 of element p // 8."""
    sorter = np.argsort(elements_flat, kind="stable").astype(np.int64)
    counts = np.bincount(elements_flat, minlength=n_nodes)
    ptr = np.zeros(n_nodes + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(counts)
    return sorter, ptr


# ----------------------------------------------------------------------------- kernels
@njit(parallel=True, cache=True)
def _matvec(K0, ef, sorter, ptr, E, u, cons, out):
    n_nodes = ptr.shape[0] - 1
    for i in prange(n_nodes):
        for k in range(3):
            out[3 * i + k] = u[3 * i + k] if cons[3 * i + k] else 0.0
        for jj in range(ptr[i], ptr[i + 1]):
            pos = sorter[jj]
            e = pos // 8
            rel = pos - 8 * e
            w = E[e]
            for k in range(3):
                if cons[3 * i + k]:
                    continue
                val = 0.0
                for l in range(24):
                    kk = ef[8 * e + l // 3] * 3 + l % 3
                    if cons[kk]:
                        continue
                    val += K0[rel * 3 + k, l] * u[kk]
                out[3 * i + k] += val * w


@njit(parallel=True, cache=True)
def _matvec_s(nel, K0, E, u, cons, out, C3):
    """The same node-basis product with each node's elements found from the structured
    numbering instead of the sorted element-node list (the same arithmetic and summation
    order; about five times faster than the list lookups on the host)."""
    nelx, nely, nelz = nel[0], nel[1], nel[2]
    nx, ny, nz = nelx + 1, nely + 1, nelz + 1
    for j in prange(ny):
        for i in range(nx):
            for k in range(nz):
                node = (j * nx + i) * nz + k
                for c in range(3):
                    out[node * 3 + c] = u[node * 3 + c] if cons[node * 3 + c] else 0.0
                for a in range(8):
                    ei, ej, ek = i - C3[a, 0], j - C3[a, 1], k - C3[a, 2]
                    if ei < 0 or ej < 0 or ek < 0 or ei >= nelx or ej >= nely or ek >= nelz:
                        continue
                    w = E[(ei * nely + ej) * nelz + ek]
                    for c in range(3):
                        if cons[node * 3 + c]:
                            continue
                        val = 0.0
                        for b in range(8):
                            nb = ((ej + C3[b, 1]) * nx + (ei + C3[b, 0])) * nz + ek + C3[b, 2]
                            for d in range(3):
                                kk = nb * 3 + d
                                if cons[kk]:
                                    continue
                                val += K0[a * 3 + c, b * 3 + d] * u[kk]
                        out[node * 3 + c] += val * w


@njit(parallel=True, cache=True)
def _diagonal(K0, ef, sorter, ptr, E, cons, out):
    n_nodes = ptr.shape[0] - 1
    for i in prange(n_nodes):
        for k in range(3):
            out[3 * i + k] = 0.0
        for jj in range(ptr[i], ptr[i + 1]):
            pos = sorter[jj]
            e = pos // 8
            rel = pos - 8 * e
            for k in range(3):
                out[3 * i + k] += K0[rel * 3 + k, rel * 3 + k] * E[e]
        for k in range(3):
            if cons[3 * i + k]:
                out[3 * i + k] = 1.0


@njit(parallel=True, cache=True)
def _dk(K0, ef, U, out):
    n_el = out.shape[0]
    for e in prange(n_el):
        s = 0.0
        for a in range(24):
            ua = U[ef[8 * e + a // 3] * 3 + a % 3]
            v = 0.0
            for b in range(24):
                v += K0[a, b] * U[ef[8 * e + b // 3] * 3 + b % 3]
            s += ua * v
        out[e] = -s


@njit(parallel=True, cache=True)
def _filter_norm(nelx, nely, nelz, offs, w, N):
    for e in prange(nelx * nely * nelz):
        ix, iy, iz = e // (nely * nelz), (e // nelz) % nely, e % nelz
        s = 0.0
        for t in range(w.shape[0]):
            jx, jy, jz = ix + offs[t, 0], iy + offs[t, 1], iz + offs[t, 2]
            if 0 <= jx < nelx and 0 <= jy < nely and 0 <= jz < nelz:
                s += w[t]
        N[e] = s


@njit(parallel=True, cache=True)
def _filter(nelx, nely, nelz, offs, w, N, v, out, transpose):
    for e in prange(nelx * nely * nelz):
        ix, iy, iz = e // (nely * nelz), (e // nelz) % nely, e % nelz
        s = 0.0
        for t in range(w.shape[0]):
            jx, jy, jz = ix + offs[t, 0], iy + offs[t, 1], iz + offs[t, 2]
            if 0 <= jx < nelx and 0 <= jy < nely and 0 <= jz < nelz:
                j = (jx * nely + jy) * nelz + jz
                s += (w[t] / N[j]) * v[j] if transpose else w[t] * v[j]
        out[e] = s if transpose else s / N[e]


@njit(cache=True)
def _wtotal(ci, cj, ck, ncx, ncy, ncz):
    nb = 0
    if ci == 0 or ci == ncx - 1:
        nb += 1
    if cj == 0 or cj == ncy - 1:
        nb += 1
    if ck == 0 or ck == ncz - 1:
        nb += 1
    return _WB[nb]


@njit(parallel=True, cache=True)
def _restrict(nel, v, out):
    nfx, nfy, nfz = nel[0] + 1, nel[1] + 1, nel[2] + 1
    ncx, ncy, ncz = nel[0] // 2 + 1, nel[1] // 2 + 1, nel[2] // 2 + 1
    for c in prange(ncx * ncy * ncz):
        ck = c % ncz
        ci = (c // ncz) % ncx
        cj = c // (ncz * ncx)
        W = _wtotal(ci, cj, ck, ncx, ncy, ncz)
        for d in range(3):
            s = 0.0
            for di in range(-1, 2):
                fi = 2 * ci + di
                if fi < 0 or fi >= nfx:
                    continue
                for dj in range(-1, 2):
                    fj = 2 * cj + dj
                    if fj < 0 or fj >= nfy:
                        continue
                    for dk in range(-1, 2):
                        fk = 2 * ck + dk
                        if fk < 0 or fk >= nfz:
                            continue
                        s += _W1[abs(di) + abs(dj) + abs(dk)] * v[((fj * nfx + fi) * nfz + fk) * 3 + d]
            out[c * 3 + d] = s / W


@njit(parallel=True, cache=True)
def _prolong(nel, v, out):
    nfx, nfy, nfz = nel[0] + 1, nel[1] + 1, nel[2] + 1
    ncx, ncy, ncz = nel[0] // 2 + 1, nel[1] // 2 + 1, nel[2] // 2 + 1
    for f in prange(nfx * nfy * nfz):
        fk = f % nfz
        fi = (f // nfz) % nfx
        fj = f // (nfz * nfx)
        for d in range(3):
            s = 0.0
            cnt = 0
            for a in range(2):
                if a == 1 and fi % 2 == 0:
                    continue
                ci = fi // 2 + a
                if ci >= ncx:
                    continue
                for b in range(2):
                    if b == 1 and fj % 2 == 0:
                        continue
                    cj = fj // 2 + b
                    if cj >= ncy:
                        continue
                    for g in range(2):
                        if g == 1 and fk % 2 == 0:
                            continue
                        ck = fk // 2 + g
                        if ck >= ncz:
                            continue
                        s += v[((cj * ncx + ci) * ncz + ck) * 3 + d] / _wtotal(ci, cj, ck, ncx, ncy, ncz)
                        cnt += 1
            out[f * 3 + d] = s / cnt


@njit(parallel=True, cache=True)
def _galerkin_l0(nel, K0, ef, sorter, ptr, E, cons, indptr, indices, data):
    """Level-1 operator R A_0 R^T, row by row (one coarse node per task): for every fine node
    in the coarse node's stencil, its row of A_0 (element blocks, or the identity row of a
    constrained DOF) mapped onto the coarse parents of each column node."""
    nfx, nfy, nfz = nel[0] + 1, nel[1] + 1, nel[2] + 1
    ncx, ncy, ncz = nel[0] // 2 + 1, nel[1] // 2 + 1, nel[2] // 2 + 1
    for c in prange(ncx * ncy * ncz):
        ck = c % ncz
        ci = (c // ncz) % ncx
        cj = c // (ncz * ncx)
        Wc = _wtotal(ci, cj, ck, ncx, ncy, ncz)
        acc = np.zeros((3, 27, 3))
        for di in range(-1, 2):
            fi = 2 * ci + di
            if fi < 0 or fi >= nfx:
                continue
            for dj in range(-1, 2):
                fj = 2 * cj + dj
                if fj < 0 or fj >= nfy:
                    continue
                for dk in range(-1, 2):
                    fk = 2 * ck + dk
                    if fk < 0 or fk >= nfz:
                        continue
                    n = (fj * nfx + fi) * nfz + fk
                    r = _W1[abs(di) + abs(dj) + abs(dk)] / Wc
                    for a in range(3):
                        if cons[3 * n + a]:  # identity row: column n itself
                            _scatter(acc, a, a, r, fi, fj, fk, ci, cj, ck, ncx, ncy, ncz)
                            continue
                        for jj in range(ptr[n], ptr[n + 1]):
                            pos = sorter[jj]
                            e = pos // 8
                            rel = pos - 8 * e
                            w = r * E[e]
                            for m in range(8):
                                mn = ef[8 * e + m]
                                mk = mn % nfz
                                mi = (mn // nfz) % nfx
                                mj = mn // (nfz * nfx)
                                for b in range(3):
                                    if cons[3 * mn + b]:
                                        continue
                                    _scatter(acc, a, b, w * K0[rel * 3 + a, m * 3 + b], mi, mj, mk, ci, cj, ck, ncx,
                                             ncy, ncz)
        for a in range(3):
            for t in range(27):
                oi, oj, ok = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
                qi, qj, qk = ci + oi, cj + oj, ck + ok
                inside = 0 <= qi < ncx and 0 <= qj < ncy and 0 <= qk < ncz
                q = (qj * ncx + qi) * ncz + qk if inside else c
                for b in range(3):
                    p = indptr[3 * c + a] + t * 3 + b
                    indices[p] = 3 * q + b if inside else 3 * c + a
                    data[p] = acc[a, t, b] if inside else 0.0


@njit(cache=True)
def _scatter(acc, a, b, v, mi, mj, mk, ci, cj, ck, ncx, ncy, ncz):
    """acc[a, parent, b] += v * R[parent, fine node (mi, mj, mk)] for every coarse parent of
    the fine node within one coarse step of (ci, cj, ck)."""
    for pi in range(mi // 2, mi // 2 + 1 + (mi % 2)):
        if pi >= ncx or abs(pi - ci) > 1:
            continue
        for pj in range(mj // 2, mj // 2 + 1 + (mj % 2)):
            if pj >= ncy or abs(pj - cj) > 1:
                continue
            for pk in range(mk // 2, mk // 2 + 1 + (mk % 2)):
                if pk >= ncz or abs(pk - ck) > 1:
                    continue
                dist = abs(mi - 2 * pi) + abs(mj - 2 * pj) + abs(mk - 2 * pk)
                wr = _W1[dist] / _wtotal(pi, pj, pk, ncx, ncy, ncz)
                t = (pi - ci + 1) * 9 + (pj - cj + 1) * 3 + (pk - ck + 1)
                acc[a, t, b] += v * wr


# ----------------------------------------------------------------------------- the problem
class CpuSimpReference:
    """One structured hex8 SIMP problem (the benchmark's cantilever) on the host cores."""

    def __init__(self, nel, vf, rmin, n_level, tol, penalty=3.0, void=1e-9, nu=0.3, move=0.2, n_smooth=3,
                 omega=0.5, min_omega=0.4, maxiter=1000, indexing="structured"):
        self.nel = tuple(int(v) for v in nel)
        self.grid = Grid(self.nel)
        g = self.grid
        self.K0 = hex8_stiffness(1.0, 1.0, 1.0, 1.0, nu)
        self.A = element_measure(g.h)
        self.vol = self.A * g.n_el
        self.vf, self.penalty, self.void, self.move = vf, penalty, void, move
        self.n_level, self.tol, self.n_smooth, self.maxiter = n_level, tol, n_smooth, maxiter
        self.omega = omega                      # carried across solves (the CPU solver)
        self.min_omega = max(omega / 2, min_omega)
        self.d_omega = omega - self.min_omega
        self.ef = element_nodes(self.nel)
        self.sorter, self.ptr = node_adjacency(self.ef, g.n_nodes)
        offs, w = ops.filter_stencil(g, rmin)
        self.offs, self.fw = offs.astype(np.int64), w
        self.N = np.empty(g.n_el)
        _filter_norm(*self.nel, self.offs, self.fw, self.N)
        # cantilever: x = 0 face clamped, unit total load (0, -1, 0) on the bottom edge at x = L
        nx, ny, nz = g.nn
        self.cons = np.zeros(g.n_dof, dtype=np.bool_)
        j, k = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
        face = (j * nx * nz + k).ravel()
        for d in range(3):
            self.cons[face * 3 + d] = True
        edge = self.nel[0] * nz + np.arange(nz)
        self.f = np.zeros(g.n_dof)
        self.f[edge * 3 + 1] = -1.0 / edge.shape[0]
        self.x = None
        self.nels = [np.array([n >> l for n in self.nel], dtype=np.int64) for l in range(n_level + 1)]
        self._R = {}
        # "list": the reference's node -> element lookups through the sorted element-node
        # list; "structured": the same product with index arithmetic (faster on the host)
        self.indexing = indexing
        self._C3 = HEX8_CORNERS.astype(np.int64)

    # --------------------------------------------------------------- operators
    def matvec(self, E, u):
        out = np.empty_like(u)
        if self.indexing == "list":
            _matvec(self.K0, self.ef, self.sorter, self.ptr, E, u, self.cons, out)
        else:
            _matvec_s(self.nels[0], self.K0, E, u, self.cons, out, self._C3)
        return out

    def filter(self, v, transpose=False):
        out = np.empty_like(v)
        _filter(*self.nel, self.offs, self.fw, self.N, v, out, transpose)
        return out

    def restrict(self, l, v):
        nel = self.nels[l]
        out = np.empty(int(np.prod(nel // 2 + 1)) * 3)
        _restrict(nel, v, out)
        return out

    def prolong(self, l, v):
        nel = self.nels[l]
        out = np.empty(int(np.prod(nel + 1)) * 3)
        _prolong(nel, v, out)
        return out

    def _rmat(self, l):
        if l not in self._R:
            self._R[l] = ops.restriction_matrix(Grid(tuple(int(v) for v in self.nels[l])), "cpu")
        return self._R[l]

    def setup(self, E):
        """Multigrid levels for K(E): Jacobi diagonals, level 1 from K0/E, coarser levels by
        R A R^T, SuperLU of the coarsest."""
        g = self.grid
        D0 = np.empty(g.n_dof)
        _diagonal(self.K0, self.ef, self.sorter, self.ptr, E, self.cons, D0)
        self.levels = [(None, 1.0 / D0)]
        rows = int(np.prod(self.nels[1] + 1)) * 3
        indptr = np.arange(rows + 1, dtype=np.int64) * 81   # 27 coarse neighbours x 3 components
        indices = np.empty(rows * 81, dtype=np.int64)
        data = np.empty(rows * 81)
        _galerkin_l0(self.nels[0], self.K0, self.ef, self.sorter, self.ptr, E, self.cons, indptr, indices, data)
        A = sp.csr_matrix((data, indices, indptr), shape=(rows, rows))
        self.levels.append((A, 1.0 / A.diagonal()))
        for l in range(1, self.n_level):
            R = self._rmat(l)
            A = (R @ A @ R.T).tocsr()
            self.levels.append((A, 1.0 / A.diagonal()))
        self.coarse = spla.splu(self.levels[-1][0].tocsc())

    def _apply(self, l, E, x):
        return self.matvec(E, x) if l == 0 else self.levels[l][0] @ x

    def _smooth(self, l, E, x, b, n):
        D = self.levels[l][1]
        for _ in range(n):
            x += self.omega * D * (b - self._apply(l, E, x))
        return x

    def vcycle(self, l, E, b):
        if l == self.n_level:
            return self.coarse.solve(b)
        x = np.zeros_like(b)
        s = 1.06 ** l
        self.omega *= s
        x = self._smooth(l, E, x, b, self.n_smooth)
        self.omega /= s
        r = b - self._apply(l, E, x)
        e = self.prolong(l, self.vcycle(l + 1, E, self.restrict(l, r)))
        self.omega *= s
        e = self._smooth(l, E, e, r, self.n_smooth)
        self.omega /= s
        return x + e

    def pcg(self, E, max_iters=None, timer=None):
        """The reference's PCG from the last solution; returns (iterations, residual).  With
        max_iters it stops early (a timing sample); timer(list) receives per-iteration times."""
        x = self.x if self.x is not None else np.zeros(self.grid.n_dof)
        r = self.f - self.matvec(E, x)
        z = self.vcycle(0, E, r)
        p = z.copy()
        rho_old = float(r @ z)
        norm_b = float(np.sqrt(self.f @ self.f))
        R = float(np.sqrt(r @ r)) / norm_b
        limit = self.maxiter if max_iters is None else min(self.maxiter, max_iters)
        it = 0
        for it in range(limit):
            t0 = time.perf_counter()
            q = self.matvec(E, p)
            alpha = rho_old / float(p @ q)
            x += alpha * p
            r -= alpha * q
            R = float(np.sqrt(r @ r)) / norm_b
            if R < self.tol:
                if timer is not None:
                    timer.append(time.perf_counter() - t0)
                break
            self.omega = self.min_omega + self.d_omega / 2 * np.exp((-np.clip(R, self.tol, 1e-1) + self.tol) * 500)
            z = self.vcycle(0, E, r)
            rho_new = float(r @ z)
            p = z + (rho_new / rho_old) * p
            rho_old = rho_new
            if timer is not None:
                timer.append(time.perf_counter() - t0)
        self.x = x
        return it + 1, R

    # --------------------------------------------------------------- one SIMP iteration
    def analysis(self, rho, max_iters=None, timer=None):
        """solve_and_process (TopOpt/_solver.py:312-335).  Returns (compliance, dr, times)
        with times = {"setup": filter + material + multigrid set-up, "pcg": the PCG loop,
        "post": compliance + sensitivity + filter transpose, "pcg_iters": n}."""
        t0 = time.perf_counter()
        rho_f = self.filter(rho)
        E = np.clip(rho_f ** self.penalty, self.void, 1.0)
        self.setup(E)
        t1 = time.perf_counter()
        n, res = self.pcg(E, max_iters, timer)
        t2 = time.perf_counter()
        comp = float(self.f @ self.x)
        dk = np.empty(self.grid.n_el)
        _dk(self.K0, self.ef, self.x, dk)
        dr = self.filter(self.penalty * np.clip(rho_f, self.void, 1.0) ** (self.penalty - 1) * dk, transpose=True)
        t3 = time.perf_counter()
        return comp, dr, {"setup": t1 - t0, "pcg": t2 - t1, "post": t3 - t2, "pcg_iters": n, "residual": res}

    def update(self, rho, dr):
        t0 = time.perf_counter()
        rho_new, lam, steps = oc_update(rho, dr, self.A, self.vol, self.vf, self.move)
        return rho_new, time.perf_counter() - t0


def warm_jit():
    """Compile every kernel once on a tiny grid (Numba caches them on disk)."""
    for indexing in ("list", "structured"):
        p = CpuSimpReference((4, 2, 2), 0.3, 1.5, 1, 1e-6, indexing=indexing)
        rho = np.full(p.grid.n_el, 0.3)
        c, dr, _ = p.analysis(rho, max_iters=2)
        p.update(rho, dr)


def measure(nel, vf, rmin, n_level, tol, samples=8, log=None):
    """Seconds per SIMP iteration of the reference's CPU algorithm on this host, timed.

    1. The first SIMP analysis at rho = vf, solved to tol (the CPU solver's own PCG count
       n0) and timed part by part: set-up (filter, material law, multigrid hierarchy),
       PCG loop, post-processing (compliance, sensitivity, filter transpose).
    2. The OC update that follows it, timed.
    3. `samples` more PCG iterations of the same system (the loop continued), each timed.
    The iteration time is set-up + post + OC + n0 * (median PCG iteration).  Later SIMP
    iterations need more PCG iterations than the cold first one, so this is an upper bound
    of the CPU rate.  Returns a dict of the parts."""
    import numba
    t0 = time.perf_counter()
    warm_jit()
    p = CpuSimpReference(nel, vf, rmin, n_level, tol)
    t_build = time.perf_counter() - t0
    if log:
        log(f"cpu reference: jit + build {t_build:.1f} s")
    rho = np.full(p.grid.n_el, float(vf))
    comp, dr, tt = p.analysis(rho)
    if log:
        log(f"cpu reference: first analysis {tt}")
    rho1, t_oc = p.update(rho, dr)
    # list-indexing product time, once, for the record (the reference's own lookups)
    E = np.clip(p.filter(rho1) ** p.penalty, p.void, 1.0)
    pl = CpuSimpReference(nel, vf, rmin, n_level, tol, indexing="list")
    t1 = time.perf_counter()
    pl.matvec(E, p.x)
    t_list = time.perf_counter() - t1
    del pl
    t1 = time.perf_counter()
    p.matvec(E, p.x)
    t_struct = time.perf_counter() - t1
    tol0, p.tol = p.tol, 0.0
    ts = []
    p.pcg(np.clip(p.filter(rho) ** p.penalty, p.void, 1.0), max_iters=samples, timer=ts)
    p.tol = tol0
    t_pcg = float(np.median(ts))
    n0 = int(tt["pcg_iters"])
    t_iter = tt["setup"] + tt["post"] + t_oc + n0 * t_pcg
    return {"seconds_per_iteration": t_iter, "setup_s": tt["setup"], "post_s": tt["post"], "oc_s": t_oc,
            "pcg_iteration_s": t_pcg, "pcg_iteration_samples_s": [round(v, 4) for v in ts],
            "first_solve_pcg_iters": n0, "first_solve_pcg_s": tt["pcg"], "first_solve_residual": tt["residual"],
            "matvec_s": t_struct, "matvec_list_indexing_s": t_list, "threads": numba.get_num_threads(),
            "compliance_first": comp, "jit_build_s": t_build}
