"""Operators of the SIMP / GMG path, FP64 (oracle; test infrastructure).

Each function states the reference function it restates.
"""
import numpy as np
import scipy.sparse as sp

from .grid import Grid


# --------------------------------------------------------------------------- stiffness
def assemble(grid: Grid, K0, E, cons=None):
    """K(E) as CSR with constrained rows/columns replaced by the identity.

    Restates mat_vec_node_basis_parallel_wcon (core/_ops.py:330-368, CUDA twin
    core/_templated_cuda.cu:782-834): out_i = sum over unconstrained j of
    sum_e E_e K0[a,b] u_j for unconstrained i, out_i = u_i for constrained i.
    """
    dm = grid.dof_map()
    nl = dm.shape[1]
    rows = np.repeat(dm, nl, axis=1).ravel()
    cols = np.tile(dm, (1, nl)).ravel()
    vals = (np.asarray(E)[:, None] * K0.ravel()[None, :]).ravel()
    if cons is not None and len(cons):
        mask = np.zeros(grid.n_dof, dtype=bool)
        mask[cons] = True
        keep = ~(mask[rows] | mask[cols])
        rows, cols, vals = rows[keep], cols[keep], vals[keep]
        rows = np.concatenate([rows, np.where(mask)[0]])
        cols = np.concatenate([cols, np.where(mask)[0]])
        vals = np.concatenate([vals, np.ones(int(mask.sum()))])
    K = sp.coo_matrix((vals, (rows, cols)), shape=(grid.n_dof, grid.n_dof)).tocsr()
    K.sum_duplicates()
    return K


def diagonal(K):
    """diag(K(E)) with 1 on constrained DOFs (core/_ops.py:45-76)."""
    return K.diagonal().copy()


def dk(grid: Grid, K0, u):
    """dk_e = -u_e^T K0 u_e, unpenalised and without BC masking (core/_ops.py:5-13)."""
    ue = np.asarray(u)[grid.dof_map()]
    return -np.einsum("ea,ab,eb->e", ue, K0, ue)


def fea_integrals(grid: Grid, K0, B, D, w, u):
    """Element strain = B u_e, stress = D strain, strain energy = 1/2 w_e u_e^T K0 u_e
    (core/_ops.py:1032-1058, the structured path of TopOpt/_solver.py:80-137)."""
    ue = np.asarray(u)[grid.dof_map()]
    strain = ue @ np.asarray(B).T
    stress = strain @ np.asarray(D).T
    energy = 0.5 * np.asarray(w) * np.einsum("ea,ab,eb->e", ue, K0, ue)
    return strain, stress, energy


def matvec_free(grid: Grid, K0, E, u, cons_mask=None):
    """Matrix-free K(E) u on the structured grid by corner slicing (numpy, for large grids).

    Same operator as ``assemble`` but never forms K: each of the 2^d corner slices of the
    node array is multiplied by its K0 block and added to the output corners.
    """
    d = grid.dof
    if grid.dim == 2:
        nx, ny = grid.nn
        U = np.asarray(u, dtype=np.float64).reshape(ny, nx, d).copy()
        if cons_mask is not None:
            U[cons_mask.reshape(ny, nx, d)] = 0.0
        Ee = np.asarray(E).reshape(grid.nel[0], grid.nel[1]).T  # (j, i)
        from .elements import Q4_CORNERS as C
        sl = [(slice(c[1], c[1] + grid.nel[1]), slice(c[0], c[0] + grid.nel[0])) for c in C]
    else:
        nx, ny, nz = grid.nn
        U = np.asarray(u, dtype=np.float64).reshape(ny, nx, nz, d).copy()
        if cons_mask is not None:
            U[cons_mask.reshape(ny, nx, nz, d)] = 0.0
        Ee = np.asarray(E).reshape(grid.nel).transpose(1, 0, 2)  # (j, i, k)
        from .elements import HEX8_CORNERS as C
        sl = [(slice(c[1], c[1] + grid.nel[1]), slice(c[0], c[0] + grid.nel[0]),
               slice(c[2], c[2] + grid.nel[2])) for c in C]
    out = np.zeros_like(U)
    n_c = len(sl)
    for a in range(n_c):
        acc = np.zeros(U[sl[a]].shape)
        for b in range(n_c):
            acc += U[sl[b]] @ K0[a * d:(a + 1) * d, b * d:(b + 1) * d].T
        out[sl[a]] += acc * Ee[..., None]
    if cons_mask is not None:
        cm = cons_mask.reshape(out.shape)
        out[cm] = np.asarray(u).reshape(out.shape)[cm]
    return out.ravel()


# --------------------------------------------------------------------------- filter
def filter_stencil(grid: Grid, rmin):
    """Cone-filter offsets and globally normalised weights (geom/_filters.py:72-161)."""
    h = np.array(grid.h)
    scales = h / h.min()
    n = int(np.ceil(rmin))
    rng = np.arange(-n, n + 1)
    mesh = np.meshgrid(*([rng] * grid.dim), indexing="ij")
    offs = np.stack([m.ravel() for m in mesh], axis=1)
    dist = np.linalg.norm(offs * scales[None], axis=1)
    w = (rmin - dist) / rmin
    keep = w > 0
    offs, w = offs[keep], w[keep]
    return offs.astype(np.int64), w / w.sum()


def filter_matrix(grid: Grid, rmin):
    """H with (H rho)_i = sum_k w_k rho_{i+o_k} / N_i, N_i = sum of in-bounds w_k.

    Restates apply_filter_{2D,3D}_parallel (core/_filter.py:78-124) and
    get_filter_weights_{2D,3D} (core/_filter.py:6-40).  Element order is the
    reference's (x slowest).  Returns (H, N).
    """
    offs, w = filter_stencil(grid, rmin)
    ijk = np.stack(grid.element_ijk(), axis=1)
    nel = np.array(grid.nel)
    rows, cols, vals = [], [], []
    for o, wk in zip(offs, w):
        nb = ijk + o[None]
        ok = np.all((nb >= 0) & (nb < nel[None]), axis=1)
        if grid.dim == 2:
            j = nb[:, 0] * nel[1] + nb[:, 1]
        else:
            j = nb[:, 0] * nel[1] * nel[2] + nb[:, 1] * nel[2] + nb[:, 2]
        rows.append(np.where(ok)[0])
        cols.append(j[ok])
        vals.append(np.full(int(ok.sum()), wk))
    rows, cols, vals = map(np.concatenate, (rows, cols, vals))
    N = np.bincount(rows, weights=vals, minlength=grid.n_el)
    H = sp.csr_matrix((vals / N[rows], (rows, cols)), shape=(grid.n_el, grid.n_el))
    return H, N


def filter_apply(H, rho):
    return H @ rho


def filter_apply_T(H, v):
    """(H^T v)_i = sum_k (w_k / N_{i+o_k}) v_{i+o_k} (core/_filter.py:42-76)."""
    return H.T @ v


# --------------------------------------------------------------------------- transfer
def _w1(d):
    return {0: 1.0, 1: 0.5, 2: 0.25, 3: 0.125}[d]


def _boundary_total(dim, nb):
    if dim == 3:
        return {3: 3.375, 2: 4.5, 1: 6.0, 0: 8.0}[nb]
    return {2: 2.25, 1: 3.0, 0: 4.0}[nb]


def restriction_matrix(grid: Grid, variant="gpu"):
    """R: coarse <- fine, full weighting {1, 1/2, 1/4, 1/8} / W_boundary.

    variant "gpu": restriction_{2d,3d}_kernel (core/_templated_cuda.cu:232-364).
    variant "cpu": restriction_matvec_{2d,3d} (core/_mgm.py:10-162); identical in 3-D,
    but the 2-D CPU twin adds the in-range stencil weights to the boundary total a
    second time (core/_mgm.py:159-160).
    """
    cg = grid.coarse()
    cc = cg.node_coords()
    nnf = np.array(grid.nn)
    rows, cols, vals = [], [], []
    offs = np.stack(np.meshgrid(*([np.arange(-1, 2)] * grid.dim), indexing="ij"), -1).reshape(-1, grid.dim)
    nb = np.zeros(cg.n_nodes, dtype=int)
    for d in range(grid.dim):
        nb += ((cc[:, d] == 0) | (cc[:, d] == cg.nn[d] - 1)).astype(int)
    W = np.array([_boundary_total(grid.dim, b) for b in nb])
    if variant == "cpu" and grid.dim == 2:
        extra = np.zeros(cg.n_nodes)
        for o in offs:
            f = 2 * cc + o[None]
            ok = np.all((f >= 0) & (f < nnf[None]), axis=1)
            extra += ok * _w1(int(np.abs(o).sum()))
        W = W + extra
    for o in offs:
        f = 2 * cc + o[None]
        ok = np.all((f >= 0) & (f < nnf[None]), axis=1)
        fid = grid.node_id(*[f[:, q] for q in range(grid.dim)]) if grid.dim == 2 else \
            grid.node_id(f[:, 0], f[:, 1], f[:, 2])
        w = _w1(int(np.abs(o).sum()))
        rows.append(np.where(ok)[0])
        cols.append(fid[ok])
        vals.append(w / W[ok])
    rows, cols, vals = map(np.concatenate, (rows, cols, vals))
    Rn = sp.csr_matrix((vals, (rows, cols)), shape=(cg.n_nodes, grid.n_nodes))
    return sp.kron(Rn, sp.identity(grid.dof), format="csr")


def prolongation_matrix(grid: Grid):
    """P: fine <- coarse, v_f = (1/count) sum over in-range parents of v_c / W_c.

    Restates prolongation_{2d,3d}_kernel (core/_templated_cuda.cu:366-475) and
    prolongation_matvec_{2d,3d} (core/_mgm.py:164-310); equals R^T on even grids.
    """
    cg = grid.coarse()
    fc = grid.node_coords()
    nnc = np.array(cg.nn)
    ccoords = cg.node_coords()
    nb = np.zeros(cg.n_nodes, dtype=int)
    for d in range(grid.dim):
        nb += ((ccoords[:, d] == 0) | (ccoords[:, d] == cg.nn[d] - 1)).astype(int)
    W = np.array([_boundary_total(grid.dim, b) for b in nb])
    base = fc // 2
    odd = fc % 2
    rows, cols, vals, cnt = [], [], [], np.zeros(grid.n_nodes)
    corner = np.stack(np.meshgrid(*([np.arange(2)] * grid.dim), indexing="ij"), -1).reshape(-1, grid.dim)
    entries = []
    for c in corner:
        use = np.all(c[None] <= odd, axis=1)
        p = base + c[None]
        ok = use & np.all(p < nnc[None], axis=1)
        cid = cg.node_id(p[:, 0], p[:, 1]) if grid.dim == 2 else cg.node_id(p[:, 0], p[:, 1], p[:, 2])
        entries.append((np.where(ok)[0], cid[ok]))
        cnt += ok
    for r, c in entries:
        rows.append(r)
        cols.append(c)
        vals.append(1.0 / (cnt[r] * W[c]))
    rows, cols, vals = map(np.concatenate, (rows, cols, vals))
    Pn = sp.csr_matrix((vals, (rows, cols)), shape=(grid.n_nodes, cg.n_nodes))
    return sp.kron(Pn, sp.identity(grid.dof), format="csr")


def galerkin(A_fine, grid: Grid):
    """A_c = R A R^T with the GPU-table restriction on both sides.

    Restates get_restricted_{2d,3d}_l0_nnz_based / _l1p_nnz_based (core/_mgm.py:739-1294,
    core/_mgm_cuda.cu:1-649): level 1 is built from K0, E and the BC mask with
    constrained fine DOFs contributing the identity, i.e. from the constrained K.
    """
    R = restriction_matrix(grid, "gpu")
    A = (R @ A_fine @ R.T).tocsr()
    A.sum_duplicates()
    return A
