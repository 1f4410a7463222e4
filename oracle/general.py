"""Unstructured meshes: stiffness operator and density filter, FP64 (oracle; test infrastructure).

Restates, for meshes of any element kind (T3, Q4, Tet4, hex8, mixed):

  mesh bookkeeping   GeneralMesh (geom/_mesh.py:146-225): element sizes, flat connectivity,
                     centroids (mean of the element's nodes), uniform = one element size
  operator           UniformStiffnessKernel / GeneralStiffnessKernel (kernels/_processors.py:
                     157-395, node-basis kernels core/_ops.py): K(rho) u = sum_e rho_e K_e u_e
                     with constrained rows and columns replaced by the identity
  diagonal           diag K(rho), 1 on constrained DOFs
  dk                 dk_e = -u_e^T K_e u_e (process_dk_full / process_dk_general)
  filter             filter_kernel_2D/3D_general (core/_filter.py:126-182): neighbours within
                     r_min of each centroid (closed ball), w = (r_min - d) / r_min normalised
                     per row; H rho and H^T rho

The element matrices K_e are inputs here (the product computes them with
edge_to_b200.physics, pinned to the reference's auto_stiffness separately).  Pinned against
tests/golden/general.npz, made by running the reference classes.
"""
import numpy as np
import scipy.sparse as sp
from scipy.spatial import cKDTree


def connectivity(sizes, flat):
    """List of per-element node arrays from element sizes and the flat connectivity."""
    ptr = np.concatenate([[0], np.cumsum(sizes)])
    return [np.asarray(flat[ptr[e]:ptr[e + 1]]) for e in range(len(sizes))]


def element_matrices(Kflat, sizes, dof):
    """Per-element K_e (nk x nk, nk = size * dof) from the flat row-major storage."""
    out, o = [], 0
    for s in sizes:
        nk = int(s) * dof
        out.append(np.asarray(Kflat[o:o + nk * nk]).reshape(nk, nk))
        o += nk * nk
    return out


def centroids(nodes, conn):
    return np.stack([np.asarray(nodes)[c].mean(axis=0) for c in conn])


def _dofs(c, dof):
    return (np.asarray(c)[:, None] * dof + np.arange(dof)[None, :]).reshape(-1)


def assemble(n_dof, dof, conn, Ks, rho, cons=None):
    rows, cols, vals = [], [], []
    for c, K, r in zip(conn, Ks, rho):
        d = _dofs(c, dof)
        rows.append(np.repeat(d, d.size))
        cols.append(np.tile(d, d.size))
        vals.append(r * K.reshape(-1))
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    if cons is not None and len(cons):
        mask = np.zeros(n_dof, dtype=bool)
        mask[cons] = True
        keep = ~(mask[rows] | mask[cols])
        rows = np.concatenate([rows[keep], np.where(mask)[0]])
        cols = np.concatenate([cols[keep], np.where(mask)[0]])
        vals = np.concatenate([vals[keep], np.ones(int(mask.sum()))])
    K = sp.coo_matrix((vals, (rows, cols)), shape=(n_dof, n_dof)).tocsr()
    K.sum_duplicates()
    return K


def dk(conn, Ks, U, dof):
    U = np.asarray(U)
    return np.array([-U[_dofs(c, dof)] @ K @ U[_dofs(c, dof)] for c, K in zip(conn, Ks)])


def filter_matrix(cent, r_min):
    """Row-normalised cone filter over element centroids (closed ball of radius r_min)."""
    cent = np.asarray(cent, dtype=np.float64)
    tree = cKDTree(cent)
    rows, cols, vals = [], [], []
    for i, nb in enumerate(tree.query_ball_point(cent, r_min)):
        nb = np.asarray(sorted(nb))
        w = (r_min - np.linalg.norm(cent[nb] - cent[i], axis=-1)) / r_min
        rows.append(np.full(nb.size, i))
        cols.append(nb)
        vals.append(w / w.sum())
    n = cent.shape[0]
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
