"""Element physics: T3, Q4 (plane stress / plane strain), Tet4 and hex8.

Host-side (numpy) set-up code with the reference's signatures
(physics/_linelas.py:1-547): ``triangle_element_stiffness``,
``tetrahedron_element_stiffness``, ``quadrilateral_element_stiffness``,
``hexahedron_element_stiffness``, their area/volume helpers and ``auto_stiffness``.
Q4 / hex8 are isoparametric with full 2x2(x2) Gauss integration and return the Gauss-point
average of B, as in the reference; T3 / Tet4 are constant-strain simplices whose shape
function gradients are read off the inverse of the coordinate matrix [1 x y (z)].
"""
import numpy as np

_G = np.array([-1.0, 1.0]) / np.sqrt(3.0)
_Q4_XI = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=np.float64)
_HEX_XI = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
# decomposition of the hexahedron into six tetrahedra used for its volume
_HEX_TETS = ((0, 1, 3, 7), (1, 2, 3, 7), (0, 1, 7, 4), (1, 2, 7, 6), (1, 5, 7, 4), (1, 5, 6, 7))


def _tri_signed_area(p):
    return (p[0, 0] * (p[1, 1] - p[2, 1]) + p[1, 0] * (p[2, 1] - p[0, 1]) + p[2, 0] * (p[0, 1] - p[1, 1])) / 2


def quadrilateral_element_area(x0s):
    x0s = np.asarray(x0s, dtype=np.float64)
    return _tri_signed_area(x0s[[0, 1, 2]]) + _tri_signed_area(x0s[[0, 2, 3]])


def tetrahedron_element_volume(x0s):
    x0s = np.asarray(x0s, dtype=np.float64)
    return np.linalg.det(np.concatenate([np.ones((4, 1)), x0s], -1)) / 6


def hexahedron_element_volume(x0s):
    x0s = np.asarray(x0s, dtype=np.float64)
    V = 0.0
    for t in _HEX_TETS:
        V += tetrahedron_element_volume(x0s[list(t)])
    return V


def _plane_D(E, nu, e_type):
    if e_type == 0:
        c = E / (1 - nu * nu)
        return c * np.array([[1, nu, 0], [nu, 1, 0], [0, 0, (1 - nu) / 2]])
    c = E / ((1 + nu) * (1 - 2 * nu))
    return c * np.array([[1 - nu, nu, 0], [nu, 1 - nu, 0], [0, 0, (1 - 2 * nu) / 2]])


def _iso_D(E, nu):
    c = E / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6))
    D[:3, :3] = nu
    D[0, 0] = D[1, 1] = D[2, 2] = 1 - nu
    D[3, 3] = D[4, 4] = D[5, 5] = (1 - 2 * nu) / 2
    return c * D


def triangle_element_area(x0s):
    return _tri_signed_area(np.asarray(x0s, dtype=np.float64))


def _simplex_gradients(x0s):
    """Gradients of the linear shape functions of a simplex (rows: nodes, columns: x, y(, z)):
    N_i(x) = [1, x] . inv(P)[:, i] with P = [1 | x0s]."""
    P = np.concatenate([np.ones((x0s.shape[0], 1)), x0s], -1)
    return np.linalg.inv(P)[1:].T


def triangle_element_stiffness(x0s, E=1.0, NU=0.33, e_type=0, t=1.0):
    """(K 6x6, D 3x3, B 3x6) of a constant-strain triangle (physics/_linelas.py:3-50)."""
    x0s = np.asarray(x0s, dtype=np.float64)
    A = _tri_signed_area(x0s)
    if A < 0:
        raise Exception("Node Order Is Not Correct")
    g = _simplex_gradients(x0s)
    B = np.zeros((3, 6))
    B[0, 0::2] = g[:, 0]
    B[1, 1::2] = g[:, 1]
    B[2, 0::2] = g[:, 1]
    B[2, 1::2] = g[:, 0]
    D = _plane_D(E, NU, e_type)
    return t * A * B.T @ D @ B, D, B


def tetrahedron_element_stiffness(x0s, E=1.0, NU=0.33):
    """(K 12x12, D 6x6, B 6x12) of a linear tetrahedron (physics/_linelas.py:70-176); strain
    order xx, yy, zz, xy, yz, zx."""
    x0s = np.asarray(x0s, dtype=np.float64)
    V = tetrahedron_element_volume(x0s)
    if V < 0:
        raise Exception("Node Order Is Not Correct")
    g = _simplex_gradients(x0s)
    B = np.zeros((6, 12))
    for d in range(3):
        B[d, d::3] = g[:, d]
    B[3, 0::3], B[3, 1::3] = g[:, 1], g[:, 0]
    B[4, 1::3], B[4, 2::3] = g[:, 2], g[:, 1]
    B[5, 0::3], B[5, 2::3] = g[:, 2], g[:, 0]
    D = _iso_D(E, NU)
    return V * B.T @ D @ B, D, B


def _reordered(fn, x0s, order, dof, E, Nu):
    """Element matrices of a clockwise (negatively oriented) element: computed on the nodes
    in `order` and permuted back to the given node order."""
    K, D, B = fn(x0s[order], E, Nu)
    idx = (np.asarray(order)[:, None] * dof + np.arange(dof)[None, :]).reshape(-1)
    inv = np.empty_like(idx)
    inv[idx] = np.arange(idx.size)
    return K[inv][:, inv], D, B[:, inv]


def quadrilateral_element_stiffness(x0s, E=1.0, NU=0.33, e_type=0, t=1.0):
    """(K 8x8, D 3x3, B 3x8) of a bilinear quadrilateral (physics/_linelas.py:195-309)."""
    x0s = np.asarray(x0s, dtype=np.float64)
    if quadrilateral_element_area(x0s) < 0:
        raise Exception("Node Order Is Not Correct")
    D = _plane_D(E, NU, e_type)
    K = np.zeros((8, 8))
    Bavg = np.zeros((3, 8))
    for r in _G:
        for s in _G:
            dN = 0.25 * np.stack([_Q4_XI[:, 0] * (1 + _Q4_XI[:, 1] * s),
                                  _Q4_XI[:, 1] * (1 + _Q4_XI[:, 0] * r)])  # (2, 4) d/d(r,s)
            J = dN @ x0s
            dNx = np.linalg.solve(J, dN)
            B = np.zeros((3, 8))
            B[0, 0::2] = dNx[0]
            B[1, 1::2] = dNx[1]
            B[2, 0::2] = dNx[1]
            B[2, 1::2] = dNx[0]
            K += B.T @ D @ B * (t * np.linalg.det(J))
            Bavg += B / 4
    return K, D, Bavg


def hexahedron_element_stiffness(x0s, E=1.0, nu=0.33):
    """(K 24x24, D 6x6, B 6x24) of a trilinear hexahedron (physics/_linelas.py:338-447)."""
    x0s = np.asarray(x0s, dtype=np.float64)
    if hexahedron_element_volume(x0s) < 0:
        raise Exception("Node Order Is Not Correct")
    D = _iso_D(E, nu)
    K = np.zeros((24, 24))
    Bavg = np.zeros((6, 24))
    xi = _HEX_XI
    for a in _G:
        for b in _G:
            for c in _G:
                p = np.array([a, b, c])
                dN = np.empty((3, 8))
                for d in range(3):
                    o = [q for q in range(3) if q != d]
                    dN[d] = 0.125 * xi[:, d] * (1 + xi[:, o[0]] * p[o[0]]) * (1 + xi[:, o[1]] * p[o[1]])
                J = dN @ x0s
                dNx = np.linalg.solve(J, dN)
                B = np.zeros((6, 24))
                for d in range(3):
                    B[d, d::3] = dNx[d]
                B[3, 0::3], B[3, 1::3] = dNx[1], dNx[0]
                B[4, 1::3], B[4, 2::3] = dNx[2], dNx[1]
                B[5, 0::3], B[5, 2::3] = dNx[2], dNx[0]
                K += B.T @ D @ B * np.linalg.det(J)
                Bavg += B / 8
    return K, D, Bavg


def auto_stiffness(x0s, E, Nu):
    """(K, D, B, area|volume) of a T3, Tet4, Q4 or hex8 element chosen by its node count and
    dimension (physics/_linelas.py:477-547).  A negatively oriented triangle or tetrahedron
    is computed in the reversed (T3) or 0,1,3,2 (Tet4) node order and permuted back, with a
    positive measure; Q4 and hex8 must be positively oriented (an Exception otherwise, as in
    the reference, whose final call uses the given order)."""
    x0s = np.asarray(x0s, dtype=np.float64)
    if x0s.shape[0] == 3:
        A = _tri_signed_area(x0s)
        if A < 0:
            K, D, B = _reordered(triangle_element_stiffness, x0s, [2, 1, 0], 2, E, Nu)
            return K, D, B, -A
        K, D, B = triangle_element_stiffness(x0s, E, Nu)
        return K, D, B, A
    if x0s.shape[0] == 4 and x0s.shape[1] == 3:
        V = tetrahedron_element_volume(x0s)
        if V < 0:
            K, D, B = _reordered(tetrahedron_element_stiffness, x0s, [0, 1, 3, 2], 3, E, Nu)
            return K, D, B, -V
        K, D, B = tetrahedron_element_stiffness(x0s, E, Nu)
        return K, D, B, V
    if x0s.shape[0] == 4 and x0s.shape[1] == 2:
        A = quadrilateral_element_area(x0s)
        if A < 0:
            A = quadrilateral_element_area(x0s[::-1])
        K, D, B = quadrilateral_element_stiffness(x0s, E, Nu)
        return K, D, B, A
    if x0s.shape[0] == 8:
        A = hexahedron_element_volume(x0s)
        if A < 0:
            A = hexahedron_element_volume(x0s[[4, 5, 6, 7, 0, 1, 2, 3]])
        K, D, B = hexahedron_element_stiffness(x0s, E, Nu)
        return K, D, B, A
    raise Exception("Element Type Not Supported")
