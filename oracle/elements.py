"""Element stiffness matrices for axis-aligned box elements (oracle; test infrastructure).

Restates physics/_linelas.py:195-309 (``quadrilateral_element_stiffness``, plane stress,
2x2 Gauss, thickness t) and physics/_linelas.py:338-447 (``hexahedron_element_stiffness``,
2x2x2 Gauss) for the element shapes the structured meshes produce: a box of edge lengths
(hx, hy[, hz]) with the reference's local node order

  Q4   : (0,0) (1,0) (1,1) (0,1)
  hex8 : (0,0,0) (1,0,0) (1,1,0) (0,1,0) (0,0,1) (1,0,1) (1,1,1) (0,1,1)

DOFs are interleaved per node: [u_x, u_y(, u_z)] (core/_geom.py:20-25, 48-57).
"""
import numpy as np

Q4_CORNERS = np.array([[0, 0], [1, 0], [1, 1], [0, 1]])
HEX8_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
_GP = np.array([-1.0, 1.0]) / np.sqrt(3.0)


def plane_stress_D(E, nu):
    c = E / (1.0 - nu * nu)
    return c * np.array([[1.0, nu, 0.0], [nu, 1.0, 0.0], [0.0, 0.0, (1.0 - nu) / 2.0]])


def iso3d_D(E, nu):
    c = E / ((1.0 + nu) * (1.0 - 2.0 * nu))
    g = (1.0 - 2.0 * nu) / 2.0
    D = np.zeros((6, 6))
    D[:3, :3] = nu
    np.fill_diagonal(D[:3, :3], 1.0 - nu)
    D[3, 3] = D[4, 4] = D[5, 5] = g
    return c * D


def q4_stiffness(hx=1.0, hy=1.0, E=1.0, nu=0.33, t=1.0):
    """8x8 plane-stress stiffness of an hx-by-hy rectangle (physics/_linelas.py:195-309)."""
    D = plane_stress_D(E, nu)
    sgn = 2 * Q4_CORNERS - 1          # corner signs in the [-1,1]^2 parent element
    K = np.zeros((8, 8))
    for r in _GP:
        for s in _GP:
            dNdr = 0.25 * sgn[:, 0] * (1 + sgn[:, 1] * s)
            dNds = 0.25 * sgn[:, 1] * (1 + sgn[:, 0] * r)
            dNdx = dNdr * 2.0 / hx
            dNdy = dNds * 2.0 / hy
            B = np.zeros((3, 8))
            B[0, 0::2] = dNdx
            B[1, 1::2] = dNdy
            B[2, 0::2] = dNdy
            B[2, 1::2] = dNdx
            K += B.T @ D @ B * (t * hx * hy / 4.0)
    return K


def hex8_stiffness(hx=1.0, hy=1.0, hz=1.0, E=1.0, nu=0.33):
    """24x24 stiffness of an hx-by-hy-by-hz box (physics/_linelas.py:338-447)."""
    D = iso3d_D(E, nu)
    sgn = 2 * HEX8_CORNERS - 1
    h = np.array([hx, hy, hz])
    K = np.zeros((24, 24))
    detJ = hx * hy * hz / 8.0
    for a in _GP:
        for b in _GP:
            for c in _GP:
                xi = np.array([a, b, c])
                dN = np.zeros((3, 8))
                for d in range(3):
                    o1, o2 = [q for q in range(3) if q != d]
                    dN[d] = 0.125 * sgn[:, d] * (1 + sgn[:, o1] * xi[o1]) * (1 + sgn[:, o2] * xi[o2])
                    dN[d] *= 2.0 / h[d]
                B = np.zeros((6, 24))
                for d in range(3):
                    B[d, d::3] = dN[d]
                B[3, 0::3] = dN[1]
                B[3, 1::3] = dN[0]
                B[4, 1::3] = dN[2]
                B[4, 2::3] = dN[1]
                B[5, 0::3] = dN[2]
                B[5, 2::3] = dN[0]
                K += B.T @ D @ B * detJ
    return K


_HEX_TETS = ((0, 1, 3, 7), (1, 2, 3, 7), (0, 1, 7, 4), (1, 2, 7, 6), (1, 5, 7, 4), (1, 5, 6, 7))


def _tri_area(p):
    return (p[0, 0] * (p[1, 1] - p[2, 1]) + p[1, 0] * (p[2, 1] - p[0, 1]) + p[2, 0] * (p[0, 1] - p[1, 1])) / 2


def element_measure(h):
    """Area (2-D) or volume (3-D) of the box element exactly as the reference computes ``A_single``.

    The reference sums two shoelace triangles (physics/_linelas.py:312-336) or six
    determinant-based tetrahedra (physics/_linelas.py:450-474, 179-192) over element 0's
    corner coordinates, which come from np.linspace; for a unit cube that gives
    0.9999999999999999, and the OC bisection sees that value.
    """
    h = [float(x) for x in h]
    if len(h) == 2:
        p = Q4_CORNERS * np.array([np.linspace(0, h[0], 2)[1], np.linspace(0, h[1], 2)[1]])
        return float(_tri_area(p[[0, 1, 2]]) + _tri_area(p[[0, 2, 3]]))
    p = HEX8_CORNERS * np.array(h)
    V = 0.0
    for t in _HEX_TETS:
        V += np.linalg.det(np.concatenate([np.ones((4, 1)), p[list(t)]], -1)) / 6
    return float(V)
