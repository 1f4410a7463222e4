"""Structured-grid numbering of the reference (oracle; test infrastructure).

Restates core/_geom.py:4-59 and geom/_mesh.py:19-78:

  2-D  node (i, j)    -> j*(nelx+1) + i                 (x fastest)
       element (i, j) -> i*nely + j                     (y fastest)
  3-D  node (i, j, k) -> j*(nx*nz) + i*nz + k           (z fastest, then x, then y)
       element (i,j,k)-> i*nely*nelz + j*nelz + k       (z fastest, then y, then x)

with nx = nelx+1 etc.  Element e connects the corners listed in oracle.elements.
"""
import numpy as np

from .elements import HEX8_CORNERS, Q4_CORNERS


class Grid:
    def __init__(self, nel, h=None):
        self.nel = tuple(int(n) for n in nel)
        self.dim = len(self.nel)
        assert self.dim in (2, 3)
        self.dof = self.dim
        self.nn = tuple(n + 1 for n in self.nel)
        self.n_nodes = int(np.prod(self.nn))
        self.n_el = int(np.prod(self.nel))
        self.n_dof = self.n_nodes * self.dof
        self.h = tuple(float(x) for x in (h if h is not None else (1.0,) * self.dim))

    def node_id(self, i, j, k=None):
        if self.dim == 2:
            return j * self.nn[0] + i
        return j * (self.nn[0] * self.nn[2]) + i * self.nn[2] + k

    def element_ijk(self):
        """(i, j[, k]) of every element in reference element order."""
        if self.dim == 2:
            e = np.arange(self.n_el)
            return e // self.nel[1], e % self.nel[1]
        e = np.arange(self.n_el)
        nyz = self.nel[1] * self.nel[2]
        return e // nyz, (e % nyz) // self.nel[2], e % self.nel[2]

    def connectivity(self):
        """(n_el, 4|8) node ids per element, corners in reference local order."""
        if self.dim == 2:
            i, j = self.element_ijk()
            c = Q4_CORNERS
            return np.stack([self.node_id(i + c[a, 0], j + c[a, 1]) for a in range(4)], axis=1)
        i, j, k = self.element_ijk()
        c = HEX8_CORNERS
        return np.stack([self.node_id(i + c[a, 0], j + c[a, 1], k + c[a, 2]) for a in range(8)], axis=1)

    def dof_map(self):
        conn = self.connectivity()
        d = self.dof
        return (conn[:, :, None] * d + np.arange(d)[None, None, :]).reshape(conn.shape[0], -1)

    def node_coords(self):
        """(n_nodes, dim) integer lattice coordinates (i, j[, k]) of every node."""
        if self.dim == 2:
            n = np.arange(self.n_nodes)
            return np.stack([n % self.nn[0], n // self.nn[0]], axis=1)
        n = np.arange(self.n_nodes)
        nxz = self.nn[0] * self.nn[2]
        return np.stack([(n % nxz) // self.nn[2], n // nxz, n % self.nn[2]], axis=1)

    def coarse(self):
        return Grid(tuple(n // 2 for n in self.nel), tuple(2 * x for x in self.h))
