"""Structured Q4 / hex8 meshes with the reference's numbering (geom/_mesh.py:81-143), and
general (unstructured) meshes of T3 / Q4 / Tet4 / hex8 elements (geom/_mesh.py:146-251).

Node and element arrays follow core/_geom.py:4-98 (2-D node j*(nelx+1)+i, element
i*nely+j; 3-D node j*nx*nz + i*nz + k, element i*nely*nelz + j*nelz + k).  They are
host numpy arrays, built on first access: the solver never reads them, since every
kernel indexes the grid implicitly.  K_single, D_single, B_single and A_single come from
the ``stiffness`` callable applied to element 0, exactly as in the reference.
"""
import numpy as np

from .physics import auto_stiffness


def _default_stiffness(x0):
    return auto_stiffness(x0, 1.0, 0.33)


class StructuredMesh:
    pass


class _StructuredBase(StructuredMesh):
    def _finish(self, stiffness, dtype):
        x0 = self._element0_coords()
        K, D, B, A = stiffness(x0)
        self.K_single = np.asarray(K, dtype=dtype)
        self.D_single = np.asarray(D, dtype=dtype)
        self.B_single = np.asarray(B, dtype=dtype)
        self.A_single = np.array([A], dtype=dtype)
        self.As = self.A_single
        self.volume = self.A_single[0] * float(np.prod(self.nel))
        self.elements_size = 2 ** len(self.nel)
        self.dof = int(self.K_single.shape[0] / self.elements_size)
        self.dtype = dtype
        self._nodes = None
        self._elements = None

    @property
    def n_nodes(self):
        return int(np.prod(self.nel + 1))

    @property
    def n_elements(self):
        return int(np.prod(self.nel))

    @property
    def nodes(self):
        if self._nodes is None:
            self._nodes = self._make_nodes()
        return self._nodes

    @property
    def elements(self):
        if self._elements is None:
            self._elements = self._make_elements()
        return self._elements


class CuStructuredMesh2D(_StructuredBase):
    def __init__(self, nx, ny, lx, ly, dtype=np.float64, stiffness=_default_stiffness):
        super().__init__()
        self.nelx, self.nely = int(nx), int(ny)
        self.lx, self.ly = lx, ly
        self.nel = np.array([nx, ny], dtype=np.int32)
        self.dim = np.array([lx, ly], dtype=dtype)
        self.dx, self.dy = lx / nx, ly / ny
        self._finish(stiffness, dtype)

    def _axes(self):
        return (np.linspace(0, self.lx, self.nelx + 1, dtype=self.dtype if hasattr(self, "dtype") else np.float64),
                np.linspace(0, self.ly, self.nely + 1, dtype=self.dtype if hasattr(self, "dtype") else np.float64))

    def _element0_coords(self):
        x, y = self._axes()
        return np.array([[x[0], y[0]], [x[1], y[0]], [x[1], y[1]], [x[0], y[1]]], dtype=np.float64)

    def _make_nodes(self):
        x, y = self._axes()
        xx, yy = np.meshgrid(x, y)
        return np.stack([xx.ravel(), yy.ravel()], axis=-1)

    def _make_elements(self):
        nx = self.nelx + 1
        e = np.arange(self.nelx * self.nely)
        i, j = e // self.nely, e % self.nely
        return np.stack([j * nx + i, j * nx + i + 1, (j + 1) * nx + i + 1, (j + 1) * nx + i], axis=1).astype(np.int32)


class CuStructuredMesh3D(_StructuredBase):
    def __init__(self, nx, ny, nz, lx, ly, lz, dtype=np.float64, stiffness=_default_stiffness):
        super().__init__()
        self.nelx, self.nely, self.nelz = int(nx), int(ny), int(nz)
        self.lx, self.ly, self.lz = lx, ly, lz
        self.nel = np.array([nx, ny, nz], dtype=np.int32)
        self.dim = np.array([lx, ly, lz], dtype=dtype)
        self.dx, self.dy, self.dz = lx / nx, ly / ny, lz / nz
        self._finish(stiffness, dtype)

    def _axes(self):
        dt = self.dtype if hasattr(self, "dtype") else np.float64
        return (np.linspace(0, self.lx, self.nelx + 1, dtype=dt), np.linspace(0, self.ly, self.nely + 1, dtype=dt),
                np.linspace(0, self.lz, self.nelz + 1, dtype=dt))

    def _element0_coords(self):
        x, y, z = self._axes()
        c = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
        return np.stack([x[c[:, 0]], y[c[:, 1]], z[c[:, 2]]], axis=1).astype(np.float64)

    def _make_nodes(self):
        x, y, z = self._axes()
        xx, yy, zz = np.meshgrid(x, y, z)
        return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=-1)

    def _make_elements(self):
        nx, nz = self.nelx + 1, self.nelz + 1
        e = np.arange(self.nelx * self.nely * self.nelz)
        nyz = self.nely * self.nelz
        i, j, k = e // nyz, (e % nyz) // self.nelz, e % self.nelz
        base = nz * i + nz * nx * j + k
        off = [0, nz, nz + nz * nx, nz * nx]
        cols = [base + o for o in off] + [base + o + 1 for o in off]
        return np.stack(cols, axis=1).astype(np.int32)


# The CPU-named classes of the reference map to the same GPU meshes here.
StructuredMesh2D = CuStructuredMesh2D
StructuredMesh3D = CuStructuredMesh3D


class CuGeneralMesh:
    """Unstructured mesh, drop-in for GeneralMesh / CuGeneralMesh (geom/_mesh.py:146-251).

    ``nodes`` (n x dim) and ``elements`` (an n_el x k integer array, or a sequence of node
    lists of mixed sizes).  Builds the reference's bookkeeping: ``element_sizes``,
    ``elements_flat``, ``elements_ptr``, ``centeroids`` (sic, the reference's name: the mean of
    each element's nodes), ``is_uniform`` (one element size), the per-element matrices from
    ``stiffness`` (``Ks``, ``Ds``, ``Bs`` stacked when uniform; ``K_flat``/``D_flat``/``B_flat``
    with ``K_ptr``/``D_ptr``/``B_ptr`` otherwise), ``As`` (n_el x 1), ``dof`` and ``volume``.
    Nodes that no element uses are removed and the connectivity renumbered; the reference
    renumbers only ``elements_flat`` and keeps reading ``elements`` with the old numbers, so
    here ``elements`` is renumbered as well.  Arrays are host numpy arrays: the device copies
    belong to the stiffness kernel and filter that consume the mesh.
    """

    def __init__(self, nodes, elements, dtype=np.float64, stiffness=_default_stiffness):
        nodes = np.asarray(nodes, dtype=dtype)
        conn = [np.asarray(e, dtype=np.int64).reshape(-1) for e in elements]
        if not conn:
            raise ValueError("mesh has no elements")
        sizes = np.array([c.size for c in conn], dtype=np.int32)
        self.is_uniform = bool((sizes == sizes[0]).all())
        self.centeroids = np.stack([nodes[c].mean(axis=0) for c in conn]).astype(dtype)
        flat = np.concatenate(conn)
        used = np.unique(flat)
        if used.size != nodes.shape[0]:
            remap = -np.ones(nodes.shape[0], dtype=np.int64)
            remap[used] = np.arange(used.size)
            conn = [remap[c] for c in conn]
            flat = remap[flat]
            nodes = nodes[used]
        self.nodes = nodes
        self.element_sizes = sizes
        self.elements_flat = flat.astype(np.int32)
        self.elements_ptr = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
        mats = [stiffness(nodes[c]) for c in conn]
        self.As = np.array([[m[3]] for m in mats], dtype=dtype)
        if self.is_uniform:
            self.elements = np.stack(conn).astype(np.int32)
            self.Ks = np.stack([m[0] for m in mats]).astype(dtype)
            self.Ds = np.stack([m[1] for m in mats]).astype(dtype)
            self.Bs = np.stack([m[2] for m in mats]).astype(dtype)
            self.dof = int(self.Ks.shape[1] // sizes[0])
        else:
            self.elements = conn
            for name, i in (("K", 0), ("D", 1), ("B", 2)):
                arrs = [np.asarray(m[i], dtype=dtype).reshape(-1) for m in mats]
                setattr(self, f"{name}_flat", np.concatenate(arrs))
                setattr(self, f"{name}_ptr", np.concatenate([[0], np.cumsum([a.size for a in arrs])]).astype(np.int32))
            self.dof = int(np.asarray(mats[-1][0]).shape[0] // sizes[-1])
        self.volume = float(np.sum(self.As))
        self.dtype = dtype

    @property
    def n_elements(self):
        return len(self.element_sizes)


GeneralMesh = CuGeneralMesh
