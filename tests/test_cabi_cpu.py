"""Host-side checks that need no GPU: the C-ABI library loads and exports every symbol
declared in include/edge_b200.h, and the package's host code (meshes, element physics,
filter stencils) matches the reference fixtures and the oracle."""
import os
import re

import numpy as np

from oracle import elements, ops
from oracle.grid import Grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "edge_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(edge_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    from edge_to_b200 import _lib
    lib = _lib.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.exported_symbols()) | {"edge_version"}
    assert lib.edge_version() >= 1


def test_error_reporting_without_gpu():
    """Argument checks run before any device work and map to ValueError."""
    import ctypes
    import pytest
    from edge_to_b200 import _lib
    h = ctypes.c_void_p()
    K0 = np.zeros(64)
    with pytest.raises(ValueError):
        _lib.call("edge_problem_create", 4, _lib.int_array([2, 2, 1]), K0.ctypes.data_as(_lib.c_double_p), 0,
                  ctypes.byref(h))
    with pytest.raises(ValueError):
        _lib.call("edge_problem_create", 2, _lib.int_array([0, 2, 1]), K0.ctypes.data_as(_lib.c_double_p), 0,
                  ctypes.byref(h))


def test_physics_matches_reference_kat(golden):
    from edge_to_b200 import physics
    kat = golden("kat_stiffness.npz")
    q = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    h = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    for nu in (0.3, 0.33):
        K, D, B, A = physics.auto_stiffness(q, 1.0, nu)
        assert np.abs(K - kat[f"q4_nu{nu}"]).max() < 1e-15
        assert A == float(kat[f"q4_nu{nu}_area"])
        K, D, B, V = physics.auto_stiffness(h, 1.0, nu)
        assert np.abs(K - kat[f"hex8_nu{nu}"]).max() < 1e-15
        assert V == float(kat[f"hex8_nu{nu}_volume"])
    K = physics.auto_stiffness(h * np.array([0.5, 0.25, 1.0]), 1.0, 0.3)[0]
    assert np.abs(K - kat["hex8_box_0.5x0.25x1_nu0.3"]).max() < 1e-15


def test_mesh_numbering_matches_oracle():
    import edge_to_b200 as eb
    m2 = eb.CuStructuredMesh2D(5, 3, 5.0, 3.0)
    g2 = Grid((5, 3))
    np.testing.assert_array_equal(m2.elements, g2.connectivity())
    np.testing.assert_array_equal(m2.nodes, g2.node_coords().astype(float))
    m3 = eb.CuStructuredMesh3D(4, 3, 2, 4.0, 3.0, 2.0)
    g3 = Grid((4, 3, 2))
    np.testing.assert_array_equal(m3.elements, g3.connectivity())
    np.testing.assert_array_equal(m3.nodes[:, [0, 1, 2]], g3.node_coords().astype(float))
    assert m3.A_single[0] == elements.element_measure((1, 1, 1))


def test_filter_stencil_matches_oracle():
    from edge_to_b200.filters import cone_stencil
    for dim, h, r in ((2, (1, 1), 1.5), (2, (0.5, 0.25), 1.5), (3, (1, 1, 1), 2.0), (3, (1, 1, 1), 3.0)):
        o1, w1 = cone_stencil(dim, h, r)
        o2, w2 = ops.filter_stencil(Grid((4,) * dim, h), r)
        np.testing.assert_array_equal(o1, o2)
        assert np.abs(w1 - w2).max() < 1e-16
