"""Host-side unstructured-mesh code of this package (CPU): element routines and the general
mesh bookkeeping, against fixtures made by running the reference's GeneralMesh and
auto_stiffness (tests/golden/general.npz)."""
import numpy as np

from oracle import general

GENERAL_TAGS = ("tri", "mixed", "tet", "hex")


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_general_element_matrices_product(golden):
    """This package's element routines (edge_to_b200.physics.auto_stiffness: T3 and Tet4 via
    the simplex coordinate matrix, isoparametric Q4 / hex8) reproduce the reference's element
    matrices and measures on the unstructured fixture meshes, including negatively oriented
    tetrahedra."""
    from edge_to_b200 import physics
    z = golden("general.npz")
    for tag in GENERAL_TAGS:
        sizes, flat, dof = z[f"{tag}_sizes"], z[f"{tag}_flat"], int(z[f"{tag}_dof"])
        conn = general.connectivity(sizes, flat)
        Ks = general.element_matrices(z[f"{tag}_Kflat"], sizes, dof)
        nodes = z[f"{tag}_nodes"]
        for e, c in enumerate(conn):
            K, D, B, A = physics.auto_stiffness(nodes[c], 1.0, 0.3)
            assert rel(K, Ks[e]) < 1e-13, (tag, e)
            assert abs(A - z[f"{tag}_As"][e]) <= 1e-14 * max(1.0, abs(A)), (tag, e)
        assert abs(sum(z[f"{tag}_As"]) - float(z[f"{tag}_volume"])) < 1e-12


def test_general_mesh_bookkeeping(golden):
    """CuGeneralMesh builds the reference GeneralMesh's arrays on the fixture meshes (sizes,
    flat connectivity, centroids, element matrices, measures, dof, volume), and removes an
    unused node with a consistent renumbering of both connectivity forms."""
    import edge_to_b200 as eb
    z = golden("general.npz")
    st = lambda x: eb.auto_stiffness(x, 1.0, 0.3)  # noqa: E731
    for tag in GENERAL_TAGS:
        sizes, flat = z[f"{tag}_sizes"], z[f"{tag}_flat"]
        conn = general.connectivity(sizes, flat)
        nodes = z[f"{tag}_nodes"]
        m = eb.CuGeneralMesh(nodes, conn, stiffness=st)
        assert m.is_uniform == bool(z[f"{tag}_uniform"]) and m.dof == int(z[f"{tag}_dof"])
        assert (m.element_sizes == sizes).all() and (m.elements_flat == flat).all()
        assert (m.elements_ptr == np.concatenate([[0], np.cumsum(sizes)])).all()
        assert rel(m.centeroids, z[f"{tag}_centroids"]) < 1e-14
        assert rel(m.As.reshape(-1), z[f"{tag}_As"]) < 1e-14
        assert abs(m.volume - float(z[f"{tag}_volume"])) < 1e-12
        Kflat = m.Ks.reshape(-1) if m.is_uniform else m.K_flat
        assert rel(Kflat, z[f"{tag}_Kflat"]) < 1e-13
    # an unused node is dropped; nodes[elements] keeps every element's coordinates
    nodes = z["mixed_nodes"]
    conn = general.connectivity(z["mixed_sizes"], z["mixed_flat"])
    extra = np.vstack([nodes[:5], [[100.0, 100.0]], nodes[5:]])
    conn2 = [np.where(c >= 5, c + 1, c) for c in conn]
    m = eb.CuGeneralMesh(extra, conn2, stiffness=st)
    assert m.nodes.shape[0] == nodes.shape[0]
    for e, c in enumerate(conn):
        assert np.array_equal(m.nodes[m.elements[e]], nodes[c])
    assert np.array_equal(m.elements_flat, z["mixed_flat"])
