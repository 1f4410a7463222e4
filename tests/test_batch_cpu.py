"""Host logic of the batching configuration's problem generator (no GPU needed)."""
import numpy as np

from edge_to_b200 import batch


def test_random_specs_follow_the_configuration():
    specs = [batch.random_spec(i, seed=0) for i in range(64)]
    for sp in specs:
        nelx, nely = sp["nelx"], sp["nely"]
        assert 64 <= nelx <= 512 and 32 <= nely <= 256
        assert 0.2 <= sp["vf"] <= 0.6 and 1.5 <= sp["rmin"] <= 3.0
        assert 1 <= len(sp["segments"]) <= 2
        for edge, start, n in sp["segments"]:
            length = nely if edge < 2 else nelx
            assert 0 <= start and start + n <= length
            assert round(0.1 * length) - 1 <= n <= round(0.5 * length) + 1
        assert 1 <= len(sp["load_nodes"]) <= 4
        assert np.allclose(np.linalg.norm(sp["forces"], axis=1), 1.0)
        # loads sit on free boundary nodes; clamped nodes lie on the boundary
        assert not np.intersect1d(sp["load_nodes"], sp["clamped_nodes"]).size
        bnd = batch._boundary_nodes(nelx, nely)
        assert np.isin(sp["load_nodes"], bnd).all() and np.isin(sp["clamped_nodes"], bnd).all()
        assert sp["clamped_nodes"].size >= 2  # a segment spans at least one element: rigid motions removed
        lv = batch.n_level_for(nelx, nely)
        assert 1 <= lv <= 4 and min(nelx, nely) >> lv >= 2


def test_random_specs_are_reproducible_and_distinct():
    a = batch.random_spec(7, seed=3)
    b = batch.random_spec(7, seed=3)
    c = batch.random_spec(8, seed=3)
    assert a["nelx"] == b["nelx"] and np.array_equal(a["load_nodes"], b["load_nodes"])
    assert np.array_equal(a["forces"], b["forces"])
    assert (a["nelx"], a["nely"], a["vf"]) != (c["nelx"], c["nely"], c["vf"])
