"""Pin the CPU oracle against fixtures produced by the reference's own CPU code.

The reference has no tests or golden files; tests/golden/make_golden.py ran its CPU
classes (kernels/_processors.py, geom/_filters.py, core/_mgm.py, solvers/_multigrid.py,
TopOpt/_solver.py) to produce them.  Everything here runs on the CPU.
"""
import numpy as np
import pytest

from oracle import elements, ops, topopt
from oracle.grid import Grid

H_OF = {2: {"even": None, "odd": None, "aniso": (0.5, 0.25)},
        3: {"even": None, "odd": None, "aniso": (0.5, 0.25, 0.5)}}


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_element_stiffness_kat(golden):
    kat = golden("kat_stiffness.npz")
    for nu in (0.3, 0.33):
        assert rel(elements.q4_stiffness(1, 1, 1, nu), kat[f"q4_nu{nu}"]) < 1e-14
        assert rel(elements.hex8_stiffness(1, 1, 1, 1, nu), kat[f"hex8_nu{nu}"]) < 1e-14
    assert rel(elements.q4_stiffness(0.5, 0.25, 1, 0.3), kat["q4_box_0.5x0.25_nu0.3"]) < 1e-14
    assert rel(elements.hex8_stiffness(0.5, 0.25, 1, 1, 0.3), kat["hex8_box_0.5x0.25x1_nu0.3"]) < 1e-14
    # hex8 K0[0,0] at nu=0.3 and symmetry / rigid-body null space
    K = elements.hex8_stiffness(1, 1, 1, 1, 0.3)
    assert abs(K[0, 0] - 0.23504273504273504) < 1e-15
    assert np.abs(K - K.T).max() < 1e-15
    assert np.abs(K.sum(axis=1)).max() < 1e-14


def _cases(golden):
    for dim, fn in ((2, "ops_2d.npz"), (3, "ops_3d.npz")):
        z = golden(fn)
        for tag in ("even", "odd", "aniso"):
            g = Grid(tuple(z[f"{tag}_nel"]), H_OF[dim][tag])
            K0 = elements.q4_stiffness(*g.h, 1, 0.3) if dim == 2 else elements.hex8_stiffness(*g.h, 1, 0.3)
            yield dim, tag, z, g, K0


def test_stiffness_ops(golden):
    for dim, tag, z, g, K0 in _cases(golden):
        E, u, cons = z[f"{tag}_E"], z[f"{tag}_u"], z[f"{tag}_cons"]
        Kc = ops.assemble(g, K0, E, cons)
        assert rel(ops.assemble(g, K0, E) @ u, z[f"{tag}_matvec_nocon"]) < 1e-13, (dim, tag)
        assert rel(Kc @ u, z[f"{tag}_matvec"]) < 1e-13, (dim, tag)
        assert rel(ops.diagonal(Kc), z[f"{tag}_diag"]) < 1e-13, (dim, tag)
        assert rel(ops.dk(g, K0, u), z[f"{tag}_dk"]) < 1e-13, (dim, tag)
        cm = np.zeros(g.n_dof, dtype=bool)
        cm[cons] = True
        assert rel(ops.matvec_free(g, K0, E, u, cm), z[f"{tag}_matvec"]) < 1e-13, (dim, tag)


def test_filter(golden):
    n = 0
    for dim, tag, z, g, K0 in _cases(golden):
        for k in z.files:
            if k.startswith(f"{tag}_filt") and k.endswith("_in"):
                r = float(k[len(tag) + 5:-3])
                H, N = ops.filter_matrix(g, r)
                x = z[k]
                assert rel(H @ x, z[f"{tag}_filt{r}_H"]) < 1e-13
                assert rel(H.T @ x, z[f"{tag}_filt{r}_HT"]) < 1e-13
                assert len(ops.filter_stencil(g, r)[1]) == int(z[f"{tag}_filt{r}_ntaps"])
                n += 1
    assert n >= 8


def test_transfer_and_galerkin(golden):
    for dim, tag, z, g, K0 in _cases(golden):
        R = ops.restriction_matrix(g, "cpu")
        assert rel(R @ z[f"{tag}_restrict_in"], z[f"{tag}_restrict"]) < 1e-13
        assert rel(ops.prolongation_matrix(g) @ z[f"{tag}_prolong_in"], z[f"{tag}_prolong"]) < 1e-13
        if dim == 3:  # CPU and GPU restriction agree in 3-D
            assert rel(ops.restriction_matrix(g, "gpu") @ z[f"{tag}_restrict_in"], z[f"{tag}_restrict"]) < 1e-13
        if f"{tag}_A1" in z.files:
            Kc = ops.assemble(g, K0, z[f"{tag}_E"], z[f"{tag}_cons"])
            A1 = ops.galerkin(Kc, g)
            A2 = ops.galerkin(A1, g.coarse())
            assert rel(A1.toarray(), z[f"{tag}_A1"]) < 1e-13
            assert rel(A2.toarray(), z[f"{tag}_A2"]) < 1e-13
            assert rel(1.0 / A1.diagonal(), z[f"{tag}_D1inv"]) < 1e-13


def test_gpu_restriction_is_twice_cpu_in_2d_interior(golden):
    g = Grid((8, 4))
    Rg = ops.restriction_matrix(g, "gpu").toarray()
    Rc = ops.restriction_matrix(g, "cpu").toarray()
    assert np.allclose(Rg, 2 * Rc)


def test_oc_update(golden):
    for dim, fn in ((2, "ops_2d.npz"), (3, "ops_3d.npz")):
        z = golden(fn)
        g = Grid(tuple(z["even_nel"]))
        A = elements.element_measure(g.h)
        rn, lam, steps = topopt.oc_update(z["even_oc_rho"], z["even_oc_df"], A, A * g.n_el, 0.4, 0.2)
        assert np.array_equal(rn, z["even_oc_out"].reshape(-1))
        assert 30 <= steps <= 60


@pytest.mark.slow
def test_mbb_trajectory_cpu_semantics(golden):
    """The oracle in the reference CPU solver's semantics retraces its 100 iterations."""
    z = golden("loop_mbb2d.npz")
    p = topopt.mbb_problem(mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=1000, variant="cpu"), vf=0.5, rmin=1.5)
    assert np.array_equal(np.nonzero(p.f)[0], z["f_idx"])
    assert np.array_equal(p.cons, z["constraints"])
    rho, h = p.optimize(0.5, 100)
    c = np.array(h["comp"])
    assert np.abs(c - z["comp_history"]).max() / c.min() < 1e-8
    assert np.abs(rho - z["rho_final"]).max() < 1e-6
    # fine matvecs per solve: 8 per PCG iteration + 1 initial residual
    assert list(8 * np.array(p.solver.pcg_iters[:5]) + 1) == list(z["matvecs_per_solve"][:5])


def test_mbb_trajectory_gpu_semantics(golden):
    """GPU-solver semantics (omega reset, GPU restriction) reach the same designs."""
    z = golden("loop_mbb2d.npz")
    p = topopt.mbb_problem(mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=1000, variant="gpu"), vf=0.5, rmin=1.5)
    rho, h = p.optimize(0.5, 100)
    c = np.array(h["comp"])
    assert np.abs(c - z["comp_history"]).max() / c.min() < 1e-6
    assert np.abs(rho - z["rho_final"]).max() < 1e-5


def test_cantilever_first_iterations(golden):
    z = golden("loop_cant3d.npz")
    p = topopt.cantilever_problem(64, 32, 32, vf=0.12, rmin=1.5,
                                  mg_kwargs=dict(tol=1e-6, n_level=4, maxiter=1000, variant="cpu"))
    assert np.array_equal(p.cons, z["constraints"])
    assert np.array_equal(np.nonzero(p.f)[0], z["f_idx"])
    rho, h = p.optimize(0.12, len(z["comp_history"]))
    c = np.array(h["comp"])
    assert np.abs(c - z["comp_history"]).max() / c.min() < 1e-6


def test_gradient_random_rho(golden):
    z = golden("grad_cant3d.npz")
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, rmin=2.0,
                                  mg_kwargs=dict(tol=1e-10, n_level=3, maxiter=2000, variant="gpu"))
    comp, dr, res, U = p.solve_and_process(z["rho"])
    assert abs(comp - float(z["compliance"])) / comp < 1e-8
    assert rel(dr, z["dr"]) < 1e-7


def test_fea_integrals_oracle_and_element_matrices(golden):
    """Oracle element integrals (strain, stress, strain energy) equal the reference's on random
    displacements, and this package's meshes build the reference's B_single / D_single."""
    import edge_to_b200 as eb
    from oracle import elements
    z = golden("fea.npz")
    for tag, nel in (("2d", (13, 7)), ("3d", (6, 5, 4))):
        g = Grid(nel)
        K0 = elements.q4_stiffness(1, 1, E=1.0, nu=0.3) if g.dim == 2 else elements.hex8_stiffness(1, 1, 1, E=1.0,
                                                                                                   nu=0.3)
        st, ss, en = ops.fea_integrals(g, K0, z[f"{tag}_B"], z[f"{tag}_D"], z[f"{tag}_w"], z[f"{tag}_U"])
        for a, b in ((st, z[f"{tag}_strain"]), (ss, z[f"{tag}_stress"]), (en, z[f"{tag}_energy"])):
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
        stiff = lambda x: eb.auto_stiffness(x, 1.0, 0.3)  # noqa: E731
        mesh = (eb.CuStructuredMesh2D(*nel, *[float(v) for v in nel], stiffness=stiff) if g.dim == 2 else
                eb.CuStructuredMesh3D(*nel, *[float(v) for v in nel], stiffness=stiff))
        assert np.abs(mesh.B_single - z[f"{tag}_B"]).max() <= 1e-13
        assert np.abs(mesh.D_single - z[f"{tag}_D"]).max() <= 1e-13


MM_CASES = ("two", "three", "shared")


def mm_law(z, tag):
    from oracle.material import MultiMaterialLaw
    n = int(z[f"{tag}_n"])
    rm = z[f"{tag}_rho_mat"]
    return MultiMaterialLaw(n_material=n, mass=z[f"{tag}_mass"].reshape(-1, 1), E_mat=z[f"{tag}_E_mat"].reshape(-1, 1),
                            rho_mat=rm.reshape(-1, 1) if rm.size else None, void=float(z[f"{tag}_void"]),
                            penalty=float(z[f"{tag}_penalty"]))


def test_multimaterial_law_oracle(golden):
    """The oracle's PenalizedMultiMaterial restatement (forward, plain, backward, mass
    constraint, ocP) equals the reference class on random designs with clip edges."""
    z = golden("multimaterial.npz")
    for tag in MM_CASES:
        law = mm_law(z, tag)
        rho = z[f"{tag}_rho"]
        assert rel(law.forward(rho), z[f"{tag}_E"]) < 1e-14, tag
        assert rel(law.forward(rho, plain=True), z[f"{tag}_Eplain"]) < 1e-14, tag
        assert rel(law.backward(rho), z[f"{tag}_dE"]) < 1e-13, tag
        dg, vol = z[f"{tag}_dg"], float(z[f"{tag}_vol"])
        cons = np.stack([law.con(rho * s, dg, vol) for s in (0.1, 0.5, 1.0)])
        assert (cons == z[f"{tag}_cons"]).all(), tag
        assert rel(law.ocp(z[f"{tag}_df"], dg, rho), z[f"{tag}_ocP"]) < 1e-14, tag
        assert rel(law.ocp(np.abs(z[f"{tag}_df"]), dg, rho), z[f"{tag}_ocP0"]) < 1e-14, tag


def test_multimaterial_oracle_loop():
    """The oracle's multi-material SIMP loop (no reference loop exists for this law): on a
    small MBB beam the compliance falls in every one of the first iterations and each
    material's mass ends within the OC bisection tolerance of its bound."""
    from oracle.material import MultiMaterialLaw
    law = MultiMaterialLaw(n_material=2, mass=[[0.25], [0.15]], E_mat=[[1.0], [0.5]], void=1e-9, penalty=3.0)
    p = topopt.mbb_problem(48, 16, law=law, rmin=1.5, move=0.2)
    rho, hist = p.optimize(np.tile([0.25, 0.15], (48 * 16, 1)), 6)
    c = [hist["comp0"]] + hist["comp"]
    assert all(b < a for a, b in zip(c, c[1:]))
    assert (rho.mean(axis=0) <= np.array([0.25, 0.15]) * (1 + 1e-4)).all()
    assert (rho >= 0).all() and (rho <= 1).all()


GENERAL_TAGS = ("tri", "mixed", "tet", "hex")


def test_general_mesh_oracle(golden):
    """Unstructured meshes (T3, T3+Q4, Tet4 of both orientations, distorted hex8): the oracle's
    operator with and without constraints, diagonal, dk, centroids and KD-tree filter equal the
    reference's UniformStiffnessKernel / GeneralStiffnessKernel / GeneralFilter."""
    from oracle import general
    z = golden("general.npz")
    for tag in GENERAL_TAGS:
        sizes, flat, dof = z[f"{tag}_sizes"], z[f"{tag}_flat"], int(z[f"{tag}_dof"])
        conn = general.connectivity(sizes, flat)
        Ks = general.element_matrices(z[f"{tag}_Kflat"], sizes, dof)
        nodes = z[f"{tag}_nodes"]
        n_dof = nodes.shape[0] * dof
        assert bool(z[f"{tag}_uniform"]) == (len(set(sizes.tolist())) == 1)
        assert rel(general.centroids(nodes, conn), z[f"{tag}_centroids"]) < 1e-14, tag
        K = general.assemble(n_dof, dof, conn, Ks, z[f"{tag}_rho"])
        assert rel(K @ z[f"{tag}_u"], z[f"{tag}_matvec"]) < 1e-13, tag
        Kc = general.assemble(n_dof, dof, conn, Ks, z[f"{tag}_rho"], z[f"{tag}_cons"])
        assert rel(Kc @ z[f"{tag}_u"], z[f"{tag}_matvec_con"]) < 1e-13, tag
        assert rel(Kc.diagonal(), z[f"{tag}_diag_con"]) < 1e-13, tag
        assert rel(general.dk(conn, Ks, z[f"{tag}_U"], dof), z[f"{tag}_dk"]) < 1e-13, tag
        H = general.filter_matrix(z[f"{tag}_centroids"], 1.6)
        assert rel(H.toarray(), z[f"{tag}_H"]) < 1e-14, tag
        assert rel(H @ z[f"{tag}_fx"], z[f"{tag}_Hx"]) < 1e-14, tag
        assert rel(H.T @ z[f"{tag}_fx"], z[f"{tag}_HTx"]) < 1e-14, tag
