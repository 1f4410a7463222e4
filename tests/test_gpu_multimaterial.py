"""Multi-material SIMP (PenalizedMultiMaterial, MaterialModels.py:102-235) on the GPU.

The law (edge_mm_law) is pinned against fixtures generated by the reference class itself
(tests/golden/multimaterial.npz); the loop (CuTopOpt on an (n_el, n_material) design) against
the oracle's restatement with exact sparse solves: the reference's own TopOpt loop cannot run
this class (it reshapes the design to one column, TopOpt/_solver.py:281).
"""
import numpy as np
import pytest

from oracle import topopt
from oracle.material import MultiMaterialLaw

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _material(z, tag):
    import edge_to_b200 as eb
    rm = z[f"{tag}_rho_mat"]
    return eb.PenalizedMultiMaterial(n_material=int(z[f"{tag}_n"]), mass=z[f"{tag}_mass"].reshape(-1, 1),
                                     E_mat=z[f"{tag}_E_mat"].reshape(-1, 1),
                                     rho_mat=rm.reshape(-1, 1) if rm.size else None, void=float(z[f"{tag}_void"]),
                                     penalty=float(z[f"{tag}_penalty"]))


def test_multimaterial_law_against_reference(golden):
    """Forward (penalised, plain), backward, mass constraint and ocP on the device equal the
    reference class on random designs (two and three materials, per-material and shared
    mass), including designs at the clip edges and positive sensitivities."""
    import torch
    z = golden("multimaterial.npz")
    for tag in ("two", "three", "shared"):
        m = _material(z, tag)
        rho = torch.as_tensor(z[f"{tag}_rho"], device="cuda")
        E = m(rho, 0)
        assert tuple(E.shape) == (rho.shape[0], 1)
        assert rel(E.cpu(), z[f"{tag}_E"]) < 1e-13, tag
        assert rel(m(rho, 0, plain=True).cpu(), z[f"{tag}_Eplain"]) < 1e-13, tag
        assert rel(m.grad(rho, 0).cpu(), z[f"{tag}_dE"]) < 1e-12, tag
        dg = torch.as_tensor(z[f"{tag}_dg"], device="cuda")
        vol = float(z[f"{tag}_vol"])
        cons = np.stack([m.evaluate_constraint(rho * s, dg, vol).cpu().numpy() for s in (0.1, 0.5, 1.0)])
        assert (cons == z[f"{tag}_cons"]).all(), tag
        df = torch.as_tensor(z[f"{tag}_df"], device="cuda")
        assert rel(m.ocP(df, dg, rho).cpu(), z[f"{tag}_ocP"]) < 1e-14, tag
        assert rel(m.ocP(df.abs(), dg, rho).cpu(), z[f"{tag}_ocP0"]) < 1e-14, tag
        # numpy designs go through the same kernel
        assert rel(m(z[f"{tag}_rho"], 0), z[f"{tag}_E"]) < 1e-13, tag


def test_multimaterial_law_argument_checks():
    import edge_to_b200 as eb
    with pytest.raises(ValueError):
        eb.PenalizedMultiMaterial(n_material=3)  # E_mat has two rows
    with pytest.raises(ValueError):
        eb.PenalizedMultiMaterial(n_material=2, rho_mat=np.array([[1.0], [0.5]]))  # two masses with rho_mat
    with pytest.raises(ValueError):
        eb.PenalizedMultiMaterial(n_material=9, E_mat=np.ones((9, 1)), mass=np.ones((9, 1)))


@pytest.mark.parametrize("shared", [False, True])
def test_multimaterial_simp_against_oracle(shared):
    """Eight SIMP iterations of a two-material 48x16 MBB beam through CuTopOpt (FP64 GMG-PCG
    at rtol 1e-10) follow the oracle (exact solves) within 1e-6 in compliance and 1e-5 in
    the design; the mass constraints hold to the OC bisection's tolerance."""
    import torch
    import edge_to_b200 as eb
    nelx, nely = 48, 16
    if shared:
        kw = dict(n_material=2, mass=np.array([[0.3]]), E_mat=np.array([[1.0], [0.4]]),
                  rho_mat=np.array([[1.0], [0.35]]), void=1e-9, penalty=3.0)
        rho0 = np.tile([0.2, 0.2], (nelx * nely, 1))
    else:
        kw = dict(n_material=2, mass=np.array([[0.25], [0.15]]), E_mat=np.array([[1.0], [0.5]]), void=1e-9,
                  penalty=3.0)
        rho0 = np.tile([0.25, 0.15], (nelx * nely, 1))
    law = MultiMaterialLaw(**kw)
    p = topopt.mbb_problem(nelx, nely, law=law, rmin=1.5, move=0.2)
    _, hist = p.optimize(rho0, 8)

    mesh = eb.CuStructuredMesh2D(nelx, nely, float(nelx), float(nely), stiffness=lambda x: eb.auto_stiffness(x, 1.0, 0.3))
    mat = eb.PenalizedMultiMaterial(**kw)
    k = eb.CuStructuredStiffnessKernel(mesh)
    filt = eb.CuStructuredFilter2D(mesh, 1.5)
    solver = eb.CuMultiGrid(mesh, k, tol=1e-10, n_level=2, maxiter=2000, precision="fp64")
    opt = eb.CuTopOpt(mesh, mat, k, solver, filt, max_iter=1, move=0.2, ch_tol=0, fun_tol=0, verbose=False)
    nodes = mesh.nodes
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], 0))[0], np.array([[True, False]]))
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], nelx) & np.isclose(nodes[:, 1], 0))[0], np.array([[False, True]]))
    opt.add_F_nodal(np.where(np.isclose(nodes[:, 0], 0) & np.isclose(nodes[:, 1], nely))[0], np.array([[0.0, -1.0]]))
    rho = torch.as_tensor(rho0, device="cuda")
    c, dr, _ = opt.solve_and_process(rho, 0)
    assert abs(float(c) - hist["comp0"]) / hist["comp0"] < 1e-8
    comps = []
    for it in range(8):
        rho = opt.update_design(rho, dr)
        assert tuple(rho.shape) == (nelx * nely, 2)
        c, dr, _ = opt.solve_and_process(rho, it)
        comps.append(float(c))
    assert rel(comps, hist["comp"]) < 1e-6
    assert np.abs(rho.cpu().numpy() - hist["rho"][-1]).max() < 1e-5
    # the OC returns the design of the last multiplier tried (TopOpt/_solver.py:298-311), so
    # the masses hold to the bisection's relative tolerance (1e-4), as in the oracle
    r = rho.cpu().numpy()
    if shared:
        assert (r @ np.array([1.0, 0.35])).mean() <= 0.3 * (1 + 1e-4)
    else:
        assert (r.mean(axis=0) <= np.array([0.25, 0.15]) * (1 + 1e-4)).all()


@pytest.mark.parametrize("n_mat,shared", [(2, False), (3, False), (2, True), (3, True)])
def test_multimaterial_oc_launch_equals_torch_bisection(n_mat, shared):
    """The multi-material OC update as one launch (edge_oc_update_multi) gives the designs of the
    bisection written in torch operations (one host read per step, the reference's loop) on
    random designs and sensitivities, per-material and shared mass constraints; the bisection's
    decisions only depend on sums that the two compute in different orders."""
    import torch
    import edge_to_b200 as eb
    nelx, nely = 40, 24
    mesh = eb.CuStructuredMesh2D(nelx, nely, float(nelx), float(nely), stiffness=lambda x: eb.auto_stiffness(x, 1.0, 0.3))
    E_mat = np.linspace(1.0, 0.3, n_mat).reshape(-1, 1)
    if shared:
        mat = eb.PenalizedMultiMaterial(n_material=n_mat, mass=np.array([[0.3]]), E_mat=E_mat,
                                        rho_mat=np.linspace(1.0, 0.4, n_mat).reshape(-1, 1), void=1e-9)
    else:
        mat = eb.PenalizedMultiMaterial(n_material=n_mat, mass=np.full((n_mat, 1), 0.6 / n_mat), E_mat=E_mat,
                                        void=1e-9)
    k = eb.CuStructuredStiffnessKernel(mesh)
    filt = eb.CuStructuredFilter2D(mesh, 1.5)
    solver = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=2, maxiter=500, precision="fp64")
    opt = eb.CuTopOpt(mesh, mat, k, solver, filt, max_iter=1, move=0.2, verbose=False)
    g = torch.Generator(device="cuda").manual_seed(5 + n_mat)
    n = nelx * nely
    for trial in range(3):
        rho = 0.05 + 0.9 * torch.rand(n, n_mat, generator=g, device="cuda", dtype=torch.float64)
        df = -torch.rand(n, n_mat, generator=g, device="cuda", dtype=torch.float64) * (10.0 ** trial)
        fast = opt.update_design(rho, df)
        As = torch.as_tensor(np.asarray(mesh.As), dtype=torch.float64, device="cuda")
        ocP = torch.clamp(mat.ocP(df, As, rho), min=1e-12)
        ref = opt._bisect_torch(rho, ocP, As)
        assert tuple(fast.shape) == (n, n_mat)
        assert float((fast - ref).abs().max()) < 1e-12, trial
