"""Solvers beyond the multigrid: CuCG (the reference's unpreconditioned CG,
solvers/_gpu.py:11-58) on grids of any extent, checked against direct solves and scipy's CG
on the oracle's assembled matrix.

Tolerances: solutions to 1e-6 relative of the direct solve at tol 1e-10 (the error bound of
CG at that residual times the matrix's conditioning on these small grids); iteration counts
within 2 of scipy's CG (same recurrences, different summation order).
"""
import numpy as np
import pytest

from oracle import ops, topopt

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _problem(nel, seed, lo=0.05):
    import torch
    import edge_to_b200 as eb
    p = topopt.mbb_problem(*nel) if len(nel) == 2 else topopt.cantilever_problem(*nel)
    rng = np.random.default_rng(seed)
    E = np.clip(rng.uniform(lo, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    st = lambda x: eb.auto_stiffness(x, 1.0, 0.3)  # noqa: E731
    mesh = (eb.CuStructuredMesh2D(*nel, *[float(v) for v in nel], stiffness=st) if len(nel) == 2 else
            eb.CuStructuredMesh3D(*nel, *[float(v) for v in nel], stiffness=st))
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    K = ops.assemble(p.grid, p.K0, E, p.cons)
    return p, k, K, torch.as_tensor(p.f, device="cuda")


@pytest.mark.parametrize("nel", [(61, 23), (13, 7, 5)])
def test_cg_matches_direct_solve(nel):
    import scipy.sparse.linalg as sla
    import edge_to_b200 as eb
    p, k, K, f = _problem(nel, 1)
    s = eb.CuCG(k, maxiter=20000, tol=1e-10)
    x, r = s.solve(f, use_last=False)
    xd = sla.spsolve(K.tocsc(), p.f)
    xg = x.cpu().numpy()
    true_res = np.linalg.norm(p.f - K @ xg) / np.linalg.norm(p.f)
    # the loop stops on the recurrence residual; the reported one is the true residual, which
    # rounding keeps within a small factor of the tolerance (the reference reports the same)
    assert r < 1e-9 and abs(r - true_res) <= 1e-3 * true_res + 1e-14
    assert rel(xg, xd) < 1e-6
    assert s.last_x0 is None  # the reference keeps a warm start only when use_last is set


def test_cg_iterations_follow_scipy_cg():
    import scipy.sparse.linalg as sla
    import edge_to_b200 as eb
    p, k, K, f = _problem((9, 5, 4), 2, lo=0.5)
    count = []
    sla.cg(K, p.f, rtol=1e-8, atol=0.0, maxiter=5000, callback=lambda xk: count.append(1))
    s = eb.CuCG(k, maxiter=5000, tol=1e-8)
    x, r = s.solve(f)
    assert abs(s.last_iters - len(count)) <= 2, (s.last_iters, len(count))
    # warm start: the second solve of the same system starts at the solution
    x2, r2 = s.solve(f)
    assert s.last_iters <= 1 and r2 < 1e-8


def test_cg_does_not_raise_on_maxiter():
    import edge_to_b200 as eb
    p, k, K, f = _problem((31, 17), 3)
    s = eb.CuCG(k, maxiter=7, tol=1e-12)
    x, r = s.solve(f, use_last=False)
    assert s.last_iters == 7 and r > 1e-12 and np.isfinite(r)


def test_fea_integrals_against_reference(golden):
    """edge_fea_integrals equals the reference's element integrals (random displacements, 1e-12),
    and CuTopOpt.FEA_integrals equals the reference's whole call on a 24x12 MBB beam with a
    random design (both solved to 1e-12: 1e-8)."""
    import torch
    import edge_to_b200 as eb
    z = golden("fea.npz")
    st = lambda x: eb.auto_stiffness(x, 1.0, 0.3)  # noqa: E731
    for tag, nel in (("2d", (13, 7)), ("3d", (6, 5, 4))):
        mesh = (eb.CuStructuredMesh2D(*nel, *[float(v) for v in nel], stiffness=st) if len(nel) == 2 else
                eb.CuStructuredMesh3D(*nel, *[float(v) for v in nel], stiffness=st))
        k = eb.CuStructuredStiffnessKernel(mesh)
        s, ss, en = k.fea_integrals(z[f"{tag}_w"], z[f"{tag}_U"], mesh.B_single, mesh.D_single)
        for a, b in ((s, z[f"{tag}_strain"]), (ss, z[f"{tag}_stress"]), (en, z[f"{tag}_energy"])):
            assert rel(a.cpu().numpy(), b) <= 1e-12, tag
    mesh = eb.CuStructuredMesh2D(24, 12, 24.0, 12.0, stiffness=st)
    mat = eb.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.5)
    k = eb.CuStructuredStiffnessKernel(mesh)
    filt = eb.CuStructuredFilter2D(mesh, 1.5)
    solver = eb.CuMultiGrid(mesh, k, tol=1e-12, n_level=2, maxiter=4000)
    opt = eb.CuTopOpt(mesh, mat, k, solver, filt, max_iter=1, verbose=False)
    nodes = mesh.nodes
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], 0.0))[0], np.array([[True, False]]))
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], 24.0) & np.isclose(nodes[:, 1], 0.0))[0],
                     np.array([[False, True]]))
    opt.add_F_nodal(np.where(np.isclose(nodes[:, 0], 0.0) & np.isclose(nodes[:, 1], 12.0))[0],
                    np.array([[0.0, -1.0]]))
    strain, stress, energy, vm = opt.FEA_integrals(torch.as_tensor(z["call_rho"], device="cuda"))
    for a, b in ((strain, z["call_strain"]), (stress, z["call_stress"]), (energy, z["call_energy"]),
                 (vm, z["call_vm"])):
        assert rel(a.cpu().numpy(), b) <= 1e-8


class _Direct:
    """Exact solve for the oracle's SIMP loop on grids the reference multigrid cannot coarsen."""

    def solve(self, K, f, use_last=True):
        import scipy.sparse.linalg as sla
        return sla.spsolve(K.tocsc(), f), 0.0


@pytest.mark.parametrize("nel,n_level", [((61, 23), 3), ((13, 7, 5), 2)])
def test_padded_multigrid_on_odd_extents(nel, n_level):
    """Element counts not divisible by 2**n_level: CuMultiGrid solves on a padded grid and
    returns the direct solution of the original system (the reference's multigrid stalls)."""
    import scipy.sparse.linalg as sla
    import edge_to_b200 as eb
    p, k, K, f = _problem(nel, 5)
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-8)):
        s = eb.CuMultiGrid(k.mesh, k, tol=tol, n_level=n_level, maxiter=500, precision=prec)
        assert s.padded
        x, r = s.solve(f, use_last=False)
        xd = sla.spsolve(K.tocsc(), p.f)
        assert r < tol and s.last_iters < 200, (prec, r, s.last_iters)
        assert rel(x.cpu().numpy(), xd) < (1e-6 if prec == "fp64" else 1e-4)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_simp_loop_on_odd_mbb_beam(precision):
    """Ten SIMP iterations on a 61x23 MBB beam (not coarsenable by the reference multigrid):
    compliance history against the oracle's loop with exact solves."""
    import torch
    import edge_to_b200 as eb
    nelx, nely = 61, 23
    ref = topopt.mbb_problem(nelx, nely, vf=0.5, rmin=1.5)
    ref.solver = _Direct()
    rho_ref, hist = ref.optimize(0.5, 10)
    st = lambda x: eb.auto_stiffness(x, 1.0, 0.3)  # noqa: E731
    mesh = eb.CuStructuredMesh2D(nelx, nely, float(nelx), float(nely), stiffness=st)
    mat = eb.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.5)
    mat.init_desvars = lambda nel, **kw: torch.full((nel,), 0.5, dtype=torch.float64, device="cuda")
    k = eb.CuStructuredStiffnessKernel(mesh)
    filt = eb.CuStructuredFilter2D(mesh, 1.5)
    solver = eb.CuMultiGrid(mesh, k, tol=1e-10 if precision == "fp64" else 1e-8, n_level=3, maxiter=1000,
                            precision=precision)
    opt = eb.CuTopOpt(mesh, mat, k, solver, filt, max_iter=10, ch_tol=0, fun_tol=0, verbose=False)
    nodes = mesh.nodes
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], 0.0))[0], np.array([[True, False]]))
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], nelx) & np.isclose(nodes[:, 1], 0.0))[0],
                     np.array([[False, True]]))
    opt.add_F_nodal(np.where(np.isclose(nodes[:, 0], 0.0) & np.isclose(nodes[:, 1], nely))[0],
                    np.array([[0.0, -1.0]]))
    assert not opt.fused
    rho, flag, h = opt.optimize(save_comp_history=True)
    c = np.array(h["comp_history"])
    err = np.abs(c - np.array(hist["comp"])) / np.array(hist["comp"])
    assert err.max() < (1e-8 if precision == "fp64" else 1e-6), err
    assert np.abs(rho.cpu().numpy() - rho_ref).max() < (1e-6 if precision == "fp64" else 1e-4)


@pytest.mark.parametrize("precision,mode", [("fp64", "threads"), ("mixed", "threads"), ("fp64", "persistent"),
                                            ("mixed", "persistent")])
def test_batch_of_random_problems_against_oracle(precision, mode):
    """Random uneven 2-D problems (the batching configuration's generator at reduced sizes),
    solved concurrently on several streams or with every solve and every OC update of a SIMP
    stage in one persistent launch (teams of two blocks): every problem's compliance history
    matches the oracle's SIMP loop with exact solves."""
    from edge_to_b200 import batch
    specs = [batch.random_spec(i, seed=100, nelx_range=(20, 44), nely_range=(12, 26)) for i in range(6)]
    tol = 1e-10 if precision == "fp64" else 1e-8
    b = batch.BatchSIMP(specs, precision=precision, tol=tol, maxiter=2000, n_threads=3,
                        persistent=mode == "persistent", team=2)
    ms = b.step(6)  # initial analysis + 5 design updates per problem
    assert ms > 0
    for spec, item in zip(specs, b.items):
        ref = topopt.SIMPOracle((spec["nelx"], spec["nely"]), vf=spec["vf"], rmin=spec["rmin"])
        ref.add_bc_nodal(spec["clamped_nodes"], [[True, True]])
        ref.add_force_nodal(spec["load_nodes"], spec["forces"])
        ref.solver = _Direct()
        _, hist = ref.optimize(spec["vf"], 5)
        c = np.array(item["comp"])
        want = np.array([hist["comp0"]] + hist["comp"])
        err = np.abs(c - want) / np.abs(want)
        assert err.max() < (1e-7 if precision == "fp64" else 1e-5), (spec["index"], err)


@pytest.mark.parametrize("threads,team,split", [(512, 1, 0), (1024, 1, 0), (512, 4, 0), (1024, 8, 0),
                                               (1024, 4, 4000)])
def test_persistent_batch_equals_per_problem_solves(threads, team, split):
    """The batched persistent solve (FP64) runs the per-problem FP64 solver's algorithm: the same
    PCG iteration counts and compliances and designs equal to rounding over five SIMP
    iterations, whatever the launch shape (blocks per problem, threads per block, small problems
    split off to single blocks in a second launch); its batched OC update gives the per-problem
    OC update's designs bit for bit."""
    import torch
    from edge_to_b200 import batch
    specs = [batch.random_spec(i, seed=7, nelx_range=(20, 90), nely_range=(12, 48)) for i in range(6)]
    a = batch.BatchSIMP(specs, precision="fp64", tol=1e-8, maxiter=1000, n_threads=2)
    c = batch.BatchSIMP(specs, precision="fp64", tol=1e-8, maxiter=1000, persistent=True, block_threads=threads,
                        team=team, split_dof=split)
    if split:
        dofs = [2 * (sp["nelx"] + 1) * (sp["nely"] + 1) for sp in specs]
        assert min(dofs) < split < max(dofs)
    a.step(5)
    c.step(5)
    for ia, ic in zip(a.items, c.items):
        assert ia["pcg"] == ic["pcg"]
        ca, cc = np.array(ia["comp"]), np.array(ic["comp"])
        assert np.max(np.abs(ca - cc) / np.abs(ca)) < 1e-9
        assert float((ia["rho"] - ic["rho"]).abs().max()) < 1e-9
    new = c.batch.update_design([it["rho"] for it in a.items], [it["dr"] for it in a.items])
    for it, nb in zip(a.items, new):
        assert torch.equal(it["opt"].update_design(it["rho"], it["dr"]), nb)


def test_persistent_batch_rejects_what_it_does_not_run():
    """Batched problems must share precision and material law; a W-cycle or springs are refused."""
    from edge_to_b200 import batch
    specs = [batch.random_spec(i, seed=3, nelx_range=(20, 30), nely_range=(12, 16)) for i in range(2)]
    o1, _ = batch.build(specs[0], "fp64", 1e-8, 100)
    o2, _ = batch.build(specs[1], "mixed", 1e-8, 100)
    with pytest.raises(ValueError):
        b = batch.BatchAnalysis([o1, o2])
        b.solve_and_process([torch_full(o1), torch_full(o2)], 0)


def torch_full(opt):
    import torch
    return torch.full((opt.mesh.n_elements,), 0.5, dtype=torch.float64, device="cuda")


def test_persistent_batch_at_full_size():
    """The batching configuration's own first eight problems at their stated sizes (64-512 x
    32-256 elements, padded multigrids up to six levels deep): three SIMP iterations with every
    solve in one persistent launch equal the per-problem FP64 solves (PCG counts, compliances
    to 1e-9), and every design meets its volume fraction after the batched OC updates."""
    from edge_to_b200 import batch
    specs = [batch.random_spec(i, seed=0) for i in range(8)]
    a = batch.BatchSIMP(specs, precision="fp64", tol=1e-6, maxiter=1000, n_threads=4, max_level=6)
    c = batch.BatchSIMP(specs, precision="fp64", tol=1e-6, maxiter=1000, persistent=True, max_level=6,
                        block_threads=1024, team=4)
    a.step(3)
    c.step(3)
    for sp, ia, ic in zip(specs, a.items, c.items):
        assert ia["pcg"] == ic["pcg"], (sp["index"], ia["pcg"], ic["pcg"])
        ca, cc = np.array(ia["comp"]), np.array(ic["comp"])
        assert np.max(np.abs(ca - cc) / np.abs(ca)) < 1e-9, sp["index"]
        assert float(ic["rho"].mean()) <= sp["vf"] * (1 + 1e-4)
