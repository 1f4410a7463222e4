"""Failure behaviour of the solve path, made on the host (no GPU fault, no hang): non-finite
loads and densities, a singular system (no boundary conditions), every DOF constrained, and
maxiter exhaustion.  The solvers follow the reference: they do not raise on non-convergence
(solvers/_multigrid_cuda.py:234-242) and report the residual; a singular coarsest Galerkin
matrix is reported as an error; every device wait is bounded."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cantilever(precision, tol=1e-8, maxiter=500, bcs=True, **kw):
    import torch
    import edge_to_b200 as eb
    from oracle import topopt
    p = topopt.cantilever_problem(16, 8, 8)
    mesh = eb.CuStructuredMesh3D(16, 8, 8, 16.0, 8.0, 8.0, stiffness=lambda x: eb.auto_stiffness(x, 1.0, 0.3))
    k = eb.CuStructuredStiffnessKernel(mesh)
    if bcs:
        k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.full((16 * 8 * 8,), 0.5 ** 3, dtype=torch.float64, device="cuda"))
    kw.setdefault("tune_sweeps", False)
    s = eb.CuMultiGrid(mesh, k, tol=tol, n_level=2, maxiter=maxiter, precision=precision, autotune=False, **kw)
    return p, k, s, torch.as_tensor(p.f, device="cuda")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_maxiter_exhaustion_returns_the_residual(precision):
    """Three iterations at rtol 1e-12: no exception, the iteration count is maxiter and the
    reported residual is the (large) residual reached."""
    p, k, s, f = _cantilever(precision, tol=1e-12, maxiter=3)
    x, r = s.solve(f, use_last=False)
    assert s.last_iters == 3
    assert math.isfinite(r) and r > 1e-12
    assert bool(torch_isfinite(x))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_load_does_not_converge_or_hang(precision):
    """A NaN in the load: the residual norm is NaN, so the stopping test never passes; the solve
    runs to maxiter and reports a non-finite residual instead of raising or hanging."""
    p, k, s, f = _cantilever(precision, maxiter=20)
    f = f.clone()
    free = int(np.nonzero(~np.isin(np.arange(f.numel()), np.asarray(p.cons)))[0][0])
    f[free] = float("nan")
    x, r = s.solve(f, use_last=False)
    assert s.last_iters == 20
    assert not math.isfinite(r)


def test_singular_system_is_reported():
    """No boundary conditions: K and the coarsest Galerkin matrix are singular (rigid-body
    modes).  The coarsest Cholesky either meets a non-positive pivot and the solve raises
    RuntimeError (EDGE_ENOTPD) before iterating on a broken preconditioner, or rounding leaves
    every pivot positive and the solve runs to maxiter without converging on the inconsistent
    system; either way it returns promptly and never reports convergence."""
    p, k, s, f = _cantilever("fp64", bcs=False, maxiter=50)
    try:
        x, r = s.solve(f, use_last=False)
    except RuntimeError as e:
        assert "positive definite" in str(e)
        return
    assert s.last_iters == 50 and not r < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_dof_constrained(precision):
    """Every DOF constrained: K is the identity, so the solution is the load itself."""
    import torch
    p, k, s, f = _cantilever(precision, bcs=False)
    k.add_constraints(np.arange(k.shape[0]))
    g = torch.linspace(-1.0, 1.0, k.shape[0], dtype=torch.float64, device="cuda")
    x, r = s.solve(g, use_last=False)
    assert r < 1e-8
    assert float(torch.linalg.norm(x - g) / torch.linalg.norm(g)) < 1e-7


def test_nonfinite_density_is_mapped_to_void_by_the_law_clip():
    """A NaN design variable: the SIMP law's clip to [void, 1] (fmax/fmin, which return the
    non-NaN operand) maps it to the void stiffness, so the analysis stays finite."""
    import torch
    import edge_to_b200 as eb
    mesh = eb.CuStructuredMesh2D(16, 8, 16.0, 8.0, stiffness=lambda x: eb.auto_stiffness(x, 1.0, 0.3))
    mat = eb.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.5)
    k = eb.CuStructuredStiffnessKernel(mesh)
    filt = eb.CuStructuredFilter2D(mesh, 1.5)
    solver = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=2, maxiter=1000, autotune=False)
    opt = eb.CuTopOpt(mesh, mat, k, solver, filt, max_iter=1, verbose=False)
    nodes = mesh.nodes
    opt.add_BC_nodal(np.where(np.isclose(nodes[:, 0], 0.0))[0], np.array([[True, True]]))
    opt.add_F_nodal(np.where(np.isclose(nodes[:, 0], 16.0))[0], np.array([[0.0, -1.0]]))
    rho = torch.full((16 * 8,), 0.5, dtype=torch.float64, device="cuda")
    rho[40] = float("nan")
    c, dr, res = opt.solve_and_process(rho, 0)
    assert math.isfinite(float(c)) and res < 1e-8


def test_fixed_omega_that_diverges_falls_back_to_the_schedule():
    """A fixed smoother weight far above 2 / lambda_max(D^-1 K) makes the preconditioner
    indefinite: the solve does not converge within maxiter, is run again from the same warm
    start with the reference's schedule, converges, and the schedule is kept afterwards."""
    import torch
    p, k, s, f = _cantilever("mixed", maxiter=200, mixed_omega=1.6)
    assert s.fixed_omega == 1.6
    x0, r0 = s.solve(f, use_last=False)        # cold start: rerun from zero
    assert r0 < 1e-8 and s.fixed_omega is None
    ref = eb_solve(p, "fp64")
    assert float(torch.linalg.norm(x0 - ref) / torch.linalg.norm(ref)) < 1e-6
    x1, r1 = s.solve(f, use_last=True)
    assert r1 < 1e-8 and s.fixed_omega is None


def test_sweep_tuner_compares_fixed_omega_with_the_schedule():
    """mixed_omega="auto": the solves before the sweep autotuner run the reference's schedule;
    the tuner times its chosen pattern with the weight fixed at omega as well and keeps the
    faster; the solver then runs that weight."""
    p, k, s, f = _cantilever("mixed", maxiter=200, tune_sweeps=True)
    assert s.fixed_omega is None
    s.solve(f, use_last=False)
    x, r = s.solve(f, use_last=True)           # the first warm-started solve tunes
    om = s.sweeps["omega"]
    assert om["fixed"] == 0.5 and om["schedule_ms"] is not None and r < 1e-8
    assert om["chosen"] in ("fixed", "schedule") and (s.fixed_omega == 0.5) == (om["chosen"] == "fixed")
    x, r = s.solve(f, use_last=True)
    assert r < 1e-8


def test_schedule_only_solver_never_fixes_omega():
    """mixed_omega=None: the tuner leaves the weight alone; the reference's schedule throughout."""
    p, k, s, f = _cantilever("mixed", maxiter=200, tune_sweeps=True, mixed_omega=None)
    s.solve(f, use_last=False)
    s.solve(f, use_last=True)
    assert s.sweeps["omega"] is None and s.fixed_omega is None


def eb_solve(p, precision):
    import torch
    _, k, s, f = _cantilever(precision, tol=1e-10)
    x, r = s.solve(f, use_last=False)
    return x


def torch_isfinite(x):
    import torch
    return torch.isfinite(x).all()
