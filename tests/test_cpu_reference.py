"""The timed CPU baseline (oracle/cpu_simp.py, the reference's CPU SIMP iteration on the
host cores) against the scipy oracle, which the golden fixtures pin to the reference: every
operator to round-off, and the PCG iterates of the CPU solver semantics (omega carried
across solves) step for step."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def small():
    from oracle import cpu_simp, ops
    p = cpu_simp.CpuSimpReference((8, 4, 4), 0.3, 1.5, 2, 1e-8)
    rng = np.random.default_rng(0)
    E = rng.uniform(0.1, 1.0, p.grid.n_el)
    K = ops.assemble(p.grid, p.K0, E, np.where(p.cons)[0])
    return p, E, K, rng


@pytest.mark.parametrize("indexing", ["list", "structured"])
def test_operator_and_transfers_match_oracle(small, indexing):
    from oracle import ops
    p, E, K, rng = small
    p.indexing = indexing
    u = rng.standard_normal(p.grid.n_dof)
    assert np.abs(p.matvec(E, u) - K @ u).max() <= 1e-13 * np.abs(K @ u).max()
    p.setup(E)
    assert np.abs(p.levels[0][1] - 1.0 / ops.diagonal(K)).max() <= 1e-13
    A1 = ops.galerkin(K, p.grid)
    assert abs(p.levels[1][0] - A1).max() <= 1e-14 * abs(A1).max()
    assert np.abs(p.restrict(0, u) - ops.restriction_matrix(p.grid, "cpu") @ u).max() <= 1e-14
    vc = rng.standard_normal(p.levels[1][0].shape[0])
    assert np.abs(p.prolong(0, vc) - ops.prolongation_matrix(p.grid) @ vc).max() <= 1e-14
    H, _ = ops.filter_matrix(p.grid, 1.5)
    rho = rng.uniform(0.0, 1.0, p.grid.n_el)
    assert np.abs(p.filter(rho) - H @ rho).max() <= 1e-14
    assert np.abs(p.filter(rho, transpose=True) - H.T @ rho).max() <= 1e-14
    p.indexing = "structured"


def test_pcg_follows_the_cpu_solver_step_for_step(small):
    from oracle import mg
    p, E, K, rng = small
    o = mg.MultiGridOracle(p.grid, tol=1e-8, n_level=2, variant="cpu")
    x_o, res_o = o.solve(K, p.f)
    p.x = None
    p.omega = 0.5
    p.setup(E)
    n, res = p.pcg(E)
    assert n == o.pcg_iters[-1]
    assert np.abs(p.x - x_o).max() <= 1e-12 * np.abs(x_o).max()
    assert abs(res - res_o) <= 1e-12


def test_measure_reports_every_part():
    from oracle import cpu_simp
    m = cpu_simp.measure((8, 4, 4), 0.3, 1.5, 2, 1e-6, samples=2)
    assert m["first_solve_pcg_iters"] > 0 and len(m["pcg_iteration_samples_s"]) == 2
    parts = m["setup_s"] + m["post_s"] + m["oc_s"] + m["first_solve_pcg_iters"] * m["pcg_iteration_s"]
    assert abs(m["seconds_per_iteration"] - parts) <= 1e-12 * parts
