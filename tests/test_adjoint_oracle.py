"""The oracle's adjoint gradients (CPU, FP64, direct solves): against central finite
differences for compliance and for the compliant-mechanism displacement objective, and
the compliance gradient against the reference's own dr fixture."""
import numpy as np

from oracle import adjoint, elements, ops
from oracle.grid import Grid


def _cantilever(nel, rmin):
    g = Grid(nel)
    K0 = elements.hex8_stiffness(1, 1, 1, 1.0, 0.3)
    H, _ = ops.filter_matrix(g, rmin)
    nelx, nely, nelz = nel
    face = np.array([g.node_id(0, j, k) for j in range(nely + 1) for k in range(nelz + 1)])
    cons = np.sort(np.concatenate([3 * face + d for d in range(3)]))
    edge = np.array([g.node_id(nelx, 0, k) for k in range(nelz + 1)])
    f = np.zeros(g.n_dof)
    f[3 * edge + 1] = -1.0 / edge.shape[0]
    return g, K0, H, f, cons


def test_compliance_gradient_matches_reference_dr(golden):
    z = golden("grad_cant3d.npz")
    g, K0, H, f, cons = _cantilever((32, 16, 16), 2.0)
    obj = adjoint.Objective(g, K0, H, f, cons)
    grad, J = obj.gradient(z["rho"])
    assert abs(J - float(z["compliance"])) / float(z["compliance"]) < 1e-9
    assert np.abs(grad - z["dr"]).max() / np.abs(z["dr"]).max() < 1e-8


def test_compliance_gradient_finite_differences():
    g, K0, H, f, cons = _cantilever((8, 4, 4), 1.5)
    rho = np.random.default_rng(0).uniform(0.2, 1.0, g.n_el)
    obj = adjoint.Objective(g, K0, H, f, cons)
    grad, _ = obj.gradient(rho)
    idx = np.random.default_rng(1).choice(g.n_el, 12, replace=False)
    fd = adjoint.central_differences(obj.value, rho, idx)
    assert np.abs(fd - grad[idx]).max() / np.abs(grad[idx]).max() < 1e-6


def test_mechanism_gradient_finite_differences():
    nel = (24, 12)
    g = Grid(nel)
    K0 = elements.q4_stiffness(1, 1, 1.0, 0.3)
    H, _ = ops.filter_matrix(g, 1.5)
    f, l, cons, springs = adjoint.inverter_problem(*nel)
    rho = np.random.default_rng(2).uniform(0.2, 1.0, g.n_el)
    obj = adjoint.Objective(g, K0, H, f, cons, l=l, springs=springs)
    grad, J = obj.gradient(rho)
    assert J < 0 or J > 0
    idx = np.random.default_rng(3).choice(g.n_el, 12, replace=False)
    fd = adjoint.central_differences(obj.value, rho, idx)
    assert np.abs(fd - grad[idx]).max() / np.abs(grad[idx]).max() < 1e-6
    # springs really enter: without them the objective changes
    J0 = adjoint.Objective(g, K0, H, f, cons, l=l).value(rho)
    assert abs(J0 - J) > 1e-6 * abs(J)
