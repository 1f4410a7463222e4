"""Differentiation (torch.autograd.Function with the hand-written adjoint) on the GPU.

Compliance: against the reference's own dr fixture and against central finite differences
(step 1e-4, 32 seeded elements) on the 128x64x64 cantilever with rho ~ U[0.2, 1].
Compliant mechanism (400x200 inverter, springs 0.1): against central finite differences
and against the oracle's adjoint gradient on a small grid.  FP64 throughout, plus the
mixed-precision solver's gradient error against FP64.

The finite differences use correction solves: J(rho +- h e_i) = l.(u0 + d) with
K(rho +- h e_i) d = f - K(rho +- h e_i) u0, so the solver tolerance applies to the small
correction d rather than to u, and the difference quotient keeps ~10 significant digits.
"""
import numpy as np
import pytest

from oracle import adjoint, elements, ops
from oracle.grid import Grid

pytestmark = pytest.mark.gpu


def _mesh(nel):
    import edge_to_b200 as eb
    st = lambda x: eb.auto_stiffness(x, 1.0, 0.3)  # noqa: E731
    if len(nel) == 2:
        return eb.CuStructuredMesh2D(nel[0], nel[1], float(nel[0]), float(nel[1]), stiffness=st)
    return eb.CuStructuredMesh3D(*nel, *map(float, nel), stiffness=st)


def _setup(nel, rmin, cons, f, n_level, precision="fp64", springs=None, l_dofs=None, tol=1e-12):
    import torch
    import edge_to_b200 as eb
    mesh = _mesh(nel)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(cons))
    if springs is not None:
        k.set_springs(*springs)
    filt = eb.CuStructuredFilter3D(mesh, rmin) if len(nel) == 3 else eb.CuStructuredFilter2D(mesh, rmin)
    solver = eb.CuMultiGrid(mesh, k, tol=tol, n_level=n_level, maxiter=5000, precision=precision)
    mat = eb.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.3)
    obj = eb.autograd.SIMPObjective(k, solver, filt, mat, torch.as_tensor(f, device="cuda"),
                                    objective="compliance" if l_dofs is None else "displacement",
                                    out_dofs=l_dofs, tol=tol)
    return obj


def _cant_bc(nel):
    g = Grid(nel)
    nelx, nely, nelz = nel
    face = np.array([g.node_id(0, j, k) for j in range(nely + 1) for k in range(nelz + 1)])
    cons = np.sort(np.concatenate([3 * face + d for d in range(3)]))
    edge = np.array([g.node_id(nelx, 0, k) for k in range(nelz + 1)])
    f = np.zeros(g.n_dof)
    f[3 * edge + 1] = -1.0 / edge.shape[0]
    return g, cons, f


def _autograd(obj, rho_np):
    import torch
    rho = torch.as_tensor(rho_np, device="cuda").requires_grad_(True)
    J = obj(rho)
    J.backward()
    return float(J), rho.grad.detach().cpu().numpy()


def _fd_correction(obj, rho_np, idx, h=1e-4):
    """Central differences of J = l.u by correction solves around u0 (see module doc)."""
    import torch
    rho0 = torch.as_tensor(rho_np, device="cuda")
    l = obj.f if obj.l is None else obj.l
    obj._set_design(rho0)
    u0, _ = obj._solve(obj.f, None)
    out = np.empty(len(idx))
    for n, i in enumerate(idx):
        dl = []
        for sgn in (1.0, -1.0):
            r = rho0.clone()
            r[int(i)] += sgn * h
            obj._set_design(r)
            res = obj.f - obj.kernel.dot(u0)
            d, _ = obj._solve(res, None)
            dl.append(float(torch.dot(l, d)))
        out[n] = (dl[0] - dl[1]) / (2 * h)
    return out


def test_compliance_autograd_matches_reference_dr(golden):
    z = golden("grad_cant3d.npz")
    g, cons, f = _cant_bc((32, 16, 16))
    obj = _setup((32, 16, 16), 2.0, cons, f, n_level=3)
    J, grad = _autograd(obj, z["rho"])
    assert abs(J - float(z["compliance"])) / float(z["compliance"]) < 1e-9
    assert np.abs(grad - z["dr"]).max() / np.abs(z["dr"]).max() < 1e-8


def test_compliance_autograd_finite_differences_128x64x64():
    nel = (128, 64, 64)
    g, cons, f = _cant_bc(nel)
    rho = np.random.default_rng(2024).uniform(0.2, 1.0, g.n_el)
    obj = _setup(nel, 2.0, cons, f, n_level=4)
    J, grad = _autograd(obj, rho)
    idx = np.random.default_rng(7).choice(g.n_el, 32, replace=False)
    fd = _fd_correction(obj, rho, idx)
    err = np.abs(fd - grad[idx]) / np.abs(grad[idx])
    assert err.max() < 1e-5, (err.max(), np.median(err))
    # mixed-precision solver: gradient and objective error against FP64
    objm = _setup(nel, 2.0, cons, f, n_level=4, precision="mixed", tol=1e-10)
    Jm, gm = _autograd(objm, rho)
    assert abs(Jm - J) / abs(J) < 1e-9
    assert np.abs(gm - grad).max() / np.abs(grad).max() < 1e-7


def test_mechanism_autograd_against_oracle():
    nel = (40, 20)
    g = Grid(nel)
    f, l, cons, springs = adjoint.inverter_problem(*nel)
    rho = np.random.default_rng(5).uniform(0.2, 1.0, g.n_el)
    H, _ = ops.filter_matrix(g, 1.5)
    ref = adjoint.Objective(g, elements.q4_stiffness(1, 1, 1.0, 0.3), H, f, cons, l=l, springs=springs)
    gref, Jref = ref.gradient(rho)
    obj = _setup(nel, 1.5, cons, f, n_level=2, springs=springs, l_dofs=np.where(l)[0])
    J, grad = _autograd(obj, rho)
    assert abs(J - Jref) / abs(Jref) < 1e-9
    assert np.abs(grad - gref).max() / np.abs(gref).max() < 1e-8


def test_mechanism_autograd_finite_differences_400x200():
    nel = (400, 200)
    g = Grid(nel)
    f, l, cons, springs = adjoint.inverter_problem(*nel)
    rho = np.random.default_rng(11).uniform(0.2, 1.0, g.n_el)
    obj = _setup(nel, 2.0, cons, f, n_level=3, springs=springs, l_dofs=np.where(l)[0])
    J, grad = _autograd(obj, rho)
    assert obj.last.get("adjoint_pcg_iters", 0) > 0
    idx = np.random.default_rng(13).choice(g.n_el, 32, replace=False)
    fd = _fd_correction(obj, rho, idx)
    scale = np.abs(grad).max()
    err = np.abs(fd - grad[idx]) / np.maximum(np.abs(grad[idx]), 1e-3 * scale)
    assert err.max() < 1e-5, (err.max(), np.median(err))


def test_springs_in_products_and_diagonal():
    import torch
    import edge_to_b200 as eb
    nel = (12, 6)
    g = Grid(nel)
    f, l, cons, springs = adjoint.inverter_problem(*nel)
    rng = np.random.default_rng(3)
    E = rng.uniform(0.1, 1.0, g.n_el)
    K = adjoint.stiffness(g, elements.q4_stiffness(1, 1, 1.0, 0.3), E, cons, springs)
    u = rng.standard_normal(g.n_dof)
    k = eb.CuStructuredStiffnessKernel(_mesh(nel))
    k.add_constraints(cons)
    k.set_springs(*springs)
    k.set_rho(torch.as_tensor(E, device="cuda"))
    ut = torch.as_tensor(u, device="cuda")
    ref = K @ u
    for out in (k.dot(ut), k.dot_dense(ut)):
        assert np.abs(out.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-12
    assert np.abs(k.diagonal().cpu().numpy() - K.diagonal()).max() < 1e-12
    k.set_springs([], [])
    assert np.abs(k.dot(ut).cpu().numpy() - ops.assemble(g, elements.q4_stiffness(1, 1, 1.0, 0.3), E, cons) @ u
                  ).max() < 1e-12 * np.abs(ref).max()
