"""Unstructured meshes on the GPU: the CUDA operator, diagonal, sensitivities, KD-tree filter
and CG of CuUniformStiffnessKernel / CuGeneralStiffnessKernel / CuGeneralFilter / CuCG against
fixtures made by running the reference's GeneralMesh, UniformStiffnessKernel /
GeneralStiffnessKernel and GeneralFilter (tests/golden/general.npz: T3, T3+Q4, Tet4 of both
orientations, distorted hex8), and against direct solves of the oracle's assembled matrix.

Tolerances: products, diagonal, dk and filter 1e-12 relative (FP64, different summation
order); CG solutions 1e-7 of the direct solve at tol 1e-11."""
import numpy as np
import pytest

from oracle import general

pytestmark = pytest.mark.gpu

TAGS = ("tri", "mixed", "tet", "hex")


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _mesh(z, tag):
    import edge_to_b200 as eb
    conn = general.connectivity(z[f"{tag}_sizes"], z[f"{tag}_flat"])
    return eb.CuGeneralMesh(z[f"{tag}_nodes"], conn, stiffness=lambda x: eb.auto_stiffness(x, 1.0, 0.3)), conn


def _kernel(mesh):
    import edge_to_b200 as eb
    return eb.CuUniformStiffnessKernel(mesh) if mesh.is_uniform else eb.CuGeneralStiffnessKernel(mesh)


@pytest.mark.parametrize("tag", TAGS)
def test_general_operator_against_reference(golden, tag):
    import torch
    z = golden("general.npz")
    mesh, _ = _mesh(z, tag)
    k = _kernel(mesh)
    k.set_rho(torch.as_tensor(z[f"{tag}_rho"], device="cuda"))
    u = torch.as_tensor(z[f"{tag}_u"], device="cuda")
    assert rel(k.dot(u).cpu().numpy(), z[f"{tag}_matvec"]) < 1e-12
    k.add_constraints(z[f"{tag}_cons"])
    assert rel((k @ u).cpu().numpy(), z[f"{tag}_matvec_con"]) < 1e-12
    assert rel(k.diagonal().cpu().numpy(), z[f"{tag}_diag_con"]) < 1e-12
    dk = k.process_grad(torch.as_tensor(z[f"{tag}_U"], device="cuda"))
    assert rel(dk.cpu().numpy(), z[f"{tag}_dk"]) < 1e-12
    # the assembled form equals the product
    K = k.construct(k.rho)
    assert rel((K @ u.unsqueeze(1)).squeeze(1).cpu().numpy(), z[f"{tag}_matvec_con"]) < 1e-12


@pytest.mark.parametrize("tag", TAGS)
def test_general_filter_against_reference(golden, tag):
    import torch
    import edge_to_b200 as eb
    z = golden("general.npz")
    mesh, _ = _mesh(z, tag)
    f = eb.CuGeneralFilter(mesh, 1.6)
    x = torch.as_tensor(z[f"{tag}_fx"], device="cuda")
    assert rel(f.kernel.to_dense().cpu().numpy(), z[f"{tag}_H"]) < 1e-14
    assert rel(f.dot(x).cpu().numpy(), z[f"{tag}_Hx"]) < 1e-12
    assert rel((f.T @ x).cpu().numpy(), z[f"{tag}_HTx"]) < 1e-12


def test_general_kernel_errors(golden):
    import torch
    import edge_to_b200 as eb
    z = golden("general.npz")
    mesh, _ = _mesh(z, "tri")
    with pytest.raises(ValueError):
        eb.CuGeneralStiffnessKernel(mesh)   # uniform mesh: the reference points to the uniform kernel
    mixed, _ = _mesh(z, "mixed")
    with pytest.raises(ValueError):
        eb.CuUniformStiffnessKernel(mixed)
    k = eb.CuUniformStiffnessKernel(mesh)
    with pytest.raises(ValueError):
        k.dot(torch.zeros(k.shape[0], dtype=torch.float64, device="cuda"))  # rho not set
    k.set_rho(torch.ones(mesh.n_elements, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        k.dot(torch.zeros(k.shape[0] + 1, dtype=torch.float64, device="cuda"))
    with pytest.raises(NotImplementedError):
        k.dot([0.0] * k.shape[0])


@pytest.mark.parametrize("tag", TAGS)
def test_general_cg_matches_direct_solve(golden, tag):
    """CuCG on a general mesh (the reference pairs general meshes with CG): a loaded,
    constrained problem solved to tol 1e-11 against scipy's direct solve of the oracle's
    assembled K; warm start from the solution converges at once."""
    import scipy.sparse.linalg as sla
    import torch
    import edge_to_b200 as eb
    z = golden("general.npz")
    mesh, conn = _mesh(z, tag)
    k = _kernel(mesh)
    dof = mesh.dof
    rho = z[f"{tag}_rho"]
    k.set_rho(torch.as_tensor(rho, device="cuda"))
    cons = z[f"{tag}_cons"]
    k.add_constraints(cons)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(k.shape[0])
    f[cons] = 0.0
    Ks = general.element_matrices(z[f"{tag}_Kflat"], z[f"{tag}_sizes"], dof)
    K = general.assemble(k.shape[0], dof, conn, Ks, rho, cons)
    xd = sla.spsolve(K.tocsc(), f)
    s = eb.CuCG(k, maxiter=20000, tol=1e-11)
    x, r = s.solve(torch.as_tensor(f, device="cuda"), use_last=True)
    assert r < 1e-10
    assert rel(x.cpu().numpy(), xd) < 1e-7
    it_cold = s.last_iters
    x2, r2 = s.solve(torch.as_tensor(f, device="cuda"), use_last=True)
    assert r2 < 1e-10 and s.last_iters <= max(2, it_cold // 10)
