"""Op-level parity of the CUDA path against the reference-generated fixtures and the oracle.

Tolerance: FP64 kernels must match to 1e-12 relative (max-norm), since only the order of
floating-point additions differs from the reference.
"""
import numpy as np
import pytest

from oracle import elements, ops, topopt
from oracle.grid import Grid

pytestmark = pytest.mark.gpu

H_OF = {2: {"even": None, "odd": None, "aniso": (0.5, 0.25)},
        3: {"even": None, "odd": None, "aniso": (0.5, 0.25, 0.5)}}
TOL = 1e-12


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _mesh(dim, nel, h, nu=0.3):
    import edge_to_b200 as eb
    st = lambda x: eb.auto_stiffness(x, 1.0, nu)  # noqa: E731
    h = h or (1.0,) * dim
    if dim == 2:
        return eb.CuStructuredMesh2D(nel[0], nel[1], nel[0] * h[0], nel[1] * h[1], stiffness=st)
    return eb.CuStructuredMesh3D(nel[0], nel[1], nel[2], nel[0] * h[0], nel[1] * h[1], nel[2] * h[2], stiffness=st)


def _cases(golden):
    for dim, fn in ((2, "ops_2d.npz"), (3, "ops_3d.npz")):
        z = golden(fn)
        for tag in ("even", "odd", "aniso"):
            yield dim, tag, z, tuple(int(v) for v in z[f"{tag}_nel"]), H_OF[dim][tag]


def test_matvec_diag_dk_against_reference(golden):
    import torch
    import edge_to_b200 as eb
    for dim, tag, z, nel, h in _cases(golden):
        mesh = _mesh(dim, nel, h)
        k = eb.CuStructuredStiffnessKernel(mesh)
        assert k.uses_transform
        E = torch.as_tensor(z[f"{tag}_E"], device="cuda")
        u = torch.as_tensor(z[f"{tag}_u"], device="cuda")
        k.set_rho(E)
        assert rel(k.dot(u).cpu(), z[f"{tag}_matvec_nocon"]) < TOL, (dim, tag)
        assert rel(k.dot_dense(u).cpu(), z[f"{tag}_matvec_nocon"]) < TOL, (dim, tag)
        k.add_constraints(z[f"{tag}_cons"])
        assert rel(k.dot(u).cpu(), z[f"{tag}_matvec"]) < TOL, (dim, tag)
        assert rel(k.dot_dense(u).cpu(), z[f"{tag}_matvec"]) < TOL, (dim, tag)
        assert rel(k.diagonal().cpu(), z[f"{tag}_diag"]) < TOL, (dim, tag)
        assert rel(k.process_grad(u).cpu(), z[f"{tag}_dk"]) < TOL, (dim, tag)


@pytest.mark.parametrize("nel", [(33, 17), (64, 31), (130, 3), (5, 70), (7, 5, 3), (40, 9, 33), (9, 33, 65), (3, 3, 130)])
def test_matvec_ragged_sizes(nel):
    """Tile edges: sizes that are not multiples of the 31-node / 7-column tiles."""
    import torch
    import edge_to_b200 as eb
    dim = len(nel)
    rng = np.random.default_rng(sum(nel))
    mesh = _mesh(dim, nel, None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    g = Grid(nel)
    E = rng.uniform(1e-3, 1, g.n_el)
    E[rng.random(g.n_el) < 0.2] = 1e-9
    u = rng.standard_normal(g.n_dof)
    cons = np.where(rng.random(g.n_dof) < 0.1)[0]
    k.set_rho(torch.as_tensor(E, device="cuda"))
    k.add_constraints(cons)
    K0 = elements.q4_stiffness(1, 1, 1, 0.3) if dim == 2 else elements.hex8_stiffness(1, 1, 1, 1, 0.3)
    ref = ops.assemble(g, K0, E, cons) @ u
    ut = torch.as_tensor(u, device="cuda")
    assert rel(k.dot(ut).cpu(), ref) < TOL
    assert rel(k.dot_dense(ut).cpu(), ref) < TOL


def test_filter_against_reference(golden):
    import torch
    import edge_to_b200 as eb
    n = 0
    for dim, tag, z, nel, h in _cases(golden):
        mesh = _mesh(dim, nel, h)
        for key in z.files:
            if key.startswith(f"{tag}_filt") and key.endswith("_in"):
                r = float(key[len(tag) + 5:-3])
                f = (eb.CuStructuredFilter2D if dim == 2 else eb.CuStructuredFilter3D)(mesh, r)
                x = torch.as_tensor(z[key], device="cuda")
                assert rel(f.dot(x).cpu(), z[f"{tag}_filt{r}_H"]) < TOL
                assert rel(f.T.dot(x).cpu(), z[f"{tag}_filt{r}_HT"]) < TOL
                n += 1
    assert n >= 8


def test_transfers_against_oracle(golden):
    import torch
    from edge_to_b200 import _lib
    for dim, tag, z, nel, h in _cases(golden):
        g = Grid(nel)
        v = z[f"{tag}_restrict_in"]
        out = torch.empty(g.coarse().n_dof, dtype=torch.float64, device="cuda")
        _lib.call("edge_restrict", dim, _lib.int_array(list(nel) + [1] * (3 - dim)),
                  _lib.ptr(torch.as_tensor(v, device="cuda")), _lib.ptr(out), _lib.stream_ptr())
        assert rel(out.cpu(), ops.restriction_matrix(g, "gpu") @ v) < TOL
        vc = z[f"{tag}_prolong_in"]
        outf = torch.empty(g.n_dof, dtype=torch.float64, device="cuda")
        _lib.call("edge_prolong", dim, _lib.int_array(list(nel) + [1] * (3 - dim)),
                  _lib.ptr(torch.as_tensor(vc, device="cuda")), _lib.ptr(outf), _lib.stream_ptr())
        assert rel(outf.cpu(), z[f"{tag}_prolong"]) < TOL


def test_oc_update_against_reference(golden):
    import torch
    import edge_to_b200 as eb
    for dim, fn in ((2, "ops_2d.npz"), (3, "ops_3d.npz")):
        z = golden(fn)
        nel = tuple(int(v) for v in z["even_nel"])
        mesh = _mesh(dim, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        mat = eb.SingleMaterial(void=1e-9, penalty=3.0, volume_fraction=0.4)
        opt = eb.CuTopOpt(mesh, mat, k, eb.CuMultiGrid(mesh, k, n_level=1), None, verbose=False)
        out = opt.update_design(torch.as_tensor(z["even_oc_rho"], device="cuda"),
                                torch.as_tensor(z["even_oc_df"], device="cuda"))
        np.testing.assert_array_equal(out.cpu().numpy(), z["even_oc_out"].reshape(-1))


def test_oc_update_edge_cases():
    """All-zero sensitivities take the 1e-3 fallback; random large problems match the oracle."""
    import torch
    import edge_to_b200 as eb
    mesh = _mesh(2, (50, 30), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    mat = eb.SingleMaterial(void=1e-9, volume_fraction=0.3)
    opt = eb.CuTopOpt(mesh, mat, k, eb.CuMultiGrid(mesh, k, n_level=1), None, verbose=False)
    rng = np.random.default_rng(3)
    A = float(mesh.As[0])
    for df in (np.zeros(1500), -rng.uniform(0, 5, 1500) ** 3, rng.standard_normal(1500)):
        rho = rng.uniform(0, 1, 1500)
        out = opt.update_design(torch.as_tensor(rho, device="cuda"), torch.as_tensor(df, device="cuda"))
        ref, lam, steps = topopt.oc_update(rho, df, A, A * 1500, 0.3, 0.2)
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
        assert opt.last_stats["oc_steps"] == steps


def test_pcg_tracks_oracle_iterations():
    """The GPU GMG-PCG follows the oracle's FP64 iteration (GPU semantics) step for step."""
    import torch
    import edge_to_b200 as eb
    for nel, nl in (((32, 16), 3), ((16, 8, 8), 2)):
        dim = len(nel)
        p = (topopt.mbb_problem(*nel, vf=0.5, mg_kwargs=dict(tol=1e-10, n_level=nl, maxiter=500, variant="gpu"))
             if dim == 2 else
             topopt.cantilever_problem(*nel, vf=0.3, mg_kwargs=dict(tol=1e-10, n_level=nl, maxiter=500,
                                                                     variant="gpu")))
        rng = np.random.default_rng(1)
        rho = rng.uniform(0.1, 1.0, p.grid.n_el)
        E = np.clip(ops.filter_apply(p.H, rho) ** 3, 1e-9, 1)
        K = ops.assemble(p.grid, p.K0, E, p.cons)
        x_ref, res_ref = p.solver.solve(K, p.f, use_last=False)
        mesh = _mesh(dim, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        cons = np.zeros(p.grid.n_dof, dtype=bool)
        cons[p.cons] = True
        k.add_constraints(np.where(cons)[0])
        k.set_rho(torch.as_tensor(E, device="cuda"))
        s = eb.CuMultiGrid(mesh, k, tol=1e-10, n_level=nl, maxiter=500)
        x, res = s.solve(torch.as_tensor(p.f, device="cuda"), use_last=False)
        assert s.last_iters == p.solver.pcg_iters[-1], (s.last_iters, p.solver.pcg_iters[-1])
        assert rel(x.cpu(), x_ref) < 1e-9
        assert res < 1e-10


def test_galerkin_levels_against_reference(golden):
    """Level-1 and level-2 Galerkin operators equal the reference's CSR matrices."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    for dim, fn in ((2, "ops_2d.npz"), (3, "ops_3d.npz")):
        z = golden(fn)
        nel = tuple(int(v) for v in z["even_nel"])
        mesh = _mesh(dim, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        k.set_rho(torch.as_tensor(z["even_E"], device="cuda"))
        k.add_constraints(z["even_cons"])
        s = eb.CuMultiGrid(mesh, k, n_level=2)
        s._configure()
        _lib.call("edge_mg_setup", k.handle)
        for lvl, key in ((1, "even_A1"), (2, "even_A2")):
            ref = z[key]
            out = torch.empty(ref.shape, dtype=torch.float64, device="cuda")
            _lib.call("edge_mg_level_dense", k.handle, lvl, _lib.ptr(out), ref.shape[0])
            assert rel(out.cpu(), ref) < TOL, (dim, lvl)


def test_galerkin_against_oracle_ragged():
    """Odd extents and boundary conditions: the GPU Galerkin chain equals R A R^T of the oracle."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    for nel in ((9, 7), (6, 5, 7)):
        dim = len(nel)
        g = Grid(nel)
        rng = np.random.default_rng(11)
        E = rng.uniform(1e-3, 1, g.n_el)
        cons = np.where(rng.random(g.n_dof) < 0.1)[0]
        K0 = elements.q4_stiffness(1, 1, 1, 0.3) if dim == 2 else elements.hex8_stiffness(1, 1, 1, 1, 0.3)
        A = ops.assemble(g, K0, E, cons)
        mesh = _mesh(dim, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        k.set_rho(torch.as_tensor(E, device="cuda"))
        k.add_constraints(cons)
        s = eb.CuMultiGrid(mesh, k, n_level=2)
        s._configure()
        _lib.call("edge_mg_setup", k.handle)
        gg = g
        for lvl in (1, 2):
            A = ops.galerkin(A, gg)
            gg = gg.coarse()
            ref = A.toarray()
            out = torch.empty(ref.shape, dtype=torch.float64, device="cuda")
            _lib.call("edge_mg_level_dense", k.handle, lvl, _lib.ptr(out), ref.shape[0])
            assert rel(out.cpu(), ref) < TOL, (nel, lvl)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_galerkin_axis_passes_equal_direct_product(precision):
    """The 3-D stencil-level Galerkin products as three one-axis passes (the default) equal the
    direct R A R^T over the fine neighbourhoods on every coarse level of ragged grids with BCs:
    to FP64 rounding, and to FP32 rounding for the mixed path's FP32 stencils."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    for nel in ((12, 10, 14), (16, 9, 12)):
        g = Grid(nel)
        rng = np.random.default_rng(5)
        E = rng.uniform(1e-3, 1, g.n_el)
        cons = np.where(rng.random(g.n_dof) < 0.05)[0]
        mesh = _mesh(3, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        k.set_rho(torch.as_tensor(E, device="cuda"))
        k.add_constraints(cons)
        s = eb.CuMultiGrid(mesh, k, n_level=3, precision=precision, autotune=False, tune_sweeps=False)
        s._configure()
        dense = {}
        for axis in (0, 1):
            _lib.call("edge_set_galerkin_axis", k.handle, axis)
            _lib.call("edge_mg_setup", k.handle)
            for lvl in (2, 3):
                gg = g
                for _ in range(lvl):
                    gg = gg.coarse()
                nd = gg.n_dof
                out = torch.empty((nd, nd), dtype=torch.float64, device="cuda")
                _lib.call("edge_mg_level_dense", k.handle, lvl, _lib.ptr(out), nd)
                dense[axis, lvl] = out.cpu().numpy()
        _lib.call("edge_set_galerkin_axis", k.handle, 1)
        for lvl in (2, 3):
            a, b = dense[1, lvl], dense[0, lvl]
            assert np.abs(b).max() > 0
            assert rel(a, b) < (1e-13 if precision == "fp64" else 1e-6), (nel, lvl, rel(a, b))


def test_jacobi_sweep_entry_point_against_oracle():
    """edge_jacobi_sweep (the V-cycle's damped-Jacobi smoother on its own) on level 0 and on a
    Galerkin level of a ragged grid with BCs equals n_step sweeps x + omega (b - A x) / diag(A)
    with the oracle's assembled and Galerkin matrices."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    for nel in ((9, 7), (6, 5, 7)):
        dim = len(nel)
        g = Grid(nel)
        rng = np.random.default_rng(23)
        E = rng.uniform(1e-3, 1, g.n_el)
        cons = np.where(rng.random(g.n_dof) < 0.1)[0]
        K0 = elements.q4_stiffness(1, 1, 1, 0.3) if dim == 2 else elements.hex8_stiffness(1, 1, 1, 1, 0.3)
        A0 = ops.assemble(g, K0, E, cons)
        mesh = _mesh(dim, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        k.set_rho(torch.as_tensor(E, device="cuda"))
        k.add_constraints(cons)
        s = eb.CuMultiGrid(mesh, k, n_level=2)
        s._configure()
        _lib.call("edge_mg_setup", k.handle)
        for lvl, A in ((0, A0), (1, ops.galerkin(A0, g))):
            A = A.toarray()
            n = A.shape[0]
            x = rng.standard_normal(n)
            b = rng.standard_normal(n)
            want = x.copy()
            for _ in range(3):
                want = want + 0.45 * (b - A @ want) / np.diag(A)
            out = torch.empty(n, dtype=torch.float64, device="cuda")
            xd, bd = torch.as_tensor(x, device="cuda"), torch.as_tensor(b, device="cuda")
            _lib.call("edge_jacobi_sweep", k.handle, lvl, _lib.ptr(xd), _lib.ptr(bd), 0.45, 3, _lib.ptr(out))
            assert rel(out.cpu(), want) < 1e-12, (nel, lvl)


@pytest.mark.parametrize("nel", [(4, 4, 4), (7, 5, 3), (40, 9, 33), (9, 33, 65), (3, 3, 130), (20, 20, 47)])
def test_fine_kernel_variants_agree(nel):
    """TMA-staged, cooperative-load and dense kernels give the same K(E) u (ragged tiles, BCs)."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    rng = np.random.default_rng(sum(nel) + 1)
    mesh = _mesh(3, nel, None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    g = Grid(nel)
    E = rng.uniform(1e-3, 1, g.n_el)
    u = rng.standard_normal(g.n_dof)
    cons = np.where(rng.random(g.n_dof) < 0.1)[0]
    k.set_rho(torch.as_tensor(E, device="cuda"))
    k.add_constraints(cons)
    ut = torch.as_tensor(u, device="cuda")
    ref = ops.assemble(g, elements.hex8_stiffness(1, 1, 1, 1, 0.3), E, cons) @ u
    a = k.dot(ut).cpu().clone()
    _lib.call("edge_set_tma", k.handle, 0)
    b = k.dot(ut).cpu().clone()
    _lib.call("edge_set_tma", k.handle, 1)
    assert rel(a, ref) < TOL and rel(b, ref) < TOL


def test_fp32_operator_accuracy():
    """The mixed-precision solver's FP32 operator agrees with FP64 to single-precision accuracy."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    for nel in ((40, 9, 33), (64, 32)):
        dim = len(nel)
        rng = np.random.default_rng(5)
        mesh = _mesh(dim, nel, None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        g = Grid(nel)
        k.set_rho(torch.as_tensor(rng.uniform(1e-3, 1, g.n_el), device="cuda"))
        k.add_constraints(np.where(rng.random(g.n_dof) < 0.05)[0])
        u = torch.as_tensor(rng.standard_normal(g.n_dof), device="cuda")
        a = k.dot(u).clone()
        b = torch.empty_like(a)
        _lib.call("edge_matvec_f32", k.handle, _lib.ptr(u), _lib.ptr(b))
        assert rel(b.cpu(), a.cpu()) < 1e-5


@pytest.mark.parametrize("nel", [(4, 4, 4), (7, 5, 3), (40, 9, 33), (9, 33, 65), (3, 3, 130), (20, 20, 47), (66, 17, 31)])
def test_fp32_tile_variants_agree(nel):
    """Every FP32 fine-kernel tile (k_fine3_tma 0-4, packed-pair k_fine3_pk 5-8, its cube form
    k_fine3_cube 9-14) gives K(E) u to single precision on ragged grids with boundary
    conditions and void elements."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    rng = np.random.default_rng(sum(nel) + 7)
    mesh = _mesh(3, nel, None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    g = Grid(nel)
    E = rng.uniform(1e-3, 1, g.n_el)
    E[rng.random(g.n_el) < 0.2] = 1e-9
    u = rng.standard_normal(g.n_dof)
    cons = np.where(rng.random(g.n_dof) < 0.1)[0]
    k.set_rho(torch.as_tensor(E, device="cuda"))
    k.add_constraints(cons)
    ref = ops.assemble(g, elements.hex8_stiffness(1, 1, 1, 1, 0.3), E, cons) @ u
    ut = torch.as_tensor(u, device="cuda")
    outs = []
    assert _lib.lib().edge_uses_cube_form(k.handle) == 1
    for v in range(15):
        for bps in (2, 16):
            _lib.call("edge_set_fine_tile", k.handle, v, bps)
            b = torch.empty_like(ut)
            _lib.call("edge_matvec_f32", k.handle, _lib.ptr(ut), _lib.ptr(b))
            outs.append(b.cpu().numpy())
            assert rel(outs[-1], ref) < 2e-6, (v, bps)
    for o in outs[10:]:
        assert rel(o, outs[8]) < 1e-6


def test_packed_kernel_in_mixed_solve():
    """Mixed-precision PCG with the packed-pair FP32 kernel follows the k_fine3_tma run."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(9)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (32, 16, 16), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=3, maxiter=500, precision="mixed", autotune=False,
                       tune_sweeps=False)
    res = []
    for v in (4, 5, 8, 9, 10):
        _lib.call("edge_set_fine_tile", k.handle, v, 8)
        x, r = s.solve(torch.as_tensor(p.f, device="cuda"), use_last=False)
        res.append((x.cpu().numpy().copy(), s.last_iters, r))
    # the variants sum the element products in different FP32 orders: the PCG iteration count at
    # rtol 1e-8 moves by a few (42-45 here), the converged solutions agree
    for x, it, r in res[1:]:
        assert abs(it - res[0][1]) <= max(2, res[0][1] // 10) and r < 1e-8
        assert rel(x, res[0][0]) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stencil_kernels_agree_in_solve(precision):
    """The one-thread-per-node, two-nodes-per-thread, four-lanes-per-node and tile-major
    coarse stencil kernels give the same PCG run (same iteration count, solutions equal to
    rounding)."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(11)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (32, 16, 16), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=3, maxiter=500, precision=precision, autotune=False,
                       tune_sweeps=False)
    res = []
    _lib.call("edge_set_coarse_bf16", k.handle, 0)  # FP32 stencils first
    for qmax, pair in ((0, -1), (1 << 40, -1), (0, 0)):
        _lib.call("edge_set_stencil_quad", k.handle, qmax)
        _lib.call("edge_set_stencil_pair", k.handle, pair)
        x, r = s.solve(torch.as_tensor(p.f, device="cuda"), use_last=False)
        res.append((x.cpu().numpy().copy(), s.last_iters, r))
    # the mixed path declares convergence only at an FP64 true-residual check: a rounding
    # difference can move the stop from one check to the next (44 against 48 iterations here)
    tol_it = 0 if precision == "fp64" else 4
    x0, it0, r0 = res[0]
    for x1, it1, r1 in res[1:]:
        assert abs(it0 - it1) <= tol_it and r0 < 1e-8 and r1 < 1e-8
        assert rel(x1, x0) < (1e-12 if precision == "fp64" else 1e-7)
    if precision == "mixed":
        # BF16 stencil copies: one node per thread and two nodes per thread (4-byte pair loads)
        _lib.call("edge_set_coarse_bf16", k.handle, 1)
        bf = []
        for pair in (-1, 0):
            _lib.call("edge_set_stencil_quad", k.handle, 0)
            _lib.call("edge_set_stencil_pair", k.handle, pair)
            x, r = s.solve(torch.as_tensor(p.f, device="cuda"), use_last=False)
            bf.append((x.cpu().numpy().copy(), s.last_iters, r))
        (xa, ia, ra), (xb, ib, rb) = bf
        assert abs(ia - ib) <= tol_it and abs(ia - it0) <= tol_it and ra < 1e-8 and rb < 1e-8
        assert rel(xb, xa) < 1e-7 and rel(xa, x0) < 1e-6
        # tile-major BF16 pair copies with packed products (every coarse level here): the same
        # terms in the same order as the pair kernel, rounded by the packed instructions
        _lib.call("edge_set_stencil_tiled", k.handle, 0)
        xt, rt = s.solve(torch.as_tensor(p.f, device="cuda"), use_last=False)
        it_ = s.last_iters
        _lib.call("edge_set_stencil_tiled", k.handle, 200000)
        _lib.call("edge_set_stencil_pair", k.handle, 200000)
        _lib.call("edge_set_stencil_quad", k.handle, 40000)
        assert abs(it_ - ib) <= tol_it and rt < 1e-8 and rel(xt.cpu().numpy(), xb) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_and_host_loop_agree(precision):
    """One CUDA-graph solve (while node over the PCG iteration, if node for the residual
    replacement) and the host-driven loop run the same launches: same iteration count and
    true-residual count, solutions equal to rounding; so does the graph with programmatic
    dependent launch; a second graph solve with a changed tolerance captures again."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(5)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (32, 16, 16), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    f = torch.as_tensor(p.f, device="cuda")
    out = {}
    for graph in (False, True):
        s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=3, maxiter=500, precision=precision, autotune=False,
                           graph=graph, tune_sweeps=False)
        x, r = s.solve(f, use_last=False)
        out[graph] = (x.cpu().numpy().copy(), s.last_iters, s.stats()["true_residuals"], r)
    (x0, it0, t0, r0), (x1, it1, t1, r1) = out[False], out[True]
    assert it0 == it1 and t0 == t1 and r0 < 1e-8 and r1 < 1e-8
    assert rel(x1, x0) < 1e-12
    # the graph with programmatic dependent launch: the same launches, overlapped
    _lib.call("edge_set_pdl", k.handle, 1)
    x3, r3 = s.solve(f, use_last=False)
    assert s.last_iters == it1 and rel(x3.cpu().numpy(), x1) < 1e-12
    _lib.call("edge_set_pdl", k.handle, 0)
    s.tol = 1e-6
    x2, r2 = s.solve(f, use_last=False)
    assert r2 < 1e-6 and s.last_iters < it1


def test_fused_fine_launches_agree():
    """Mixed precision with the cube kernel and one sweep per level: the fused fine launches
    (the first Jacobi sweep computed inside the residual launch and the last-sweep launch, the
    search direction formed inside the product with p ping-ponging between two buffers by
    iteration parity) against the same arithmetic as separate launches: iteration counts
    within 2, both solutions within the tolerance of the FP64 solve; the fused graph solve
    and the fused host-driven loop are the same launches (identical iterates)."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(13)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (32, 16, 16), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    f = torch.as_tensor(p.f, device="cuda")
    s64 = eb.CuMultiGrid(mesh, k, tol=1e-11, n_level=3, maxiter=2000, precision="fp64", autotune=False)
    x64 = s64.solve(f, use_last=False)[0].cpu().numpy().copy()
    out = {}
    for fuse, graph in ((0, True), (1, True), (1, False)):
        s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=3, maxiter=500, precision="mixed", autotune=False,
                           tune_sweeps=False, graph=graph)
        s._configure()
        _lib.call("edge_set_fine_tile", k.handle, 10, 8)
        _lib.call("edge_mg_set_sweeps", k.handle, _lib.int_array([1, 1, 1]), 3)
        _lib.call("edge_set_fuse", k.handle, fuse)
        x, r = s.solve(f, use_last=False)
        out[(fuse, graph)] = (x.cpu().numpy().copy(), s.last_iters, r)
    _lib.call("edge_set_fuse", k.handle, 1)
    (xu, iu, ru), (xf, i_f, rf), (xh, ih, rh) = out[(0, True)], out[(1, True)], out[(1, False)]
    print("iterations unfused / fused / fused host loop", iu, i_f, ih)
    assert ru < 1e-8 and rf < 1e-8 and rh < 1e-8
    assert abs(iu - i_f) <= 2 and i_f > 3
    assert rel(xu, x64) < 1e-6 and rel(xf, x64) < 1e-6
    assert ih == i_f and rel(xh, xf) < 1e-12


def test_fused_xr_update_agrees():
    """Mixed precision, fixed smoother weight: the PCG's x/r update folded into the next
    iteration's first fine launch (residual, written into a ping-pong pair, with r.r) and
    search-direction launch (solution) against the separate update launch: the same
    arithmetic except the order of the r.r sum, so iteration counts within 1 and solutions
    within the tolerance of the FP64 solve; the graph solve and the host-driven loop are the
    same launches (identical iterates); warm-started solves (a pending update from the
    previous solve must not leak into the next) agree as well."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(17)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (32, 16, 16), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    f = torch.as_tensor(p.f, device="cuda")
    s64 = eb.CuMultiGrid(mesh, k, tol=1e-11, n_level=3, maxiter=2000, precision="fp64", autotune=False)
    x64 = s64.solve(f, use_last=False)[0].cpu().numpy().copy()
    out = {}
    for xr, graph in ((0, True), (1, True), (1, False)):
        s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=3, maxiter=500, precision="mixed", autotune=False,
                           tune_sweeps=False, graph=graph, mixed_omega="max")
        s._configure()
        _lib.call("edge_set_fine_tile", k.handle, 10, 8)
        _lib.call("edge_mg_set_sweeps", k.handle, _lib.int_array([1, 1, 1]), 3)
        _lib.call("edge_set_fuse_xr", k.handle, xr)
        x, r = s.solve(f, use_last=False)
        it0 = s.last_iters
        x0 = x.cpu().numpy().copy()
        # a second solve warm-started from a perturbed solution
        s.last_x0 = x * (1.0 + 1e-3 * torch.cos(torch.arange(x.numel(), device="cuda", dtype=torch.float64)))
        x2, r2 = s.solve(f, use_last=True)
        out[(xr, graph)] = (x0, it0, r, x2.cpu().numpy().copy(), s.last_iters, r2)
    _lib.call("edge_set_fuse_xr", k.handle, 1)
    a, b, c = out[(0, True)], out[(1, True)], out[(1, False)]
    print("iterations separate / fused / fused host loop", a[1], b[1], c[1], "warm", a[4], b[4], c[4])
    for o in (a, b, c):
        assert o[2] < 1e-8 and o[5] < 1e-8
        assert rel(o[0], x64) < 1e-6 and rel(o[3], x64) < 1e-6
    assert abs(a[1] - b[1]) <= 1 and abs(a[4] - b[4]) <= 1 and b[1] > 3
    assert c[1] == b[1] and c[4] == b[4]
    assert rel(c[0], b[0]) < 1e-12 and rel(c[3], b[3]) < 1e-12


@pytest.mark.parametrize("sweeps", [(1, 1, 1, 1), (1, 2, 3, 1)])
def test_persistent_vcycle_tail_agrees(sweeps):
    """Mixed precision: the V-cycle below level 1 as one persistent cooperative launch
    (edge_set_tail 2) against one launch per step (edge_set_tail 0, the default), with one and
    with several sweeps per level: the same arithmetic per node except for the summation order
    of the small levels' stencils, so iteration counts within 1 and solutions within 1e-7;
    graph and host-driven loops agree exactly."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(64, 32, 32, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=4, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(17)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (64, 32, 32), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    f = torch.as_tensor(p.f, device="cuda")
    out = {}
    for tail, graph in ((0, True), (2, True), (2, False)):
        s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=4, maxiter=500, precision="mixed", autotune=False,
                           tune_sweeps=False, graph=graph)
        s._configure()
        _lib.call("edge_mg_set_sweeps", k.handle, _lib.int_array(list(sweeps)), 4)
        _lib.call("edge_set_tail", k.handle, tail)
        x, r = s.solve(f, use_last=False)
        out[(tail, graph)] = (x.cpu().numpy().copy(), s.last_iters, r)
    _lib.call("edge_set_tail", k.handle, 0)
    (x0, i0, r0), (x1, i1, r1), (xh, ih, rh) = out[(0, True)], out[(2, True)], out[(2, False)]
    print("iterations per-launch / persistent / persistent host loop", i0, i1, ih)
    assert r0 < 1e-8 and r1 < 1e-8 and rh < 1e-8
    assert abs(i0 - i1) <= 1
    assert rel(x1, x0) < 1e-7
    assert ih == i1 and rel(xh, x1) < 1e-12


def test_residual_recurrence_precisions_agree():
    """Mixed precision with the residual recurrence stored in FP32 (default) and in FP64: both
    meet the tolerance on the FP64 true residual, take about the same iterations and give the
    same solution to the tolerance."""
    import torch
    import edge_to_b200 as eb
    from edge_to_b200 import _lib
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(9)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    mesh = _mesh(3, (32, 16, 16), None)
    k = eb.CuStructuredStiffnessKernel(mesh)
    k.add_constraints(np.asarray(p.cons))
    k.set_rho(torch.as_tensor(E, device="cuda"))
    s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=3, maxiter=500, precision="mixed", autotune=False,
                       tune_sweeps=False)
    f = torch.as_tensor(p.f, device="cuda")
    out = {}
    for r32 in (1, 0):
        _lib.call("edge_set_residual32", k.handle, r32)
        x, r = s.solve(f, use_last=False)
        out[r32] = (x.cpu().numpy().copy(), s.last_iters, r)
    (x1, i1, r1), (x0, i0, r0) = out[1], out[0]
    assert r1 < 1e-8 and r0 < 1e-8 and abs(i1 - i0) <= 3
    assert rel(x1, x0) < 1e-6


def test_sweep_autotuner_mixed():
    """The mixed-precision solver picks per-level sweep counts on its first warm-started solve;
    the solve still meets the tolerance and matches a tight FP64 solve; the FP64 solver keeps
    n_smooth."""
    import torch
    import edge_to_b200 as eb
    p = topopt.cantilever_problem(32, 16, 16, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=3, maxiter=500,
                                                                       variant="gpu"))
    rng = np.random.default_rng(3)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    f = torch.as_tensor(p.f, device="cuda")
    xs = {}
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-8)):
        mesh = _mesh(3, (32, 16, 16), None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        k.add_constraints(np.asarray(p.cons))
        k.set_rho(torch.as_tensor(E, device="cuda"))
        s = eb.CuMultiGrid(mesh, k, tol=tol, n_level=3, maxiter=500, precision=prec, autotune=False)
        x, r = s.solve(f, use_last=False)
        assert r < tol and s.sweeps is None  # a cold solve uses n_smooth
        k.set_rho(torch.as_tensor(E * 0.9, device="cuda"))  # the next design
        x, r = s.solve(f * 1.0, use_last=True)
        assert r < tol
        xs[prec] = (x.cpu().numpy(), s.sweeps)
    assert xs["fp64"][1] is None
    sw = xs["mixed"][1]
    assert sw is not None and len(sw["per_level"]) == 3 and all(1 <= v <= 3 for v in sw["per_level"])
    assert rel(xs["mixed"][0], xs["fp64"][0]) < 1e-5


def test_precision_switch_on_one_problem():
    """An FP64 solve followed by a mixed-precision solve on the same kernel handle: the mixed
    solve converges like on a fresh handle (buffers shared by both precisions are cleared)."""
    import torch
    import edge_to_b200 as eb
    p = topopt.cantilever_problem(16, 8, 8, vf=0.3, mg_kwargs=dict(tol=1e-8, n_level=2, maxiter=500,
                                                                     variant="gpu"))
    rng = np.random.default_rng(4)
    E = np.clip(rng.uniform(0.05, 1.0, p.grid.n_el) ** 3, 1e-9, 1)
    f = torch.as_tensor(p.f, device="cuda")
    out = []
    for first64 in (False, True):
        mesh = _mesh(3, (16, 8, 8), None)
        k = eb.CuStructuredStiffnessKernel(mesh)
        k.add_constraints(np.asarray(p.cons))
        k.set_rho(torch.as_tensor(E, device="cuda"))
        if first64:
            eb.CuMultiGrid(mesh, k, tol=1e-10, n_level=2, maxiter=500, precision="fp64", autotune=False).solve(
                f, use_last=False)
        s = eb.CuMultiGrid(mesh, k, tol=1e-8, n_level=2, maxiter=500, precision="mixed", autotune=False,
                           tune_sweeps=False)
        x, r = s.solve(f, use_last=False)
        out.append((x.cpu().numpy(), s.last_iters, r))
    assert out[1][2] < 1e-8 and out[1][1] == out[0][1]
    assert rel(out[1][0], out[0][0]) < 1e-12
