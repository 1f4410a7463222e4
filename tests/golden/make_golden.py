"""Generate the golden fixtures in this folder by running the reference's own CPU path.

The reference (ahnobari/EDGE-TO) is pure Python + Numba.  Its package root imports
cupy, cupyx, scikit-sparse, matplotlib, vtk and k3d at import time
(EDGETO/__init__.py:4-10), none of which exist in this image, so this script
injects inert stand-in modules for those names before importing it.  Nothing in the
reference is copied or modified; only its CPU classes are exercised:
``StructuredMesh2D/3D`` (geom/_mesh.py:19-78), ``StructuredStiffnessKernel``
(kernels/_processors.py:46-155), ``StructuredFilter2D/3D`` (geom/_filters.py:72-161),
``MultiGrid`` (solvers/_multigrid.py:11-230), the MG transfer/Galerkin kernels
(core/_mgm.py), ``SingleMaterial`` (MaterialModels.py:31-99) and ``TopOpt``
(TopOpt/_solver.py:17-417).

Run from the repository root with the reference checked out at REFERENCE_ROOT (the
EDGETO_REFERENCE environment variable, else a folder "reference" beside the repository):

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py [--only NAME]

Outputs (all small .npz files, committed):
  kat_stiffness.npz   element stiffness matrices (Q4 / hex8, several nu and box sizes)
  ops_2d.npz, ops_3d.npz   op-level cases: matvec (with/without BCs), diagonal, dk,
                      filter / filter transpose, restriction / prolongation,
                      Galerkin level-1 and level-2 operators, OC update
  loop_mbb2d.npz      120x40 MBB half-beam, 100 SIMP iterations, MG-PCG rtol 1e-8
  loop_cant3d.npz     64x32x32 cantilever, first SIMP iterations, 4-level MG rtol 1e-6
  loop_cant3d_50.npz  the same cantilever, 50 SIMP iterations, 4-level MG rtol 1e-6
  loop_cant3d_50t.npz the same 50 iterations with the solves at rtol 1e-10 (the trajectory of
                      (nearly) exact solves)
  grad_cant3d.npz     32x16x16 cantilever, random rho, compliance and filtered dr
  fea.npz             FEA_integrals, op level and the whole call
  multimaterial.npz   PenalizedMultiMaterial law: forward, plain, backward, constraint, ocP
  general.npz         unstructured meshes (T3, T3+Q4, Tet4, distorted hex8): element
                      matrices, matvec, diagonal, dk, KD-tree filter
"""
import argparse
import os
import sys
import time
import types
from unittest import mock

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: EDGETO_REFERENCE, else a sibling "reference" folder of the repository
REFERENCE_ROOT = os.environ.get("EDGETO_REFERENCE",
                                os.path.normpath(os.path.join(HERE, "..", "..", "..", "reference")))


def _import_reference():
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
    os.environ.setdefault("NUMBA_NUM_THREADS", str(os.cpu_count() or 1))
    for name in ["cupy", "cupyx", "cupyx.scipy", "cupyx.scipy.sparse", "cupyx.scipy.sparse.linalg",
                 "sksparse", "sksparse.cholmod", "matplotlib", "matplotlib.pyplot", "matplotlib.path",
                 "matplotlib.collections", "matplotlib.colors", "matplotlib.cm", "vtk", "k3d", "pygmsh",
                 "vtk.util", "vtk.util.numpy_support"]:
        sys.modules.setdefault(name, mock.MagicMock(name=name))
    sys.path.insert(0, REFERENCE_ROOT)
    import EDGETO  # noqa: F401
    from EDGETO.geom._mesh import StructuredMesh2D, StructuredMesh3D
    from EDGETO.kernels._processors import StructuredStiffnessKernel
    from EDGETO.geom._filters import StructuredFilter2D, StructuredFilter3D
    from EDGETO.solvers._multigrid import MultiGrid
    from EDGETO.MaterialModels import SingleMaterial
    from EDGETO.TopOpt._solver import TopOpt
    from EDGETO.physics._linelas import auto_stiffness
    from EDGETO.core import _mgm
    ns = types.SimpleNamespace(**locals())
    return ns


def _stiff(nu):
    ref = _REF

    def f(x0):
        return ref.auto_stiffness(x0, 1.0, nu)
    return f


def make_kat():
    ref = _REF
    out = {}
    q = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64)
    for nu in (0.3, 0.33):
        K, D, B, A = ref.auto_stiffness(q, 1.0, nu)
        out[f"q4_nu{nu}"] = K
        out[f"q4_nu{nu}_area"] = np.array(A)
    q2 = np.array([[0, 0], [0.5, 0], [0.5, 0.25], [0, 0.25]], dtype=np.float64)
    out["q4_box_0.5x0.25_nu0.3"] = ref.auto_stiffness(q2, 1.0, 0.3)[0]
    h = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                  [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
    for nu in (0.3, 0.33):
        K, D, B, A = ref.auto_stiffness(h, 1.0, nu)
        out[f"hex8_nu{nu}"] = K
        out[f"hex8_nu{nu}_volume"] = np.array(A)
    hb = h * np.array([0.5, 0.25, 1.0])
    out["hex8_box_0.5x0.25x1_nu0.3"] = ref.auto_stiffness(hb, 1.0, 0.3)[0]
    np.savez_compressed(os.path.join(HERE, "kat_stiffness.npz"), **out)


def _random_constraints(rng, n_nodes, dof, frac=0.15):
    cons = np.zeros(n_nodes * dof, dtype=bool)
    full = rng.choice(n_nodes, size=max(1, int(frac * n_nodes)), replace=False)
    for d in range(dof):
        cons[full * dof + d] = True
    single = rng.choice(n_nodes * dof, size=max(1, int(frac * n_nodes)), replace=False)
    cons[single] = True
    return np.where(cons)[0]


def _ops_case(out, tag, mesh, rng, rmins, with_galerkin=True):
    ref = _REF
    dof = mesh.dof
    nel = mesh.elements.shape[0]
    n_nodes = mesh.nodes.shape[0]
    E = rng.uniform(1e-3, 1.0, nel)
    E[rng.choice(nel, size=max(1, nel // 5), replace=False)] = 1e-9
    u = rng.standard_normal(n_nodes * dof)
    out[f"{tag}_E"] = E
    out[f"{tag}_u"] = u
    out[f"{tag}_nel"] = mesh.nel.copy()
    k = ref.StructuredStiffnessKernel(mesh)
    k.set_rho(E)
    out[f"{tag}_matvec_nocon"] = k.dot(u).copy()
    cons = _random_constraints(rng, n_nodes, dof)
    k.add_constraints(cons)
    out[f"{tag}_cons"] = cons
    out[f"{tag}_matvec"] = k.dot(u).copy()
    out[f"{tag}_diag"] = k.diagonal().copy()
    out[f"{tag}_dk"] = k.process_grad(u).copy()
    for r in rmins:
        filt = (ref.StructuredFilter3D(mesh, r) if dof == 3 else ref.StructuredFilter2D(mesh, r))
        rho = rng.uniform(0.0, 1.0, nel)
        out[f"{tag}_filt{r}_in"] = rho
        out[f"{tag}_filt{r}_H"] = filt.dot(rho)
        out[f"{tag}_filt{r}_HT"] = filt._rmatvec(rho)
        out[f"{tag}_filt{r}_ntaps"] = np.array(len(filt.weights))
    v = rng.standard_normal(n_nodes * dof)
    out[f"{tag}_restrict_in"] = v
    out[f"{tag}_restrict"] = ref._mgm.apply_restriction(v, mesh.nel.astype(np.int32), dof)
    nel_c = mesh.nel // 2
    n_coarse = int(np.prod(nel_c + 1))
    vc = rng.standard_normal(n_coarse * dof)
    out[f"{tag}_prolong_in"] = vc
    out[f"{tag}_prolong"] = ref._mgm.apply_prolongation(vc, mesh.nel.astype(np.int32), dof)
    if with_galerkin:
        solver = ref.MultiGrid(mesh, k, n_level=2, tol=1e-8)
        solver._setup()
        A1 = solver.levels[1][0]
        A2 = solver.levels[2][0]
        out[f"{tag}_A1"] = A1.toarray()
        out[f"{tag}_A2"] = A2.toarray()
        out[f"{tag}_D1inv"] = np.asarray(solver.levels[1][1])
        out[f"{tag}_D0inv"] = np.asarray(solver.levels[0][1])
        del solver.levels


def _oc_case(out, tag, mesh, rng):
    ref = _REF
    mat = ref.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.4)
    k = ref.StructuredStiffnessKernel(mesh)
    solver = ref.MultiGrid(mesh, k, n_level=1, tol=1e-8)
    filt = ref.StructuredFilter3D(mesh, 1.5) if mesh.dof == 3 else ref.StructuredFilter2D(mesh, 1.5)
    opt = ref.TopOpt(mesh, mat, k, solver, filt, max_iter=1, move=0.2, verbose=False)
    nel = mesh.elements.shape[0]
    rho = rng.uniform(0.05, 0.95, nel)
    df = -rng.uniform(0.0, 10.0, nel) ** 2
    df[rng.choice(nel, size=nel // 10, replace=False)] = 0.0
    out[f"{tag}_oc_rho"] = rho
    out[f"{tag}_oc_df"] = df
    out[f"{tag}_oc_vf"] = np.array(0.4)
    out[f"{tag}_oc_out"] = opt.update_design(rho.copy(), df.reshape(-1, 1).copy())


def make_ops():
    ref = _REF
    rng = np.random.default_rng(20240601)
    out = {}
    m = ref.StructuredMesh2D(8, 4, 8.0, 4.0, stiffness=_stiff(0.3))
    _ops_case(out, "even", m, rng, (1.5, 2.0, 3.0))
    _oc_case(out, "even", m, rng)
    m = ref.StructuredMesh2D(7, 5, 7.0, 5.0, stiffness=_stiff(0.3))
    _ops_case(out, "odd", m, rng, (1.5, 2.5), with_galerkin=False)
    m = ref.StructuredMesh2D(6, 4, 3.0, 1.0, stiffness=_stiff(0.3))
    _ops_case(out, "aniso", m, rng, (1.5,), with_galerkin=False)
    np.savez_compressed(os.path.join(HERE, "ops_2d.npz"), **out)

    out = {}
    m = ref.StructuredMesh3D(4, 4, 4, 4.0, 4.0, 4.0, stiffness=_stiff(0.3))
    _ops_case(out, "even", m, rng, (1.5, 2.0))
    _oc_case(out, "even", m, rng)
    m = ref.StructuredMesh3D(5, 3, 3, 5.0, 3.0, 3.0, stiffness=_stiff(0.3))
    _ops_case(out, "odd", m, rng, (1.5,), with_galerkin=False)
    m = ref.StructuredMesh3D(4, 2, 2, 2.0, 0.5, 1.0, stiffness=_stiff(0.3))
    _ops_case(out, "aniso", m, rng, (1.5,), with_galerkin=False)
    np.savez_compressed(os.path.join(HERE, "ops_3d.npz"), **out)


class _Recorder:
    """Wraps solver.solve to record the residual and the number of fine matvecs per solve."""

    def __init__(self, solver, kernel):
        self.solver = solver
        self.kernel = kernel
        self.residuals = []
        self.matvecs = []
        self._count = 0
        orig_dot = kernel.dot

        def counting_dot(rhs):
            self._count += 1
            return orig_dot(rhs)
        kernel.dot = counting_dot
        orig_solve = solver.solve

        def recording_solve(*a, **kw):
            self._count = 0
            x, res = orig_solve(*a, **kw)
            self.residuals.append(float(res))
            self.matvecs.append(self._count)
            return x, res
        solver.solve = recording_solve


def _run_loop(mesh, vf, rmin, rho0, n_iter, mg_kwargs, bc_fn, f_fn, keep_rho=None):
    ref = _REF
    mat = ref.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=vf)
    mat.init_desvars = lambda nel, **kw: np.full(nel, rho0, dtype=np.float64)
    k = ref.StructuredStiffnessKernel(mesh)
    filt = ref.StructuredFilter3D(mesh, rmin) if mesh.dof == 3 else ref.StructuredFilter2D(mesh, rmin)
    solver = ref.MultiGrid(mesh, k, **mg_kwargs)
    rec = _Recorder(solver, k)
    opt = ref.TopOpt(mesh, mat, k, solver, filt, max_iter=n_iter, move=0.2, ch_tol=0.0, fun_tol=0.0,
                     verbose=False)
    bc_nodes, bc_vals = bc_fn(mesh)
    opt.add_BC_nodal(bc_nodes, bc_vals)
    f_nodes, f_vals = f_fn(mesh)
    opt.add_F_nodal(f_nodes, f_vals)
    t0 = time.time()
    rho, flag, hist = opt.optimize(save_comp_history=True, save_change_history=True, save_rho_history=True)
    dt = time.time() - t0
    if keep_rho is not None:  # a few designs only: the whole history would be tens of MB
        out = {
            "rho_final": rho,
            "comp_history": np.array(hist["comp_history"]),
            "change_history": np.array(hist["change_history"]),
            "residuals": np.array(rec.residuals),
            "matvecs_per_solve": np.array(rec.matvecs),
            "f_idx": np.nonzero(opt.f)[0],
            "f_val": opt.f[np.nonzero(opt.f)[0]],
            "constraints": np.where(k.constraints)[0],
            "wall_s": np.array(dt),
        }
        for i in keep_rho:
            out[f"rho_{i}"] = hist["rho_history"][i - 1]
        return out
    out = {
        "rho_final": rho,
        "comp_history": np.array(hist["comp_history"]),
        "change_history": np.array(hist["change_history"]),
        "residuals": np.array(rec.residuals),
        "matvecs_per_solve": np.array(rec.matvecs),
        "rho_1": hist["rho_history"][0],
        "f_idx": np.nonzero(opt.f)[0],
        "f_val": opt.f[np.nonzero(opt.f)[0]],
        "constraints": np.where(k.constraints)[0],
        "wall_s": np.array(dt),
    }
    return out


def make_loop_mbb():
    ref = _REF
    mesh = ref.StructuredMesh2D(120, 40, 120.0, 40.0, stiffness=_stiff(0.3))

    def bc(mesh):
        nodes = mesh.nodes
        left = np.where(np.isclose(nodes[:, 0], 0.0))[0]
        br = np.where(np.isclose(nodes[:, 0], 120.0) & np.isclose(nodes[:, 1], 0.0))[0]
        ids = np.concatenate([left, br])
        vals = np.zeros((ids.shape[0], 2), dtype=bool)
        vals[: left.shape[0], 0] = True
        vals[left.shape[0]:, 1] = True
        return ids, vals

    def force(mesh):
        nodes = mesh.nodes
        tl = np.where(np.isclose(nodes[:, 0], 0.0) & np.isclose(nodes[:, 1], 40.0))[0]
        return tl, np.array([[0.0, -1.0]])

    out = _run_loop(mesh, 0.5, 1.5, 0.5, 100, dict(tol=1e-8, n_level=3, maxiter=1000), bc, force)
    np.savez_compressed(os.path.join(HERE, "loop_mbb2d.npz"), **out)
    print("mbb2d: comp", out["comp_history"][0], "->", out["comp_history"][-1], "wall", out["wall_s"])


def _cant_bc_force(L):
    def bc(mesh):
        nodes = mesh.nodes
        ids = np.where(np.isclose(nodes[:, 0], 0.0))[0]
        return ids, np.array([[True, True, True]])

    def force(mesh):
        nodes = mesh.nodes
        ids = np.where(np.isclose(nodes[:, 0], L) & np.isclose(nodes[:, 1], 0.0))[0]
        return ids, np.array([[0.0, -1.0, 0.0]]) / ids.shape[0]
    return bc, force


def make_loop_cant3d():
    ref = _REF
    mesh = ref.StructuredMesh3D(64, 32, 32, 64.0, 32.0, 32.0, stiffness=_stiff(0.3))
    bc, force = _cant_bc_force(64.0)
    out = _run_loop(mesh, 0.12, 1.5, 0.12, 4, dict(tol=1e-6, n_level=4, maxiter=1000), bc, force)
    np.savez_compressed(os.path.join(HERE, "loop_cant3d.npz"), **out)
    print("cant3d: comp", out["comp_history"], "wall", out["wall_s"])


def _loop_cant3d_50(tol, name):
    """64x32x32 cantilever, 50 SIMP iterations (TopOpt/_solver.py:336-417), 4-level MG at the
    given rtol; keeps the compliance history, the final design, the design after 10 and 25
    iterations and the per-solve matvec counts (a few hundred KB)."""
    ref = _REF
    mesh = ref.StructuredMesh3D(64, 32, 32, 64.0, 32.0, 32.0, stiffness=_stiff(0.3))
    bc, force = _cant_bc_force(64.0)
    out = _run_loop(mesh, 0.12, 1.5, 0.12, 50, dict(tol=tol, n_level=4, maxiter=4000), bc, force, keep_rho=(10, 25))
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, "comp", out["comp_history"][[0, 9, 24, 49]], "wall", out["wall_s"])


def make_loop_cant3d_50():
    _loop_cant3d_50(1e-6, "loop_cant3d_50.npz")


def make_loop_cant3d_50t():
    _loop_cant3d_50(1e-10, "loop_cant3d_50t.npz")


def make_grad():
    ref = _REF
    mesh = ref.StructuredMesh3D(32, 16, 16, 32.0, 16.0, 16.0, stiffness=_stiff(0.3))
    bc, force = _cant_bc_force(32.0)
    rng = np.random.default_rng(7)
    rho = rng.uniform(0.2, 1.0, mesh.elements.shape[0])
    mat = ref.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.3)
    k = ref.StructuredStiffnessKernel(mesh)
    filt = ref.StructuredFilter3D(mesh, 2.0)
    solver = ref.MultiGrid(mesh, k, tol=1e-10, n_level=3, maxiter=2000)
    opt = ref.TopOpt(mesh, mat, k, solver, filt, max_iter=1, verbose=False)
    ids, vals = bc(mesh)
    opt.add_BC_nodal(ids, vals)
    ids, vals = force(mesh)
    opt.add_F_nodal(ids, vals)
    comp, dr, res = opt.solve_and_process(rho, 0)
    np.savez_compressed(os.path.join(HERE, "grad_cant3d.npz"), rho=rho, compliance=np.array(comp),
                        dr=dr.reshape(-1), residual=np.array(res), f=opt.f.copy())
    print("grad: comp", comp, "res", res)


def make_fea():
    """FEA_integrals (TopOpt/_solver.py:80-137 and its structured kernel, core/_ops.py:1032-1058):
    op-level with a random displacement on 2-D and 3-D grids, and the whole call (material
    'plain' clip, solve, integrals) on a small MBB beam with a random design."""
    ref = _REF
    from EDGETO.core._ops import FEA_Integrals_node_basis_parallel
    out = {}
    rng = np.random.default_rng(11)
    for tag, mesh in (("2d", ref.StructuredMesh2D(13, 7, 13.0, 7.0, stiffness=_stiff(0.3))),
                      ("3d", ref.StructuredMesh3D(6, 5, 4, 6.0, 5.0, 4.0, stiffness=_stiff(0.3)))):
        k = ref.StructuredStiffnessKernel(mesh)
        nel = mesh.elements.shape[0]
        w = rng.uniform(1e-3, 1.0, nel)
        U = rng.standard_normal(mesh.nodes.shape[0] * mesh.dof)
        strain, stress, energy = FEA_Integrals_node_basis_parallel(
            mesh.K_single, mesh.D_single, mesh.B_single, k.elements_flat, nel, w, U, mesh.dof,
            mesh.elements_size, mesh.B_single.shape[0])
        out.update({f"{tag}_w": w, f"{tag}_U": U, f"{tag}_strain": strain, f"{tag}_stress": stress,
                    f"{tag}_energy": energy, f"{tag}_B": mesh.B_single, f"{tag}_D": mesh.D_single})
    # whole call on a 24x12 MBB beam
    mesh = ref.StructuredMesh2D(24, 12, 24.0, 12.0, stiffness=_stiff(0.3))
    mat = ref.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=0.5)
    k = ref.StructuredStiffnessKernel(mesh)
    filt = ref.StructuredFilter2D(mesh, 1.5)
    solver = ref.MultiGrid(mesh, k, tol=1e-12, n_level=2, maxiter=4000)
    opt = ref.TopOpt(mesh, mat, k, solver, filt, max_iter=1, verbose=False)
    nodes = mesh.nodes
    left = np.where(np.isclose(nodes[:, 0], 0.0))[0]
    opt.add_BC_nodal(left, np.array([[True, False]]))
    br = np.where(np.isclose(nodes[:, 0], 24.0) & np.isclose(nodes[:, 1], 0.0))[0]
    opt.add_BC_nodal(br, np.array([[False, True]]))
    tl = np.where(np.isclose(nodes[:, 0], 0.0) & np.isclose(nodes[:, 1], 12.0))[0]
    opt.add_F_nodal(tl, np.array([[0.0, -1.0]]))
    rho = rng.uniform(0.05, 1.0, mesh.elements.shape[0])
    strain, stress, energy, vm = opt.FEA_integrals(rho)
    out.update(call_rho=rho, call_strain=strain, call_stress=stress, call_energy=energy, call_vm=np.asarray(vm))
    np.savez_compressed(os.path.join(HERE, "fea.npz"), **out)
    print("fea: energy sum", float(np.sum(energy)))


def make_multimaterial():
    """PenalizedMultiMaterial (MaterialModels.py:102-235) run on random designs: forward
    (penalised and plain), backward, the mass constraint and ocP, for two and three
    materials with per-material masses and for two materials with a shared mass over
    rho_mat.  The reference's TopOpt loop cannot run this class (its update_design reshapes
    the design to one column, TopOpt/_solver.py:281), so only the law is pinned here."""
    from EDGETO.MaterialModels import PenalizedMultiMaterial
    out = {}
    rng = np.random.default_rng(21)
    cases = {
        "two": dict(n_material=2, mass=np.array([[0.25], [0.25]]), E_mat=np.array([[1.0], [0.5]]), rho_mat=None,
                    void=1e-6, penalty=3.0),
        "three": dict(n_material=3, mass=np.array([[0.2], [0.15], [0.1]]), E_mat=np.array([[1.0], [0.6], [0.3]]),
                      rho_mat=None, void=1e-6, penalty=3.0),
        "shared": dict(n_material=2, mass=np.array([[0.3]]), E_mat=np.array([[1.0], [0.4]]),
                       rho_mat=np.array([[1.0], [0.35]]), void=1e-9, penalty=2.5),
    }
    nel = 64
    for tag, kw in cases.items():
        m = PenalizedMultiMaterial(**kw)
        n = kw["n_material"]
        rho = rng.uniform(0.0, 1.0, (nel, n))
        rho[0, :] = 0.0  # clip edges
        rho[1, :] = 1.0
        rho[2, 0] = 1.0
        E = m(rho, 0)
        Ep = m(rho, 0, plain=True)
        dE = m.grad(rho, 0)
        dg = rng.uniform(0.5, 1.5, nel)
        vol = float(dg.sum())
        cons = np.stack([m.evaluate_constraint(rho * s, dg, vol) for s in (0.1, 0.5, 1.0)])
        df = -rng.uniform(0.0, 2.0, (nel, n))
        df[3, :] = 0.5  # positive sensitivities: NaN -> 0 in ocP
        ocP = m.ocP(df, dg, rho)
        ocP0 = m.ocP(np.abs(df), dg, rho)  # all positive: the 1e-3 fallback
        out.update({f"{tag}_rho": rho, f"{tag}_E": np.asarray(E).reshape(-1), f"{tag}_Eplain": np.asarray(Ep).reshape(-1),
                    f"{tag}_dE": np.asarray(dE).reshape(nel, n), f"{tag}_dg": dg, f"{tag}_vol": np.array(vol),
                    f"{tag}_cons": cons, f"{tag}_df": df, f"{tag}_ocP": ocP, f"{tag}_ocP0": ocP0,
                    f"{tag}_n": np.array(n), f"{tag}_E_mat": kw["E_mat"].reshape(-1),
                    f"{tag}_mass": kw["mass"].reshape(-1), f"{tag}_void": np.array(kw["void"]),
                    f"{tag}_penalty": np.array(kw["penalty"]),
                    f"{tag}_rho_mat": (kw["rho_mat"].reshape(-1) if kw["rho_mat"] is not None else np.zeros(0))})
    np.savez_compressed(os.path.join(HERE, "multimaterial.npz"), **out)
    print("multimaterial: E sums", {t: float(out[f"{t}_E"].sum()) for t in cases})


def general_meshes(rng):
    """Small unstructured meshes (nodes, elements) shared by the fixture script and the tests:
    'tri' jittered triangles (uniform), 'mixed' triangles and quadrilaterals (general),
    'tet' jittered tetrahedra with both orientations (uniform), 'hex' distorted hexahedra."""
    out = {}
    nx, ny = 6, 4
    xs, ys = np.meshgrid(np.arange(nx + 1, dtype=float), np.arange(ny + 1, dtype=float), indexing="xy")
    P = np.stack([xs.ravel(), ys.ravel()], 1)
    interior = (P[:, 0] > 0) & (P[:, 0] < nx) & (P[:, 1] > 0) & (P[:, 1] < ny)
    P[interior] += rng.uniform(-0.2, 0.2, (int(interior.sum()), 2))
    nid = lambda i, j: j * (nx + 1) + i  # noqa: E731
    tris, mixed = [], []
    for j in range(ny):
        for i in range(nx):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            tris += [[a, b, c], [a, c, d]]
            if (i + j) % 2 == 0:
                mixed.append([a, b, c, d])
            else:
                mixed += [[a, b, c], [a, c, d]]
    out["tri"] = (P.copy(), np.array(tris, dtype=np.int64))
    out["mixed"] = (P.copy(), mixed)
    nx, ny, nz = 3, 2, 2
    g = np.stack(np.meshgrid(np.arange(nx + 1.0), np.arange(ny + 1.0), np.arange(nz + 1.0), indexing="ij"), -1)
    P3 = g.reshape(-1, 3).copy()
    inner = (P3 > 0).all(1) & (P3 < [nx, ny, nz]).all(1)
    P3[inner] += rng.uniform(-0.15, 0.15, (int(inner.sum()), 3))
    nid3 = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k  # noqa: E731
    tets, hexes = [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                c = [nid3(i + a, j + b, k + e) for (a, b, e) in
                     ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))]
                hexes.append(c)
                for t in ((0, 1, 3, 4), (1, 2, 3, 6), (1, 3, 4, 6), (1, 4, 5, 6), (3, 4, 6, 7)):
                    tets.append([c[q] for q in t])
    out["tet"] = (P3.copy(), np.array(tets, dtype=np.int64))
    Ph = P3.copy()
    out["hex"] = (Ph, np.array(hexes, dtype=np.int64))
    return out


def make_general():
    """Unstructured meshes through the reference's CPU classes: GeneralMesh (geom/_mesh.py:
    146-225), UniformStiffnessKernel / GeneralStiffnessKernel (kernels/_processors.py:157-395)
    and GeneralFilter (geom/_filters.py:256-270): element matrices, areas, centroids, matvec
    with and without constraints, diagonal, dk and the filter matrix."""
    from EDGETO.geom._mesh import GeneralMesh
    from EDGETO.kernels._processors import UniformStiffnessKernel, GeneralStiffnessKernel
    from EDGETO.geom._filters import GeneralFilter
    rng = np.random.default_rng(31)
    out = {}
    for tag, (P, els) in general_meshes(rng).items():
        el_arg = np.array(els, dtype=object) if isinstance(els, list) else els
        if isinstance(els, list):
            el_arg = np.empty(len(els), dtype=object)
            for i, e in enumerate(els):
                el_arg[i] = list(e)
        mesh = GeneralMesh(P, el_arg, stiffness=_stiff(0.3))
        k = UniformStiffnessKernel(mesh) if mesh.is_uniform else GeneralStiffnessKernel(mesh)
        n_el = len(els)
        ndof = mesh.nodes.shape[0] * mesh.dof
        rho = rng.uniform(0.1, 1.0, n_el)
        u = rng.standard_normal(ndof)
        k.set_rho(rho)
        mv = np.array(k.dot(u), copy=True)
        U = rng.standard_normal(ndof)
        dk = np.array(k.process_grad(U), copy=True)
        cons = np.unique(rng.choice(ndof, size=max(2, ndof // 8), replace=False))
        k.set_constraints(cons)
        mvc = np.array(k.dot(u), copy=True)
        diag = np.array(k.diagonal(), copy=True)
        filt = GeneralFilter(mesh, 1.6)
        H = filt.kernel.toarray()
        x = rng.uniform(0, 1, n_el)
        sizes = np.array([len(e) for e in els], dtype=np.int64)
        flat = np.concatenate([np.asarray(e, dtype=np.int64) for e in els])
        if mesh.is_uniform:
            Kflat = np.concatenate([K.reshape(-1) for K in mesh.Ks])
        else:
            Kflat = np.asarray(mesh.K_flat)
        out.update({f"{tag}_nodes": P, f"{tag}_sizes": sizes, f"{tag}_flat": flat,
                    f"{tag}_uniform": np.array(bool(mesh.is_uniform)), f"{tag}_dof": np.array(mesh.dof),
                    f"{tag}_centroids": mesh.centeroids, f"{tag}_As": np.asarray(mesh.As).reshape(-1),
                    f"{tag}_volume": np.array(float(mesh.volume)), f"{tag}_Kflat": Kflat, f"{tag}_rho": rho,
                    f"{tag}_u": u, f"{tag}_matvec": mv, f"{tag}_U": U, f"{tag}_dk": dk, f"{tag}_cons": cons,
                    f"{tag}_matvec_con": mvc, f"{tag}_diag_con": diag, f"{tag}_H": H, f"{tag}_fx": x,
                    f"{tag}_Hx": np.asarray(filt._matvec(x)), f"{tag}_HTx": np.asarray(filt._rmatvec(x))})
        print(f"general {tag}: n_el {n_el} ndof {ndof} uniform {mesh.is_uniform}")
    np.savez_compressed(os.path.join(HERE, "general.npz"), **out)


_REF = None

if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    _REF = _import_reference()
    jobs = {"kat": make_kat, "ops": make_ops, "mbb": make_loop_mbb, "cant": make_loop_cant3d,
            "cant50": make_loop_cant3d_50, "cant50t": make_loop_cant3d_50t, "grad": make_grad,
            "fea": make_fea, "mm": make_multimaterial, "general": make_general}
    for name, fn in jobs.items():
        if args.only and name not in args.only.split(","):
            continue
        t0 = time.time()
        fn()
        print(f"[{name}] done in {time.time() - t0:.1f}s", flush=True)
