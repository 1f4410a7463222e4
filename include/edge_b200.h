/* C ABI of the B200 SIMP / GMG-PCG library (libedge_b200.so).
 *
 * Every pointer argument named *_dev is a CUDA device pointer owned by the caller; the
 * library owns only the workspaces it allocates in *_create / edge_mg_config and never
 * allocates on the solve path.  Arrays use the reference's (ahnobari/EDGE-TO) layouts:
 *   DOF vectors      v[node*dof + c], node = j*nx*nz + i*nz + k (3-D) or j*nx + i (2-D)
 *   element arrays   e = i*nely*nelz + j*nelz + k (3-D) or i*nely + j (2-D)
 *   constraint mask  one byte per DOF (nonzero = constrained)
 * (core/_geom.py:4-59).  All calls return EDGE_OK or an error code; edge_last_error()
 * gives the message of the last failing call on the calling thread.  A handle is not
 * thread-safe; calls on one handle are ordered on the handle's stream.
 */
#ifndef EDGE_B200_H
#define EDGE_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDGE_OK 0
#define EDGE_EINVAL 1   /* bad argument or shape: Python ValueError             */
#define EDGE_ECUDA 2    /* CUDA runtime error: Python RuntimeError              */
#define EDGE_ENOTPD 3   /* coarsest Galerkin matrix not positive definite       */
#define EDGE_ESTATE 4   /* call out of order (e.g. rho not set): ValueError     */

#define EDGE_FP64 0     /* every level and vector in FP64 (the plain FP64 path) */
#define EDGE_MIXED 1    /* FP32 operator/V-cycle, BF16 fine Jacobi diagonal,
                           FP64 x, r, dot products, true residuals, coarse solve */

typedef struct edge_problem edge_problem;
typedef struct edge_filter edge_filter;
typedef struct edge_gen edge_gen;
typedef struct edge_batch edge_batch;
typedef struct edge_csr edge_csr;

const char* edge_last_error(void);
int edge_version(void);

/* ---- structured mesh + stiffness operator.
 * Replaces StructuredStiffnessKernel (kernels/_cuda.py:62-302) built on
 * CuStructuredMesh2D/3D (geom/_mesh.py:81-143).  K0 is the element stiffness of
 * element 0 (host, row-major (2^dim*dim)^2, the reference's local node order).
 * precision is the initial solver precision (edge_mg_config can change it). */
int edge_problem_create(int dim, const int* nel, const double* K0, int precision, edge_problem** out);
int edge_problem_destroy(edge_problem* p);
int edge_set_stream(edge_problem* p, void* stream);
/* kernels/_cuda.py:141-150 (set_constraints / add_constraints after the caller merged them) */
int edge_set_constraints(edge_problem* p, const uint8_t* cons_dev);
/* kernels/_cuda.py:36-38 : E is the penalised density per element (user order, FP64) */
int edge_set_rho(edge_problem* p, const double* E_dev);
/* kernels/_cuda.py:173-204, 278-302 : out = K(E) u with BC rows/cols -> identity */
int edge_matvec(edge_problem* p, const double* u_dev, double* out_dev);
/* kernels/_cuda.py:105-139 : diag(K(E)), 1 on constrained DOFs */
int edge_diagonal(edge_problem* p, double* diag_dev);
/* kernels/_cuda.py:152-156 : dk_e = -u_e^T K0 u_e */
int edge_process_grad(edge_problem* p, const double* U_dev, double* dk_dev);
/* Adjoint sensitivity for a linear objective J = l.u with K u = f and K v = l:
 * dk_e = -v_e^T K0 u_e (dJ/dE_e).  No counterpart in the reference (compliance only). */
int edge_process_grad_adjoint(edge_problem* p, const double* U_dev, const double* V_dev, double* dk_dev);
/* Grounded point springs added to K: K_ii += k on the n user DOF indices (host arrays, at
 * most 64; a constrained DOF keeps its identity row).  They enter every product, the PCG
 * operator and the diagonal; the multigrid preconditioner is built from K without them.
 * n = 0 removes them.  No counterpart in the reference (compliant-mechanism springs). */
int edge_set_springs(edge_problem* p, int n, const long long* dofs, const double* k);
/* The same product through the FP32 operator of the mixed-precision solver. */
int edge_matvec_f32(edge_problem* p, const double* u_dev, double* out_dev);
/* Same product through the dense node-centric kernel (an independent path for tests). */
int edge_matvec_dense(edge_problem* p, const double* u_dev, double* out_dev);
/* Tuning/testing switch: 1 (default) stages 3-D fine-level tiles with TMA, 0 uses the
 * cooperative-load version of the same kernel. */
int edge_set_tma(edge_problem* p, int enable);
/* Fine-kernel tile: variant 0..4 = k_fine3_tma (warps, TMA stages) (8,4) (8,3) (8,2) (4,4)
 * (4,3); FP32 only: 5..8 = packed-pair k_fine3_pk, 9..15 = its cube-element block form
 * k_fine3_cube (used when edge_uses_cube_form is 1, else 9..15 run k_fine3_pk); and the
 * target of resident blocks per SM that sets the y-chunking of the grid. */
int edge_set_fine_tile(edge_problem* p, int variant, int blocks_per_sm);
/* Tiles of the three fused launch kinds (first sweep + residual, last sweep + correction,
 * search direction + product): variant (-1: the common tile) and y-chunking target each. */
int edge_fine_kind_tiles(const edge_problem* p, int* variants, int* blocks_per_sm);
int edge_set_kind_tune(edge_problem* p, int enable);
/* Autotuner: times every tile variant and y-chunking on the current density with the plain
 * operator in `precision` (reps launches each; for the mixed path with the cube kernel, the
 * iteration's three fused fine launches together), keeps the fastest, reports it.  Then, unless
 * edge_set_kind_tune(p, 0), it times each fused launch kind alone over the cube-kernel variants
 * and keeps a kind's own tile where it is at least 2 % faster (edge_fine_kind_tiles reports
 * them: variant -1 = the common tile).  edge_set_fine_tile sets one tile for every launch. */
int edge_autotune_fine(edge_problem* p, int precision, int reps, double* best_ms, int* best_variant,
                       int* best_bps);
/* Benchmark helper: average device time (ms) of `reps` fine-operator launches with the given
 * tile, with the smoother-sweep epilogue (sweep != 0; needs edge_mg_config/solve of that
 * precision) or the plain product.  The problem's own tile choice is left unchanged. */
int edge_time_fine(edge_problem* p, int precision, int variant, int blocks_per_sm, int sweep, int reps,
                   double* ms);
/* ---- FEA_integrals.  Replaces TopOpt/_solver.py:80-137 (TopOpt/_cuda.py:78-129) for
 * structured meshes: per element (reference element order) strain = B u_e, stress = D strain,
 * strain energy = 1/2 w_e u_e^T K0 u_e, with u_e from the user-layout displacement U in the
 * reference's corner order.  B is nb x (corners*dim), D nb x nb, row-major (the mesh's
 * B_single, D_single); w per element (the reference passes the 'plain' material values).
 * Outputs: strain, stress [n_el][nb], energy [n_el].  All pointers are device memory. */
int edge_fea_integrals(edge_problem* p, const double* U_dev, const double* w_dev, const double* B_dev,
                       const double* D_dev, int nb, double* strain_dev, double* stress_dev, double* energy_dev);
/* ---- conjugate gradients without a preconditioner.  Replaces the reference's CG solver
 * (solvers/_gpu.py:11-58: cupyx.scipy.sparse.linalg.cg on the matrix-free kernel, M = None,
 * stop at ||r|| <= tol ||f||, residual reported as ||f - K x|| / ||f||).  FP64; needs the
 * density set; no multigrid configuration.  Runs as one CUDA graph launch (while node),
 * captured on the first call.  use_last: start from x_dev (user layout) instead of zero.
 * Does not fail on non-convergence: *iters_out == maxiter and the residual tell. */
int edge_cg_solve(edge_problem* p, const double* f_dev, double* x_dev, int use_last, double tol, int maxiter,
                  double* residual_out, int* iters_out);
/* Per-level smoothing sweeps (pre- and post-smoothing each), sweeps[l] for level l < n;
 * levels from n on use edge_mg_config's n_smooth (n = 0 restores that everywhere).  The
 * reference smooths every level n_smooth times (solvers/_multigrid_cuda.py:133-186); this
 * is the knob the sweep autotuner of the mixed-precision solver turns. */
int edge_mg_set_sweeps(edge_problem* p, const int* sweeps, int n);
/* Smoother weight across solves.  enable = 0 (default): every solve starts at min_omega, as
 * the GPU solver does (CuMultiGrid.solve, solvers/_multigrid_cuda.py:210).  enable = 1: the
 * first solve after this call starts at edge_mg_config's omega and every later solve keeps
 * the weight the previous one ended with, as the CPU solver does (MultiGrid.__init__ and
 * MultiGrid.solve, solvers/_multigrid.py:11-30, 178-225), so the iterates are the CPU
 * solver's. */
int edge_mg_set_omega_carry(edge_problem* p, int enable);
/* Mixed precision, 3-D cube elements: 1 (default) fuses the fine level's work into fewer
 * launches when the level smooths once - the first damped-Jacobi sweep from zero is computed
 * inside the residual launch and again inside the last sweep instead of being stored, and the
 * PCG search direction p = z + beta p is formed inside the product q = A p; 0 runs the same
 * arithmetic as separate launches.  No counterpart in the reference. */
int edge_set_fuse(edge_problem* p, int enable);
/* With the fused launches and a fixed smoother weight (omega == min_omega): 1 folds the PCG's
 * x/r update into the next iteration's launches - the residual update r = r - alpha q into
 * the first fine launch (which writes it into the other buffer of a ping-pong pair with r.r)
 * and the solution update x += alpha p into the search direction's product; 0 (default) keeps
 * the separate update launch (at 12.8M DOF it is faster: the two fused launches grow by more
 * than the update launch costs).  Same arithmetic either way (r.r summed in another order).
 * No counterpart in the reference. */
int edge_set_fuse_xr(edge_problem* p, int enable);
/* Mixed precision, 3-D: the V-cycle from `level` down to the coarsest solve (smoothing
 * sweeps, residuals, transfers, the dense coarsest solve) as one persistent cooperative
 * launch with bounded grid barriers between its stages, instead of one launch per step;
 * 0 (default) = every step its own launch.  The same arithmetic per node.  No counterpart
 * in the reference. */
int edge_set_tail(edge_problem* p, int level);
/* Kernel launches made through this problem so far (a launch inside a graph counts once per
 * execution; edge_profile_begin resets the tally). */
int edge_launch_count(const edge_problem* p, long long* n);
/* enable != 0 (the default): edge_mg_solve and edge_simp_solve_and_process run the
 * multigrid set-up and the whole PCG loop as one CUDA graph launch (a while node repeats
 * the iteration, an if node makes the mixed-precision residual replacement; captured on the
 * first solve and again when a solver setting changes).  0: the same launches from a host
 * loop that reads the solver state once per iteration.  Per-launch profiling
 * (edge_profile_begin, edge_breakdown_begin) always uses the host loop. */
int edge_set_graph(edge_problem* p, int enable);
/* FP32 3-D coarse levels with at least min_slots slots use two nodes per thread (pair loads
 * of the centre and stored blocks; default 200000); min_slots < 0: one node per thread. */
int edge_set_stencil_pair(edge_problem* p, long long min_slots);
/* Mixed precision, 3-D: coarse levels (below the coarsest, above the four-lanes-per-node
 * size) with at least min_slots slots keep a tile-major BF16 pair copy of their stencil,
 * filled by every hierarchy set-up, and are applied from it two nodes per thread with
 * constant-offset coefficient loads and packed FP32 products (k_st3_apply2t); min_slots < 0:
 * off (k_st3_apply2 on the linear BF16 copy).  Default 200000.  Levels already allocated get
 * their copy at this call. */
int edge_set_stencil_tiled(edge_problem* p, long long min_slots);
/* 3-D: enable != 0 (default) forms the Galerkin operators of levels >= 2 (A_{l+1} = R A_l R^T)
 * as three one-axis passes through FP64 intermediates, the restriction being the product of
 * three 1-D full weightings; 0: one direct pass over the fine neighbourhoods.  Same operator,
 * summed in another order. */
int edge_set_galerkin_axis(edge_problem* p, int enable);
/* Mixed precision only: enable != 0 applies the coarse-level stencils (levels >= 1, below the
 * coarsest) from BF16 copies made after each Galerkin set-up (half the bytes of the largest
 * coarse kernel); the Jacobi diagonals and the Galerkin chain stay FP32.  Default 1 (at 12.8M
 * DOF: the same PCG iteration counts as FP32 stencils, 3 % more SIMP iterations/s). */
int edge_set_coarse_bf16(edge_problem* p, int enable);
/* Mixed precision only: enable != 0 (default) stores the PCG residual recurrence in FP32
 * between the FP64 true-residual replacements (each replacement recomputes r = b - A x in FP64
 * after the recurrence has dropped 100-fold, and before convergence is declared; the update
 * itself and r.r are computed in FP64).  0: FP64 recurrence plus an FP32 copy for the V-cycle. */
int edge_set_residual32(edge_problem* p, int enable);
/* enable != 0: the kernels of the captured solve graph are launched with programmatic stream
 * serialization (programmatic dependent launch), so that each kernel's blocks can be
 * scheduled while the previous kernel drains; every kernel waits for its predecessor on
 * entry.  0 (default): plain stream order (at 12.8M DOF the SIMP loop ran 1.5 % faster so).
 * Host-driven solves always use plain order. */
int edge_set_pdl(edge_problem* p, int enable);
/* Coarse 3-D levels with at most max_slots slots use the four-lanes-per-node stencil kernel
 * (latency-bound small levels); larger levels one thread per node.  Default 40000 (at 70k
 * slots one thread per node is already faster). */
int edge_set_stencil_quad(edge_problem* p, long long max_slots);
/* Benchmark helper: average device time (ms) of `reps` Jacobi sweeps of the stencil operator
 * on coarse level 1 <= level < n_level, in the problem's precision (hierarchy built). */
int edge_time_level(edge_problem* p, int level, int reps, double* ms);
/* 1 when the element matrix has the box structure used by the transform kernels */
int edge_uses_transform(const edge_problem* p);
/* 1 when the transformed element matrix has the cube block form (eight coefficients) used by
 * the k_fine3_cube tiles (equal edge lengths, isotropic material) */
int edge_uses_cube_form(const edge_problem* p);

/* ---- geometric multigrid PCG.  Replaces CuMultiGrid (solvers/_multigrid_cuda.py:15-242).
 * cycle_w != 0 reproduces cycle == 'w' (second coarse visit on the levels in w_levels).
 * precision: EDGE_FP64 or EDGE_MIXED (see above). */
int edge_mg_config(edge_problem* p, int n_level, int n_smooth, double omega, double min_omega, int cycle_w,
                   const int* w_levels, int n_w, int precision);
/* Solves K(E) x = f to ||r||/||f|| < tol.  x_dev holds the warm start when use_last != 0
 * and receives the solution.  Never fails on non-convergence: *residual_out reports it. */
int edge_mg_solve(edge_problem* p, const double* f_dev, double* x_dev, int use_last, double tol, int maxiter,
                  double* residual_out, int* iters_out);

/* A real grid of nel_real elements per axis embedded in the lower corner of the problem's
 * grid (a padded grid whose padding elements have no stiffness and whose padding nodes are
 * constrained): E_dev in the real grid's element order sets E (zero on the padding), and
 * the solve takes f_dev / x_dev in the real grid's user layout (the padding's load is zero, its
 * solution is not returned).  The multigrid of a grid whose extents do not divide by
 * 2^n_level runs on such a padded problem (CuMultiGrid's padded path). */
int edge_set_rho_embedded(edge_problem* p, const double* E_dev, const int* nel_real);
int edge_mg_solve_embedded(edge_problem* p, const int* nel_real, const double* f_dev, double* x_dev, int use_last,
                           double tol, int maxiter, double* residual_out, int* iters_out);

/* Builds the hierarchy for the current E / BCs without solving (CuMultiGrid._setup,
 * solvers/_multigrid_cuda.py:64-118), and returns level l (1..n_level) as a dense
 * row-major n x n FP64 matrix in the reference's coarse DOF order (test inspection). */
int edge_mg_setup(edge_problem* p);
int edge_mg_level_dense(edge_problem* p, int level, double* out_dev, long long n);
/* The damped-Jacobi smoother of the V-cycle on its own.  Replaces CuMultiGrid._jacobi_smoother
 * (solvers/_multigrid_cuda.py:59-62): n_step times x <- x + omega Dinv (b - A_level x) on level
 * 0 <= level < n_level of the hierarchy that the last edge_mg_setup or solve built (level 0:
 * K(E) with its BC rows, Dinv = 1 / diag), FP64 (precision EDGE_FP64).  x_dev, b_dev, out_dev
 * in the level's user layout (the reference's node numbering of that level's grid, DOFs
 * interleaved); omega is the weight as used (the V-cycle passes omega * 1.06^level).
 * Synchronises the problem's stream. */
int edge_jacobi_sweep(edge_problem* p, int level, const double* x_dev, const double* b_dev, double omega, int n_step,
                      double* out_dev);

/* ---- multi-material OC update.  Replaces the bisection of TopOpt.update_design
 * (TopOpt/_cuda.py:242-280) for PenalizedMultiMaterial (constraint MaterialModels.py:204-215):
 * rho_dev and ocp_dev (the material's ocP, clipped to >= 1e-12) are n_el x n_sets row-major,
 * A_dev the element areas (n_el values, or one value when A_per_element == 0); every column's
 * multiplier is bisected while any column's gap exceeds 1e-4.  mass: n_sets per-column mass
 * fractions, or with rho_mat (n_sets densities, may be NULL) the one shared mass fraction
 * mass[0] of sum_e sum_m rho[e, m] A_e rho_mat[m].  rho_new_dev receives the design at the last
 * multipliers.  One launch on stream, no host synchronisation; 1 <= n_sets <= 8. */
int edge_oc_update_multi(long long n_el, int n_sets, const double* rho_dev, const double* ocp_dev, const double* A_dev,
                         int A_per_element, double move, double vol, const double* mass, const double* rho_mat,
                         double* rho_new_dev, void* stream);

/* ---- multi-material SIMP law.  Replaces PenalizedMultiMaterial.__forward__ / __backward__
 * (MaterialModels.py:146-205): rho_dev is the n_el x n_mat row-major design (filtered),
 * E_mat the n_mat Young's moduli (host array), 1 <= n_mat <= 8.  E_dev (n_el) receives
 * max(void, sum_m E_m a_m prod_{k!=m} (1 - a_k)), a_m = clip(rho_m, void, 1)^penalty, or with
 * plain != 0 clip(sum_m E_m rho_m, void, 1); dE_dev (n_el x n_mat, may be NULL; ignored when
 * plain) receives dE/drho.  Asynchronous on stream. */
int edge_mm_law(long long n_el, int n_mat, const double* rho_dev, const double* E_mat, double void_, double penalty,
                int plain, double* E_dev, double* dE_dev, void* stream);

/* ---- grid transfers.  Replace apply_restriction_cuda / apply_prolongation_cuda
 * (core/_mgm_cuda.py:223-314); nel is the FINE grid. */
int edge_restrict(int dim, const int* nel, const double* in_dev, double* out_dev, void* stream);
int edge_prolong(int dim, const int* nel, const double* in_dev, double* out_dev, void* stream);

/* ---- density filter.  Replaces CuStructuredFilter2D/3D (geom/_filters.py:164-254):
 * offsets (n_taps x 3 ints, dz = 0 in 2-D) and globally normalised weights. */
int edge_filter_create(int dim, const int* nel, int n_taps, const int* offsets, const double* weights,
                       edge_filter** out);
int edge_filter_destroy(edge_filter* f);
int edge_filter_apply(edge_filter* f, const double* in_dev, double* out_dev, void* stream);
int edge_filter_apply_T(edge_filter* f, const double* in_dev, double* out_dev, void* stream);

/* ---- unstructured meshes (any mix of element kinds, dof 2 or 3).  Replaces the reference's
 * UniformStiffnessKernel / GeneralStiffnessKernel (kernels/_cuda.py:305-815: node-basis
 * product, diagonal, process_grad) on CuGeneralMesh (geom/_mesh.py:146-251).  Host arrays at
 * creation: elem_ptr[n_el+1] offsets into elem_flat (node ids), K the element matrices
 * row-major back to back with K_ptr[n_el+1] offsets (element e: (size*dof)^2 entries).  The
 * product: out = K(rho) u with constrained rows/columns -> identity; the diagonal has 1 on
 * constrained DOFs; dk_e = -u_e^T K_e u_e.  Device vectors use the reference's interleaved
 * DOF layout; cons is one byte per DOF. */
int edge_gen_create(int dof, long long n_nodes, long long n_el, const int* elem_ptr, const int* elem_flat,
                    const double* K, const long long* K_ptr, edge_gen** out);
int edge_gen_destroy(edge_gen* m);
int edge_gen_set_stream(edge_gen* m, void* stream);
int edge_gen_set_rho(edge_gen* m, const double* rho_dev);
int edge_gen_set_constraints(edge_gen* m, const uint8_t* cons_dev);
int edge_gen_matvec(edge_gen* m, const double* u_dev, double* out_dev);
int edge_gen_diagonal(edge_gen* m, double* diag_dev);
int edge_gen_process_grad(edge_gen* m, const double* U_dev, double* dk_dev);
/* The reference's CG on a general mesh (solvers/_gpu.py:11-58: cupyx cg, M = None, stop at
 * ||r|| <= tol ||f||, residual reported as ||f - K x|| / ||f||), FP64, matrix-free; use_last:
 * start from x_dev.  Does not fail on non-convergence. */
int edge_gen_cg_solve(edge_gen* m, const double* f_dev, double* x_dev, int use_last, double tol, int maxiter,
                      double* residual_out, int* iters_out);
/* Density filter of a general mesh as a CSR matrix H (host arrays: the KD-tree cone weights
 * of CuGeneralFilter, geom/_filters.py:278-298): out = H in, or H^T in with transpose != 0. */
int edge_csr_create(long long n, const long long* indptr, const int* indices, const double* data, edge_csr** out);
int edge_csr_destroy(edge_csr* f);
int edge_csr_apply(edge_csr* f, const double* in_dev, double* out_dev, int transpose, void* stream);

/* ---- OC update.  Replaces TopOpt.update_design (TopOpt/_cuda.py:242-280) with
 * SingleMaterial.ocP / evaluate_constraint (MaterialModels.py:75-90).  Also returns
 * sum((rho_new - rho)^2) for the RMS design change. */
int edge_oc_update(edge_problem* p, const double* rho_dev, const double* dr_dev, double A, double vol, double vf,
                   double move, double* rho_new_dev, double* lambda_out, int* steps_out, double* sqchange_out);

/* The same OC update for callers that must not allocate device memory, and need no
 * problem handle: for example an optimiser whose sensitivities come from another solver,
 * running where every byte of device memory belongs to another allocator's pool, or where
 * creating an edge_problem (which allocates the multigrid workspaces) is not wanted.
 * No counterpart in the reference.  n elements of uniform measure A, on `stream`.
 * It allocates nothing: its workspace is a fixed 8.1 MiB device array inside the library,
 * so n is limited to 1,048,576 elements (larger n: EDGE_EINVAL; use edge_oc_update).  Every
 * call looks up that array's address on the current device (a runtime query, no
 * allocation); `stream` must belong to the current device (otherwise EDGE_EINVAL).  The call
 * waits for `stream` before it returns.  It zeroes the workspace's reduction counter itself; nothing has to
 * be initialised by the caller.  There is one workspace per device: calls whose work
 * overlaps on the same device (different streams or host threads) race and give wrong
 * results, so order them on one stream or synchronise between them.  Results equal
 * edge_oc_update's for the same inputs. */
int edge_oc_update_static(long long n, const double* rho_dev, const double* dr_dev, double A, double vol, double vf,
                          double move, double* rho_new_dev, double* lambda_out, int* steps_out,
                          double* sqchange_out, void* stream);

/* ---- one SIMP analysis, fused.  Replaces TopOpt.solve_and_process (TopOpt/_cuda.py:282-302)
 * for SingleMaterial: rho_f = H rho, E = clip(rho_f^p, void, 1), solve, c = f.U,
 * dr = H^T (p clip(rho_f, void, 1)^(p-1) dk). */
int edge_simp_solve_and_process(edge_problem* p, edge_filter* f, const double* rho_dev, double penalty,
                                double void_, const double* f_dev, double* U_dev, int use_last, double tol,
                                int maxiter, double* compliance_out, double* dr_dev, double* rho_f_dev,
                                double* residual_out, int* iters_out);

/* ---- one whole SIMP iteration as one CUDA graph launch.  Replaces TopOpt.update_design
 * followed by TopOpt.solve_and_process (TopOpt/_cuda.py:242-302) for SingleMaterial: the OC
 * update of rho_dev with the sensitivities dr_dev (the bisection loop runs on the device as a
 * conditional node: no host read inside it) into rho_new_dev, then the analysis of rho_new_dev
 * exactly as edge_simp_solve_and_process (new sensitivities into dr_new_dev, U_dev updated,
 * the filtered density into rho_f_dev when given).  The host reads the results once.  The
 * graph is captured on the first call and again when a setting baked into it changes; the
 * first call allocates the four element-sized buffers the graph works on.  Not available
 * while profiling (edge_profile_begin / edge_breakdown_begin): EDGE_ESTATE. */
int edge_simp_iteration(edge_problem* p, edge_filter* f, const double* rho_dev, const double* dr_dev, double A,
                        double vol, double vf, double move, double penalty, double void_, const double* f_dev,
                        double* U_dev, int use_last, double tol, int maxiter, double* rho_new_dev, double* dr_new_dev,
                        double* rho_f_dev, double* compliance_out, double* residual_out, int* iters_out,
                        double* lambda_out, int* oc_steps_out, double* sqchange_out);

/* ---- many independent 2-D problems: every analysis's solve in one persistent launch.
 * No reference counterpart (the reference solves problems one at a time; its randomizer,
 * randomizer/ConfigSolve.py:6-26, is the intent): the batched form of
 * edge_simp_solve_and_process.  problems[i] is the problem the multigrid runs on, with its
 * multigrid configured (edge_mg_config, 1 <= n_level < 8, V-cycle, no springs) and its BCs
 * set; its grid may be larger than the real nelx[i] x nely[i] grid (a padded grid: the
 * real grid in its lower corner, padding elements without stiffness that the SIMP law never
 * writes, padding nodes constrained).  filters[i] is the density filter of the real grid.
 * Every problem has the same precision.  The handle keeps pointers to the problems and
 * filters: destroy it before them.  */
int edge_batch_create(int n, edge_problem* const* problems, edge_filter* const* filters, const int* nelx,
                      const int* nely, edge_batch** out);
int edge_batch_destroy(edge_batch* b);
/* Shape of the solve launch: `threads` per block and `team` blocks per problem (team > 1: a
 * thread block cluster of that many blocks solves each problem together).  Supported: team 1
 * with 256, 512 (default) or 1024 threads; team 2, 4 or 8 with 512 or 1024 threads. */
int edge_batch_set_threads(edge_batch* b, int threads, int team);
/* With team > 1: problems with fewer than split_dof DOFs (default 0 = none) are solved
 * by single blocks of small_threads threads (256, 512 or 1024, the default) in a second
 * launch beside the teams' launch, each launch on a share of the SMs proportional to its
 * problems' expected work. */
int edge_batch_set_split(edge_batch* b, long long split_dof, int small_threads);
/* Device time (ms) of the three phases of the last edge_batch_solve_and_process: the
 * per-problem preparation (filter, law, loads, hierarchy set-up), the solve launch, and the
 * per-problem post-processing. */
int edge_batch_last_times(const edge_batch* b, double* setup_ms, double* solve_ms, double* post_ms);
/* Start and end (ms after the first start) of each problem's solve in the last solve launch,
 * from the device's global timer: the launch's load balance.  Synchronises the device. */
int edge_batch_last_problem_times(edge_batch* b, double* start_ms, double* end_ms);
/* The OC update of every problem (edge_oc_update, TopOpt/_cuda.py:242-280) in one launch on
 * `stream`: one block per problem, the bisection's sums as block sums; rho[i], dr[i],
 * rho_new[i] on the real grid (nelx[i] * nely[i]), A[i] the element area, vol[i] the domain
 * volume, vf[i] the volume fraction.  The last lambda and the bisection steps per problem
 * into lambda_out / steps_out when given (then it synchronises `stream`; otherwise it only
 * enqueues). */
int edge_batch_oc_update(edge_batch* b, const double* const* rho, const double* const* dr, const double* A,
                         const double* vol, const double* vf, double move, double* const* rho_new, double* lambda_out,
                         int* steps_out, void* stream);
/* One SIMP analysis of every problem, on `stream`, arrays in each problem's real-grid user
 * layout (rho[i], dr[i]: nelx[i] * nely[i]; f[i], U[i]: 2 (nelx[i] + 1)(nely[i] + 1)):
 * per problem the filter and SIMP law of edge_simp_solve_and_process into the problem's
 * grid, the load and warm start (use_last) and the multigrid hierarchy for the new E; then
 * ONE launch that solves all n systems to ||r|| / ||f|| < tol (a block takes the next
 * unsolved problem, largest first, and runs its whole PCG: FP64 Krylov vectors, products of
 * the search direction and inner products, preconditioned by the problem's V-cycle in its
 * precision); then per problem c = f . U, dr = H^T (p clip(rho_f, void, 1)^(p-1) dk) and U.
 * Results per problem in compliance, residual, iters (any may be null).  Never fails on
 * non-convergence; a coarsest Galerkin matrix that is not positive definite is EDGE_ENOTPD
 * after the call (the other problems' results are valid).  Synchronises `stream` once. */
int edge_batch_solve_and_process(edge_batch* b, const double* const* rho, double penalty, double void_,
                                 const double* const* f, double* const* U, int use_last, double tol, int maxiter,
                                 double* compliance, double* const* dr, double* residual, int* iters, void* stream);

/* Benchmark instrumentation: between begin and end, every fine-level operator launch
 * (the dominant kernel) is bracketed by CUDA events on the problem's stream and its
 * algorithmic bytes recorded (input vector + E + epilogue traffic); end() returns their
 * summed device time, bytes and count, and the number of library kernels launched. */
int edge_profile_begin(edge_problem* p, int max_launches);
int edge_profile_end(edge_problem* p, double* kernel_ms, double* kernel_bytes, int* kernel_launches,
                     long long* total_launches);
/* Per-category device time of every library launch between begin and end (categories:
 * 0 other, 1 fine operator, 2 coarse stencils, 3 transfers, 4 vector/PCG, 5 hierarchy
 * setup, 6 coarsest solve, 7 OC update, 8 filter/sensitivities). */
int edge_breakdown_begin(edge_problem* p, int max_launches);
int edge_breakdown_end(edge_problem* p, double* ms_by_cat, int* n_by_cat, int n_cat);
/* Kernel timing of the last edge_mg_solve (ms), for the benchmarks. */
int edge_last_solve_stats(const edge_problem* p, double* setup_ms, double* solve_ms, int* pcg_iters,
                          int* true_residuals);

#ifdef __cplusplus
}
#endif
#endif
