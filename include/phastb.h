/*
 * phastb.h -- C ABI of the B200 backend for PhAST's matrix-free phase-field
 * hot path (structured Q4 grids in 2D, periodic voxel H8 cells in 3D).
 *
 * Conventions
 *   - Every entry point returns an int status (PHASTB_OK on success) and never
 *     throws or traps.  Device errors surface as PHASTB_ERR_CUDA.
 *   - Pointers named d_* / arrays are DEVICE pointers unless stated otherwise;
 *     they are caller-owned.  `stream` is a cudaStream_t (NULL = legacy stream).
 *   - Field layouts follow PhAST: 2D u/v/a (N,2) node-major, d (N,), Gauss
 *     fields (E,4); 3D x = [u~ (3 n_red), E (6)], d (n_red,), Gauss fields (E,8).
 *     Node and element numbering are those of structured_q4_mesh and of
 *     PeriodicVoxelMap (x fastest).
 *   - `dtype` selects the storage/arithmetic type of the vectors: PHASTB_F64 or
 *     PHASTB_F32.  Inner products, norms and reductions are always FP64.
 *   - Scratch memory comes from a caller-provided workspace whose size is given
 *     by the matching *_workspace_bytes function.
 *
 * Each declaration cites the PhAST function (src/phast/..., file:line) whose
 * behaviour it reproduces.
 */
#ifndef PHASTB_H
#define PHASTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define PHASTB_OK 0
#define PHASTB_ERR_ARG 1         /* bad shape/option (ValueError in PhAST)      */
#define PHASTB_ERR_CUDA 2        /* CUDA runtime error                           */
#define PHASTB_NONCONVERGED 3    /* iteration cap reached                        */
#define PHASTB_DIVERGED 4        /* residual grew past the divergence guard      */
#define PHASTB_BREAKDOWN 5       /* non-positive curvature / non-SPD             */
#define PHASTB_NONFINITE 6       /* NaN/Inf met                                  */
#define PHASTB_ERR_WORKSPACE 7   /* workspace too small                          */
#define PHASTB_UNSUPPORTED 8     /* option not implemented (NotImplementedError) */
#define PHASTB_ERR_CAPACITY 9    /* problem larger than a fixed-capacity entry point allows */

#define PHASTB_F64 0
#define PHASTB_F32 1

/* energy splits of the 2D operators (fem_operators.py:283-560, 951-1161) */
#define PHASTB_SPLIT_LINEAR 0          /* undegraded C eps (internal_force_linear) */
#define PHASTB_SPLIT_ISOTROPIC 1
#define PHASTB_SPLIT_AMOR 2
#define PHASTB_SPLIT_SPECTRAL 3        /* strain-spectral, algebraic projector     */
#define PHASTB_SPLIT_STAR_CONVEX 4
#define PHASTB_SPLIT_SPECTRAL_STRESS 5

/* --------------------------------------------------------------- 2D (Q4) */
typedef struct {
  int nx, ny;        /* elements along x and y (structured_q4_mesh, quad_elements.py:458) */
  double hx, hy;     /* element edge lengths */
} phastb_q4_grid;

typedef struct {
  double E, nu;
  double lam;          /* Material.lam (plane-stress reduced when plane_stress) */
  double mu;           /* Material.mu */
  double kappa;        /* Material.kappa, the 3D bulk modulus */
  double eta;          /* eta_residual of g(d) = (1-d)^2 (1-eta) + eta */
  double spectral_eps; /* FEMOperators._spectral_eps */
  int plane_stress;
  int stress_split;    /* PHASTB_SPLIT_* of effective_stress_split() */
  int psi_split;       /* PHASTB_SPLIT_* of energy_split (history driver) */
} phastb_q4_material;

/* Strain at the 2x2 Gauss points, three (E,4) arrays.
 * FEMOperators._compute_strain_q4, core/fem_operators.py:244-254 */
int phastb_q4_strain(const phastb_q4_grid* g, int dtype, const void* u, void* exx, void* eyy,
                     void* gxy, void* stream);

/* Degraded internal force f (N,2); d == NULL gives the undegraded linear force.
 * FEMOperators.internal_force / internal_force_linear, fem_operators.py:598-612,655-659 */
int phastb_q4_internal_force(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype,
                             const void* u, const void* d, void* f, void* stream);

/* Transposed Gauss-point energy gradient f (N,2) = sum_q wq[e][q] B_q^T sigma0(u)_q of the
 * undegraded energy psi0 (isotropic split only, FP64): the adjoint of the history update
 * H = max(H_prev, psi+(u)) where psi+ won.  compute_psi_plus (isotropic),
 * core/fem_operators.py:951-990 */
int phastb_q4_psi_grad_t(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u,
                         const double* wq, double* f, void* stream);

/* out (N,) = d/dd [z . f_int(u, d)] = sum_q w g'(d_q) N_q eps(z)_q . sigma0(u)_q (isotropic split,
 * FP64): the damage derivative of the degraded internal force, contracted with z.
 * internal_force, core/fem_operators.py:598-699; degradation, physics/material.py:497-529 */
int phastb_q4_force_dd_t(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u,
                         const double* z, const double* d, double* out, void* stream);

/* Jacobi diagonal (N,2) of K(d); d == NULL means g = 1.
 * FEMOperators.stiffness_diagonal, fem_operators.py:1284-1320 */
int phastb_q4_stiffness_diagonal(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype,
                                 const void* d, void* diag, void* stream);

/* psi+ at Gauss points and the history max H_out = max(H_in, psi+), (E,4) each.
 * Any of H_in/H_out/psi may be NULL (H_in NULL means H_in = 0).
 * compute_psi_plus fem_operators.py:951-1161 + StaggeredSolver._H_update
 * staggered_solver.py:804-845 (hard_max, h_update.py:47-49) */
int phastb_q4_psi_history(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype,
                          const void* u, const void* H_in, void* H_out, void* psi, void* stream);

/* AT2 damage operator y = Gc l0 K d + M(rho) d with Gauss reaction density
 * rho_q = rd_scale * Hq + (rd_shift_e ? rd_shift_e[e] : rd_shift) and Laplacian weight
 * (gcl0_e ? gcl0_e[e] : gcl0).  Always FP64.
 * PhaseFieldDamageSolver._Ax_q4, solvers/damage_solver.py:1797-1838 */
int phastb_q4_damage_apply(const phastb_q4_grid* g, const double* d, const double* Hq,
                           double rd_scale, double rd_shift, const double* rd_shift_e, double gcl0,
                           const double* gcl0_e, double* y, void* stream);

/* Right-hand side b = sum_q N 2 H_q w and Jacobi inverse M_inv = 1/(diag + 1e-30).
 * _prepare_cg_q4, damage_solver.py:2270-2301 */
int phastb_q4_damage_prepare(const phastb_q4_grid* g, const double* Hq, double gc_over_l0,
                             const double* gc_over_l0_e, double gcl0, const double* gcl0_e,
                             double* b, double* m_inv, void* stream);

/* Bound-projected PCG damage solve, d in [d_prev, 1] with optional pinned nodes.
 * d_init NULL starts from d_prev.  fixed (N,) uint8 and fixed_vals may be NULL.
 * info[0] = last_iter, info[1] = reason (0 converged, 1 max_iter, 2 non-SPD, 3 diverged).
 * PhaseFieldDamageSolver._solve_projected_cg, damage_solver.py:3528-3775 */
size_t phastb_q4_damage_solve_workspace_bytes(int n_nodes);
int phastb_q4_damage_solve(const phastb_q4_grid* g, const double* Hq, double gc_over_l0,
                           const double* gc_over_l0_e, double gcl0, const double* gcl0_e,
                           const double* d_prev, const double* d_init, const uint8_t* fixed,
                           const double* fixed_vals, double tol, int max_iter, int check_every,
                           double* d_out, int* info, void* workspace, size_t workspace_bytes,
                           void* stream);

/* Linear AT2 damage system A x = rhs (the operator of phastb_q4_damage_solve, no bounds) with
 * the rows in `fixed` eliminated and held at fixed_vals (0 when fixed_vals is NULL); Jacobi PCG
 * from x0 (NULL: zero) to ||r|| <= rtol ||rhs_free||.  This is the adjoint solve of the damage
 * step: A is symmetric, so A^T lam = g is the same system.  info[0] iterations, info[1] 0 converged,
 * 1 max_iter, 2 breakdown, 3 non-finite; rinfo[0] ||rhs_free||, rinfo[1] final ||r||.
 * _pcg_solve_adjoint_system, solvers/damage_solver.py:423-480 */
size_t phastb_q4_damage_linear_workspace_bytes(int n_nodes);
int phastb_q4_damage_linear_solve(const phastb_q4_grid* g, const double* Hq, double gc_over_l0,
                                  const double* gc_over_l0_e, double gcl0, const double* gcl0_e,
                                  const double* rhs, const uint8_t* fixed, const double* fixed_vals,
                                  const double* x0, double rtol, int max_iter, int check_every,
                                  double* x_out, int* info, double* rinfo, void* workspace,
                                  size_t workspace_bytes, void* stream);

/* Adjoint sensitivities of the AT2 damage system for an adjoint field lam (N,) and damage d (N,),
 * per element: lam_K_d_e = lam^T K_e d, lam_M_d_e = lam^T M_e d (Gauss-point sums),
 * grad_gc_e = -(l0 lam_K_d_e + lam_M_d_e / l0), grad_H (E,4) = 2 w lam_q (1 - d_q).  Any output may
 * be NULL.  _adjoint_quadratic_forms_perelem and _AdjointDamageSolveField.backward,
 * solvers/damage_solver.py:284-331, 998-1016, written for the Q4 Gauss rule */
int phastb_q4_damage_adjoint_grads(const phastb_q4_grid* g, const double* lam, const double* d, double l0,
                                   double* grad_gc_e, double* grad_H, double* lam_K_d_e,
                                   double* lam_M_d_e, void* stream);

/* One central-difference step, fused: predictor, f_int(u_new, d), corrector,
 * Dirichlet zeroing; optionally the history update H_out = max(H_in, psi+(u_new)).
 * m_inv (N,) = 1/(rho M + 1e-30) per node; bc_mask (N,2) uint8.
 * ExplicitDynamics.step, mechanics_solver.py:153-239 (+ step_compute_driving_force) */
int phastb_q4_explicit_step(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype,
                            double dt, const void* m_inv, const void* u, const void* v,
                            const void* a, const void* d, const void* f_ext, const uint8_t* bc_mask,
                            const void* bc_vals, void* u_out, void* v_out, void* a_out,
                            const void* H_in, void* H_out, void* stream);

/* Reverse of one phastb_q4_explicit_step (FP64, stress splits linear in u at fixed d:
 * isotropic or linear; others return PHASTB_UNSUPPORTED).  Given the adjoints ub, vb, ab of the
 * step's outputs (u', v', a'), writes the adjoints of its inputs (u, v, a) to ub_out, vb_out,
 * ab_out, adds the f_ext adjoint to fb_acc and, when db_acc is given, the adjoint of d to db_acc
 * (u_new = the step's u').  The history update of the forward step is not differentiated.
 * scratch: 4 N doubles.  No reference counterpart for Q4; the reference differentiates its explicit
 * loop through torch autograd with chunked recomputation (ChunkedExplicitDynamicsAutograd,
 * solvers/mechanics_solver.py:4057-4137). */
int phastb_q4_explicit_adjoint_step(const phastb_q4_grid* g, const phastb_q4_material* m, double dt,
                                    const double* m_inv, const double* d, const uint8_t* bc_mask,
                                    const double* u_new, const double* ub, const double* vb,
                                    const double* ab, double* ub_out, double* vb_out, double* ab_out,
                                    double* fb_acc, double* db_acc, double* scratch, void* stream);

/* ---- unstructured linear triangles (T3), FP64 ----------------------------------------------
 * Greedily coloured elements: no two elements of one colour share a node, so each colour's
 * elements scatter their nodal contributions without atomics (one launch per colour; the
 * per-node summation order is fixed, hence deterministic results).  elem, order, grad, areas
 * are device arrays; color_off is a HOST array of n_colors + 1 offsets into order, which the
 * caller keeps unchanged for the lifetime of the mesh.  Geometry as FEMMesh (T3 branch,
 * core/mesh.py:236-303): grad (E,3,2) P1 gradients, areas (E,). */
typedef struct {
  int n_nodes, n_elems, n_colors, reserved; /* reserved: 0 */
  const int* elem;       /* (E,3) node ids */
  const int* order;      /* (E,) element ids sorted by colour */
  const int* color_off;  /* host, (n_colors+1) */
  const double* grad;    /* (E,3,2) */
  const double* areas;   /* (E,) */
} phastb_t3_mesh;

/* A T3 damage model beyond element-history AT2 (PhaseFieldDamageSolver, damage_solver.py:1316-1340):
 * AT1 (element history): gcl0 = 3 Gc l0 / 4, gc_over_l0 = 0, source = 3 Gc / (8 l0) subtracted from
 * the reaction 2 H on the right-hand side; AT2 with nodal history (nodal_h = 1, H of length
 * n_nodes, triple-product reaction mass, damage_solver.py:1840-1912, 2303-2348; the reference
 * supports nodal history with AT2 only, so source must be 0).  The *_e arrays (may be NULL)
 * override the scalars per element. */
typedef struct {
  int nodal_h, reserved;   /* reserved: 0 */
  double gcl0, gc_over_l0, source;
  const double* gcl0_e;
  const double* gc_over_l0_e;
  const double* source_e;
} phastb_t3_damage_model;

/* y = A d of the model's damage system.  _Ax / _Ax_nodal, damage_solver.py:1702-1912 */
int phastb_t3_damage_apply_ex(const phastb_t3_mesh* mesh, const phastb_t3_damage_model* model, const double* d,
                              const double* H, double* y, void* stream);
/* b and M_inv = 1/(diag + 1e-30) of the model.  _prepare_cg / _prepare_cg_nodal,
 * damage_solver.py:2040-2348 */
int phastb_t3_damage_prepare_ex(const phastb_t3_mesh* mesh, const phastb_t3_damage_model* model, const double* H,
                                double* b, double* m_inv, void* stream);
/* Bound-projected PCG solve of the model's system (as phastb_t3_damage_solve; workspace
 * phastb_t3_damage_solve_workspace_bytes).  _solve_projected_cg, damage_solver.py:3528-3775 */
int phastb_t3_damage_solve_ex(const phastb_t3_mesh* mesh, const phastb_t3_damage_model* model, const double* H,
                              const double* d_prev, const double* d_init, const uint8_t* fixed,
                              const double* fixed_vals, double tol, int max_iter, int check_every, double* d_out,
                              int* info, void* workspace, size_t workspace_bytes, void* stream);

/* Host check of a T3 colouring before it is used (all HOST arrays): node ids in range,
 * `order` a permutation of the elements, colour offsets from 0 to n_elems, and no node shared
 * by two elements of one colour.  PHASTB_ERR_ARG otherwise.  The element kernels trust the
 * colouring (a conflict would race); the reference assembles with scatter-adds and has no
 * colouring, so this check has no counterpart there. */
int phastb_t3_check_mesh(int n_nodes, int n_elems, const int* elem, const int* order, int n_colors,
                         const int* color_off);

/* Internal force at the element centroid stress of the split (d NULL: undegraded linear).
 * FEMOperators.internal_force / _assemble_force, core/fem_operators.py:598-680 */
int phastb_t3_internal_force(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                             const double* d, double* f, void* stream);
/* psi+ per element and H_out = max(H_in, psi+) (either output may be NULL).
 * compute_psi_plus, fem_operators.py:951-1025 (T3 branch) + _H_update */
int phastb_t3_psi_history(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                          const double* H_in, double* H_out, double* psi, void* stream);
/* AT2 damage operator y = Gc l0 K d + consistent mass with rc_e = (2 H_e + Gc/l0) A_e / 12;
 * per-element overrides gc_over_l0_e, gcl0_e may be NULL.  PhaseFieldDamageSolver._Ax,
 * solvers/damage_solver.py:1702-1755 */
int phastb_t3_damage_apply(const phastb_t3_mesh* mesh, const double* d, const double* H, double gc_over_l0,
                           const double* gc_over_l0_e, double gcl0, const double* gcl0_e, double* y,
                           void* stream);
/* b = sum 2 H_e A_e / 3 and Jacobi M_inv = 1 / (diag + 1e-30), diag = Gc l0 A |grad phi|^2 + 2 rc_e.
 * _prepare_cg + _compute_preconditioner, damage_solver.py:2095-2265 */
int phastb_t3_damage_prepare(const phastb_t3_mesh* mesh, const double* H, double gc_over_l0,
                             const double* gc_over_l0_e, double gcl0, const double* gcl0_e, double* b,
                             double* m_inv, void* stream);
/* Bound-projected PCG damage solve on T3 (as phastb_q4_damage_solve).
 * _solve_projected_cg, damage_solver.py:3528-3775 */
size_t phastb_t3_damage_solve_workspace_bytes(int n_nodes);
int phastb_t3_damage_solve(const phastb_t3_mesh* mesh, const double* H, double gc_over_l0,
                           const double* gc_over_l0_e, double gcl0, const double* gcl0_e,
                           const double* d_prev, const double* d_init, const uint8_t* fixed,
                           const double* fixed_vals, double tol, int max_iter, int check_every,
                           double* d_out, int* info, void* workspace, size_t workspace_bytes, void* stream);

/* T3 adjoint pieces (isotropic split, FP64), the element analogues of the Q4 entries:
 * f (N,2) = sum_e w[e] B_e^T sigma0(u)_e, the transpose of u -> psi+_e where w is the history
 * gradient on the elements where psi+ won (compute_psi_plus, fem_operators.py:951-990);
 * out (N,) = d/dd [z . f_int(u, d)] = sum_e A_e g'(d_e) / 3 eps(z)_e . sigma0(u)_e with d_e the
 * element mean (internal_force, fem_operators.py:598-680). */
int phastb_t3_psi_grad_t(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                         const double* w, double* f, void* stream);
int phastb_t3_force_dd_t(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                         const double* z, const double* d, double* out, void* stream);
/* Per-element adjoint quadratic forms of the T3 AT2 system for an adjoint lam and damage d:
 * lam_K_d_e = A (grad lam . grad d), lam_M_d_e = A/12 (sum lam sum d + lam . d),
 * grad_gc_e = -(l0 lam_K_d_e + lam_M_d_e / l0), grad_H_e = 2 A sum_a lam_a (1/3 - (d_a + sum d)/12);
 * any output may be NULL.  _adjoint_quadratic_forms_perelem and the history pullback of
 * _AdjointDamageSolveField, solvers/damage_solver.py:284-336, 1017-1027 */
int phastb_t3_damage_adjoint_grads(const phastb_t3_mesh* mesh, const double* lam, const double* d, double l0,
                                   double* grad_gc_e, double* grad_H, double* lam_K_d_e, double* lam_M_d_e,
                                   void* stream);
/* Dirichlet-eliminated linear AT2 solve A x = rhs on T3 (as phastb_q4_damage_linear_solve):
 * the adjoint system of the damage step.  _pcg_solve_adjoint_system, damage_solver.py:423-480 */
size_t phastb_t3_damage_linear_workspace_bytes(int n_nodes);
int phastb_t3_damage_linear_solve(const phastb_t3_mesh* mesh, const double* H, double gc_over_l0,
                                  const double* gc_over_l0_e, double gcl0, const double* gcl0_e, const double* rhs,
                                  const uint8_t* fixed, const double* fixed_vals, const double* x0, double rtol,
                                  int max_iter, int check_every, double* x_out, int* info, double* rinfo,
                                  void* workspace, size_t workspace_bytes, void* stream);
/* Quasi-static Newton with matrix-free CG on a T3 mesh (as phastb_q4_qs_solve; isotropic split;
 * the stiffness action is the coloured internal-force scatter).  QuasiStaticSolver.solve,
 * mechanics_solver.py:1597-1831 */
size_t phastb_t3_qs_workspace_bytes(int n_nodes);
int phastb_t3_qs_solve(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* d,
                       const double* f_ext, const uint8_t* bc_mask, const double* bc_vals, double* u, double tol,
                       double cg_tol, int cg_max_iter, int max_iter, int line_search, int ls_max_steps,
                       double ls_min_alpha, double ls_c, int* info, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Energy sums (FP64): out[0] elastic, out[1] fracture surface term d^T M d,
 * out[2] gradient term d^T K d, out[3] kinetic sum_i |v_i|^2 M_i (v may be NULL).
 * compute_energy_components, fem_operators.py:1430-1496 (caller scales by Gc etc.) */
int phastb_q4_energy_sums(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u,
                          const double* d, const double* v, double* out_host, void* workspace,
                          size_t workspace_bytes, void* stream);

/* Size of the small reduction workspace used by the *_sums / *_change entry points. */
size_t phastb_reduce_workspace_bytes(void);

/* Reaction sum_{i in nodes} f_int[i, comp] (- f_ext[i, comp]), FP64, host result.
 * compute_reaction_force, fem_operators.py:1502-1530 */
int phastb_q4_reaction(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u,
                       const double* d, const int64_t* nodes, int n_nodes_sel, int comp,
                       const double* f_ext, double* out_host, void* workspace,
                       size_t workspace_bytes, void* stream);
size_t phastb_q4_reaction_workspace_bytes(int n_nodes);

/* Consistent tangent action y = d f_int(u, d)/du [du] of the material's stress split at the
 * state u (FP64; d NULL: g = 1): the directional derivative of internal_force that
 * QuasiStaticSolver takes by autograd JVP for the spectral, Amor and star-convex splits,
 * mechanics_solver.py:1705-1733, 2000-2012.  For the linear splits it equals the force of du;
 * for the stress-spectral split it returns the force of du (the reference's linearisation). */
int phastb_q4_tangent_apply(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u,
                            const double* du, const double* d, double* y, void* stream);

/* Quasi-static Newton with matrix-free CG on K du = r, K the consistent tangent at the
 * iterate for the spectral, Amor and star-convex splits and K(d) itself for the linear ones.
 * QuasiStaticSolver.solve / _cg_solve / _accept_newton_step,
 * mechanics_solver.py:1597-1831, 1984-2043.  info[0] = Newton iterations,
 * info[1] = converged, info[2] = total CG iterations. */
size_t phastb_q4_qs_workspace_bytes(int n_nodes);
int phastb_q4_qs_solve(const phastb_q4_grid* g, const phastb_q4_material* m, const double* d,
                       const double* f_ext, const uint8_t* bc_mask, const double* bc_vals,
                       double* u, double tol, double cg_tol, int cg_max_iter, int max_iter,
                       int line_search, int ls_max_steps, double ls_min_alpha, double ls_c,
                       int* info, void* workspace, size_t workspace_bytes, void* stream);

/* ----------------------------------------------------- 3D (periodic H8) */
#define PHASTB_MAX_SLOTS 8
#define PHASTB_DRIVER_NONE 0
#define PHASTB_DRIVER_FULL 1
#define PHASTB_DRIVER_SPECTRAL 2

typedef struct {
  int nx, ny, nz;          /* voxels per axis (VoxelGrid.shape) */
  int px, py, pz;          /* periodic flags */
  double hx, hy, hz;       /* voxel size */
} phastb_voxel_grid;

typedef struct {
  int n_slots;                           /* material slots (<= PHASTB_MAX_SLOTS) */
  int isotropic;                         /* every slot isotropic: C from lam, mu */
  double C[PHASTB_MAX_SLOTS][36];        /* engineering-Voigt stiffness per slot */
  double lam[PHASTB_MAX_SLOTS], mu[PHASTB_MAX_SLOTS], Gc[PHASTB_MAX_SLOTS];
  int driver[PHASTB_MAX_SLOTS];          /* PHASTB_DRIVER_* */
  double kappa;                          /* residual stiffness of g */
  double ell;                            /* phase-field length */
} phastb_voxel_material;

/* Element scratch for the element->node gather: 24 values per element. */
size_t phastb_h8_scratch_bytes(const phastb_voxel_grid* g, int dtype);

/* g (E,8) = (1-kappa)(1-d_q)^2 + kappa.  operator.py:939-946, splits.py:56-59 */
int phastb_h8_degradation(const phastb_voxel_grid* g, int dtype, const void* d, double kappa,
                          void* g_out, void* stream);

/* y = [P^T sum_q w B^T g C (B u~ + E), sum w g C eps]; gq (E,8) or, when NULL, g from
 * d (n_red) (d NULL too: g = 1).  mask (n_mech,) uint8 zeroes fixed rows (NULL: none).
 * mech_action / _stress_pass, solid3d/operator.py:1108-1194 */
int phastb_h8_mech_apply(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                         int dtype, const void* x, const void* gq, const void* d, const uint8_t* mask,
                         void* y, void* scratch, void* stream);

/* Allocation-free variant of phastb_h8_mech_apply (same arguments, same result, no
 * scratch argument).  It has no counterpart in the reference: it serves callers that
 * cannot allocate device memory, such as a host runtime bound through a thin FFI with
 * no device-memory API, or an application whose GPU memory belongs entirely to another
 * allocator.  Its element scratch is a file-scope device array for at most
 * PHASTB_NOALLOC_MAX_VOXELS voxels (about 6.4 MB), held on every GPU that loads the
 * library until exit.  Larger grids return PHASTB_ERR_CAPACITY.  The array holds the
 * same workspace layout as the caller workspace of phastb_h8_mech_apply: a region of 24
 * words per voxel followed by the reduction block of the macro-stress rows; the tiled
 * action writes only the reduction block, whose offset grows with the grid, and that
 * layout is what bounds the voxel count.  The first call on a device looks up the
 * array's device address and keeps it for the process (make that first call before any
 * stream capture; a device reset, cudaDeviceReset, in the same process is not supported
 * afterwards, because the kept address may no longer be the array's).  The device current
 * at the call must own `stream`.  All calls share the one array, so calls that overlap on
 * the GPU (other streams, other host threads) race. */
#define PHASTB_NOALLOC_MAX_VOXELS 32768
int phastb_h8_mech_apply_noalloc(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                 const uint8_t* slot, int dtype, const void* x, const void* gq,
                                 const void* d, const uint8_t* mask, void* y, void* stream);

/* Tile shape of the elastic action for a grid and word size (no reference counterpart: the
 * reference action is a batched gather/matmul/scatter).  shape = {ox, oy, kz}: owned nodes per
 * block in x and y and node layers per block in z; (ox+1)(oy+1) <= 256; kz = 0 lets each launch
 * pick the depth from the kernel's occupancy.  set = 0 reads the shape in use (the recorded
 * one, else a heuristic), set = 1 records `shape` for this grid. */
int phastb_h8_tile_shape(const phastb_voxel_grid* g, int dtype, int set, int* shape);

/* Times the elastic action over candidate tile shapes on the caller's buffers (x, d, slot
 * as for phastb_h8_mech_apply; y is overwritten), records the fastest for this grid and
 * word size and returns it in shape[3] and its time per action in *ms.  Must not be called
 * while `stream` is being captured.  scratch: phastb_h8_scratch_bytes. */
int phastb_h8_autotune(const phastb_voxel_grid* g, const phastb_voxel_material* m, int dtype,
                       const uint8_t* slot, const void* x, const void* d, void* y, void* scratch,
                       size_t scratch_bytes, int* shape, float* ms, void* stream);

/* Jacobi diagonal of A(g).  mech_diagonal, operator.py:1196-1254 */
int phastb_h8_mech_diagonal(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                            const uint8_t* slot, int dtype, const void* gq, const void* d, void* diag,
                            void* scratch, void* stream);

/* r_E (6) and elastic energy, FP64 host results.  macro_stress/elastic_energy,
 * operator.py:1303-1340 */
int phastb_h8_stress_energy(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                            const uint8_t* slot, const double* x, const double* gq, const double* d,
                            double* rE_host, double* energy_host, void* scratch, void* stream);

/* Y (E,8) undamaged driving energy and H_out = max(H_prev, Y) (either output NULL).
 * driving_force operator.py:1415-1444, spectral_tensile_energy splits.py:146-161,
 * history max staggered.py:1302 */
int phastb_h8_driving_history(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                              const uint8_t* slot, const double* x, const double* H_prev,
                              double* Y, double* H_out, void* stream);

/* scale * [Gc_e (M/ell + ell L) d + 2(1-kappa) sum_q w H_q N_q N_q^T d]; H NULL drops
 * the history term.  damage_action, operator.py:1450-1466 */
int phastb_h8_damage_apply(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                           const uint8_t* slot, const double* d, const double* H, double scale,
                           double* y, void* scratch, void* stream);

/* scale * rhs and scale * Jacobi diagonal.  damage_rhs/damage_diagonal, operator.py:1468-1493 */
int phastb_h8_damage_rhs_diag(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                              const uint8_t* slot, const double* H, double scale, double* rhs,
                              double* diag, void* scratch, void* stream);

/* Constrained Jacobi-PCG mechanics solve at fixed damage (g from d, or gq).
 * solve_constrained + pcg, solid3d/linalg.py:99-287.
 * info[0] iterations, info[1] converged; rinfo[0] ||b_f||, rinfo[1] ||r||. */
size_t phastb_h8_mech_solve_workspace_bytes(const phastb_voxel_grid* g, int dtype);
int phastb_h8_mech_solve(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                         const uint8_t* slot, const double* gq, const double* d,
                         const uint8_t* fixed, const double* fixed_values, const double* x0,
                         double rtol, double atol, int maxiter, int check_every, double* x_out,
                         int* info, double* rinfo, void* workspace, size_t workspace_bytes,
                         void* stream);

/* Options of the extended mechanics solve. */
typedef struct {
  int precond;        /* 0 Jacobi (the reference's), 1 geometric multigrid V-cycle */
  int mixed;          /* 0 FP64 PCG; 1 FP32 inner PCG (FP64 dot products) + FP64 iterative refinement */
  int levels;         /* multigrid levels, 2 or 3 (grid edges divisible by 2^(levels-1)) */
  int smooth_degree;  /* Chebyshev degree of the pre/post smoother */
  int coarse_degree;  /* Chebyshev degree on the coarsest level */
  int power_iters;    /* power iterations for lambda_max(D^-1 A) per level */
  double lmax_safety; /* Chebyshev interval [lambda_max/30, lmax_safety * lambda_max] */
  double inner_rtol;  /* mixed: relative residual reduction of each inner FP32 solve */
  int max_refine;     /* mixed: most refinement steps */
} phastb_mech_opts;

/* Constrained mechanics solve A(g(d)) x = 0 with x = fixed_values on fixed, stopped on the
 * FP64 residual ||r|| <= max(rtol ||b_f||, atol) like solve_constrained (linalg.py:223-287),
 * with a multigrid preconditioner and/or FP32 inner solves under FP64 iterative refinement
 * (after mixed_precision_cg.py:18-95).  The voxel multigrid has no counterpart in PhAST's 3D
 * code (its 2D GMG/AMG semantics: multigrid.py:534-576, 996-1089).  info[0] iterations,
 * info[1] converged; rinfo[0] ||b_f||, rinfo[1] final FP64 ||r||.  lmax_io (host, one value per
 * multigrid level, may be NULL): when lmax_io[0] > 0 these lambda_max(D^-1 A) estimates are used,
 * otherwise they are estimated by power iteration and written back, so a caller can reuse them
 * across the solves of one load increment.  Returns 0 bytes for unsupported options (grid not
 * divisible for the requested levels). */
size_t phastb_h8_mech_solve_ex_workspace_bytes(const phastb_voxel_grid* g, const phastb_mech_opts* o);
int phastb_h8_mech_solve_ex(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                            const uint8_t* slot, const double* d, const uint8_t* fixed,
                            const double* fixed_values, const double* x0, double rtol, double atol,
                            int maxiter, int check_every, const phastb_mech_opts* o, double* lmax_io,
                            double* x_out, int* info, double* rinfo, void* workspace,
                            size_t workspace_bytes, void* stream);

/* phastb_h8_mech_solve_ex with a Gauss-point degradation gq (E,8) in every operator (the fine
 * action, the smoother, the Jacobi diagonal and the coarse moduli) in place of g(d): the
 * multigrid and FP32 forms for the PF-CZM law, whose g is not the AT2 g(d). */
size_t phastb_h8_mech_solve_ex_g_workspace_bytes(const phastb_voxel_grid* g, const phastb_mech_opts* o);
int phastb_h8_mech_solve_ex_g(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* gq, const uint8_t* fixed, const double* fixed_values, const double* x0,
                              double rtol, double atol, int maxiter, int check_every, const phastb_mech_opts* o,
                              double* lmax_io, double* x_out, int* info, double* rinfo, void* workspace,
                              size_t workspace_bytes, void* stream);

/* Box-constrained damage solve lower <= d <= upper by the primal active-set method
 * with a Dirichlet PCG per set (scale applied to the system).
 * solve_h8_scalar_box_kkt + solve_h8_scalar_dirichlet_pcg, solvers/box_kkt_h8.py:256-778.
 * info[0] total PCG iterations, info[1] active-set iterations, info[2] kkt_ok. */
size_t phastb_h8_box_kkt_workspace_bytes(const phastb_voxel_grid* g);
int phastb_h8_damage_box_kkt(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                             const uint8_t* slot, const double* H, double scale, const double* lower,
                             double upper, const double* initial, double lin_tol, double kkt_tol,
                             int max_lin, int max_active, double* d_out, int* info, void* workspace,
                             size_t workspace_bytes, void* stream);

/* f = dF/du . du on T3: the consistent tangent of the split-aware internal force at u, the
 * autograd JVP QuasiStaticSolver takes as its CG operator (mechanics_solver.py:1705-1733); the
 * T3 counterpart of phastb_q4_tangent_apply.  d NULL means g = 1. */
int phastb_t3_tangent_apply(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                            const double* du, const double* d, double* f, void* stream);

/* ---- Anderson mixing of the staggered damage fixed point ----
 * Type II Anderson mixing of d = G(d) with the last depth + 1 pairs
 * (_AndersonAccelerator.step, solvers/staggered_solver.py:165-255).  hist holds
 * 2 (depth + 1) n doubles owned by the caller: rows 0..depth the residuals G(d) - d, rows
 * depth+1.. the outputs G(d), used as a ring.  `count` is the number of pairs already stored
 * (0 after a reset) and `head` the row the new pair (d_in, d_out) goes to; the caller advances
 * head = (head + 1) mod (depth + 1) and count = min(count + 1, depth + 1) after each call.
 * d_mix = G(d) when there is no history, the normal equations (+ reg I) are singular or the
 * mix's residual is above 1.5x that of G(d) (*used_host = 0); otherwise the mix clamped to
 * [floor, 1] (floor NULL: 0), *used_host = 1.  depth <= 6. */
size_t phastb_anderson_workspace_bytes(int depth);
int phastb_anderson_step(int n, int depth, int count, int head, double* hist, const double* d_in,
                         const double* d_out, const double* floor, double reg, double* d_mix, int* used_host,
                         void* workspace, size_t workspace_bytes, void* stream);

/* Projected Anderson mixing of the 3D staggered damage fixed point (ProjectedAnderson,
 * solid3d/staggered.py:290-376) on the same ring: push (d_in, d_out) into row `head`; with
 * want_mix and at least two pairs, d_mix = clamp(d_out - dG gamma, lower, upper) where gamma
 * solves the normal equations of the unit-norm residual differences (zero columns dropped)
 * with `reg` on the diagonal.  *status_host: 0 no mix (too few pairs, every difference zero, a
 * singular system or a non-finite mix), 1 a mix that differs from d_out, 2 a mix equal to it. */
int phastb_anderson_projected(int n, int depth, int count, int head, double* hist, const double* d_in,
                              const double* d_out, int want_mix, const double* lower, double upper, double reg,
                              double* d_mix, int* status_host, void* workspace, size_t workspace_bytes,
                              void* stream);

/* ---- PF-CZM damage law (SolverConfig.damage_law = 'pfczm') ----
 * Wu's rational degradation g = (1 - kappa) A/(A + Q) + kappa, A = (1 - d)^p,
 * Q = a1 d (1 + a2 d + a2 a3 d^2) (physics/pfczm.py:79-125) with a1 per material slot,
 * a1 = 4 E_ref Gc / (pi ell f_t^2 (1 - kappa)) (pfczm.py:16-31, operator.py:326-392), and the
 * softening constants of pfczm_softening_parameters (pfczm.py:57-65).  Gc, ell and kappa
 * come from the phastb_voxel_material. */
typedef struct {
  double a1[PHASTB_MAX_SLOTS];
  double a2, a3;  /* softening: linear (-1/2, 0), exponential (2^(5/3) - 3, 0) */
  double p;       /* exponent of A, >= 2 */
} phastb_pfczm_law;

/* gq (E,8) = g(d_q), the degradation the elastic action and solve take as gq.
 * degradation, operator.py:939-946 */
int phastb_h8_pfczm_degradation(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                const phastb_pfczm_law* law, const uint8_t* slot, const double* d,
                                double* gq, void* stream);

/* Workspace of the PF-CZM energy, gradient, tangent action and diagonal. */
size_t phastb_h8_pfczm_workspace_bytes(const phastb_voxel_grid* g);

/* out_host[0] = the damage energy sum_q w H_q g(d_q) + Gc/(pi ell) int (2d - d^2)
 * + Gc ell/pi int |grad d|^2 (H NULL: no history term), [1] the history term, [2] the local
 * surface part, [3] the gradient surface part, [4..4+PHASTB_MAX_SLOTS) the surface energy by
 * slot.  pfczm_damage_energy operator.py:465-489, _pfczm_fracture_energy :608-631 */
#define PHASTB_PFCZM_ENERGY_WORDS (4 + PHASTB_MAX_SLOTS)
int phastb_h8_pfczm_energy(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                           const phastb_pfczm_law* law, const uint8_t* slot, const double* d, const double* H,
                           double* out_host, void* workspace, size_t workspace_bytes, void* stream);

/* grad = scale * d(energy)/dd.  pfczm_damage_gradient, operator.py:491-513 */
int phastb_h8_pfczm_gradient(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                             const phastb_pfczm_law* law, const uint8_t* slot, const double* d, const double* H,
                             double scale, double* grad, void* workspace, size_t workspace_bytes, void* stream);

/* W (E,8) = max(H g''(d_q) - 2 Gc/(pi ell), 0.25 * 2 Gc/(pi ell)), the Gauss-point curvatures
 * of the Newton tangent.  pfczm_tangent_weights, operator.py:515-539 */
int phastb_h8_pfczm_tangent_weights(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                    const phastb_pfczm_law* law, const uint8_t* slot, const double* d,
                                    const double* H, double* W, void* stream);

/* y = scale * [Gc (2 ell/pi) L f + sum_q w W_q N_q N_q^T f], and its Jacobi diagonal.
 * pfczm_tangent_action / pfczm_tangent_diagonal, operator.py:541-566 */
int phastb_h8_pfczm_tangent_apply(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                  const uint8_t* slot, const double* W, const double* f, double scale, double* y,
                                  void* workspace, size_t workspace_bytes, void* stream);
int phastb_h8_pfczm_tangent_diagonal(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                     const uint8_t* slot, const double* W, double scale, double* diag,
                                     void* workspace, size_t workspace_bytes, void* stream);

/* Projected Newton solve of the PF-CZM damage energy over lower <= d <= 1 from `initial`,
 * each step a box-QP of the tangent (the box-KKT solve above, at kkt_tol / 10) with an
 * Armijo line search and projected step doubling, stopped when the projected scaled gradient
 * is at most kkt_tol in the max norm.  lin_tol is SolverConfig.damage_linear_tol.
 * info[0] PCG iterations, info[1] active-set iterations, info[2] Newton iterations,
 * info[3] failure reason (0 none, 1 non-finite energy, 2 non-finite gradient, 3 box-QP
 * failed, 4 line search failed, 5 Newton limit); rinfo[0] final projected gradient,
 * rinfo[1] final energy.  StaggeredSolver._damage_pfczm, solid3d/staggered.py:843-1096 */
size_t phastb_h8_pfczm_solve_workspace_bytes(const phastb_voxel_grid* g);
int phastb_h8_pfczm_damage_solve(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                 const phastb_pfczm_law* law, const uint8_t* slot, const double* H, double scale,
                                 const double* lower, const double* initial, double kkt_tol, double lin_tol,
                                 int max_lin, int max_active, int max_newton, double* d_out, int* info,
                                 double* rinfo, void* workspace, size_t workspace_bytes, void* stream);

/* The increment record (phastb_h8_increment_record) with the elastic part at the given
 * degradation gq (NULL: g(d) of AT2) and, with law non-NULL, the PF-CZM surface energy
 * Gc/(pi ell) int (2d - d^2) + Gc ell/pi int |grad d|^2 in [13:23).  _pfczm_fracture_energy,
 * operator.py:608-631 */
int phastb_h8_increment_record_ex(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                  const uint8_t* slot, const double* x, const double* gq, const double* d,
                                  const double* H, double threshold, const phastb_pfczm_law* law,
                                  double* out_host, void* workspace, size_t workspace_bytes, void* stream);

/* ---- crack closure (SolverConfig.crack_closure = 'axes'), isotropic group ----
 * Elements with a damage driver add back (1 - g) of psi_c = sum_k k_k/2 <v_k . eps>-^2 with
 * the rows v = (trace, e_x, e_y, e_z) and moduli (lam, 2 mu, 2 mu, 2 mu) of their slot
 * (splits.py:486-503).  A sign pattern is one byte per Gauss point, (E,8): bit k set where
 * v_k . eps < 0 (ClosurePattern.iso, model.py:1200-1223); a fixed pattern makes the
 * add-back linear.  Workspace of the calls below: phastb_h8_closure_workspace_bytes. */
size_t phastb_h8_closure_workspace_bytes(const phastb_voxel_grid* g);

/* pattern (E,8) of state x.  closure_pattern, operator.py:821-834 */
int phastb_h8_closure_pattern(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* x, uint8_t* pattern, void* stream);

/* New pattern of x and *changed_host = whether a flipped bit's stress jump (1 - g) k |v . eps|
 * exceeds tolerance x the largest k |v . eps|.  closure_pattern_change, operator.py:836-873 */
int phastb_h8_closure_pattern_change(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                     const uint8_t* slot, const double* x, const double* gq,
                                     const uint8_t* pattern_old, double tolerance, uint8_t* pattern_new,
                                     int* changed_host, void* workspace, size_t workspace_bytes, void* stream);

/* y += the add-back's internal force at x (pattern NULL: each point's own signs); rows with
 * mask set are left alone.  The closure terms of _stress_pass_closure, operator.py:1039-1108 */
int phastb_h8_closure_apply_add(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                const double* x, const double* gq, const uint8_t* pattern, const uint8_t* mask,
                                double* y, void* workspace, size_t workspace_bytes, void* stream);

/* diag += the add-back's Jacobi-diagonal terms (pattern NULL: every bit).  _closure_diagonal,
 * operator.py:1274-1302 */
int phastb_h8_closure_diagonal_add(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                   const uint8_t* slot, const double* gq, const uint8_t* pattern, double* diag,
                                   void* workspace, size_t workspace_bytes, void* stream);

/* out_host[0] = the add-back's energy sum w (1 - g) psi_c, [1..3] its r_E rows xx, yy, zz
 * (pattern NULL: each point's own signs), to add to phastb_h8_stress_energy.
 * operator.py:1039-1108 */
int phastb_h8_closure_energy(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                             const double* x, const double* gq, const uint8_t* pattern, double* out_host,
                             void* workspace, size_t workspace_bytes, void* stream);

/* out_host[0..2] = [smallest element-mean normal strain, smallest principal value of the
 * element-mean strains, smallest Gauss-point det(I + grad u)], out_host[3..5] the same over the
 * elements whose mean nodal damage exceeds threshold (+inf when there are none or d is NULL).
 * kinematic_guard, operator.py:1713-1770; workspace phastb_reduce_workspace_bytes. */
int phastb_h8_kinematic_guard(const phastb_voxel_grid* g, const double* x, const double* d, double threshold,
                              double* out_host, void* workspace, size_t workspace_bytes, void* stream);

/* The constrained mechanics solve of phastb_h8_mech_solve with the closure add-back of a fixed
 * pattern in the operator and in its Jacobi diagonal (the linear solve of each closure pattern
 * iteration, StaggeredSolver._linear_mechanics, staggered.py:550-587). */
size_t phastb_h8_mech_solve_closure_workspace_bytes(const phastb_voxel_grid* g);
int phastb_h8_mech_solve_closure(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                 const double* gq, const uint8_t* pattern, const uint8_t* fixed,
                                 const double* fixed_values, const double* x0, double rtol, double atol,
                                 int maxiter, int check_every, double* x_out, int* info, double* rinfo,
                                 void* workspace, size_t workspace_bytes, void* stream);

/* Staggered change parts out[0..4] = ||du~||, ||u~||, max|dE|, max|E|, max|dd| (FP64, host).
 * StaggeredSolver._change, solid3d/staggered.py:1097-1124 */
int phastb_h8_stagger_change(int n_u, const double* x_new, const double* x_old, int n_d,
                             const double* d_new, const double* d_old, double* out_host,
                             void* workspace, size_t workspace_bytes, void* stream);

/* Scalars of an accepted increment, FP64, one host read (out_host[PHASTB_RECORD_WORDS]):
 * [0:6] E (the macro unknowns of x), [6:12] r_E = sum w g sigma with g = g(d) (macro stress
 * times volume), [12] elastic energy 0.5 x.A(g) x, [13:13+PHASTB_MAX_SLOTS] fracture energy
 * by material slot, [21] its local part Gc/(2 ell) d.M d, [22] its gradient part
 * Gc ell/2 d.L d, [23] sum of the element-mean damage (mean of the 8 corners), [24] number
 * of elements whose mean damage >= threshold, [25] max H (0 when H is NULL), [26] max d.
 * x NULL skips the mechanics part ([0:13] are then 0).
 * The record of StaggeredSolver._attempt, solid3d/staggered.py:1436-1499, with
 * macro_stress / elastic_energy (operator.py:1303-1340) and fracture_energy
 * (operator.py:1511-1545). */
#define PHASTB_RECORD_WORDS 27
size_t phastb_h8_record_workspace_bytes(const phastb_voxel_grid* g);
int phastb_h8_increment_record(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                               const uint8_t* slot, const double* x, const double* d, const double* H,
                               double threshold, double* out_host, void* workspace,
                               size_t workspace_bytes, void* stream);

/* ||rhs - A d|| of the (scaled) damage system of history H, FP64, host result: the
 * residual that sets the linear tolerance of the damage solve.
 * StaggeredSolver._damage, solid3d/staggered.py:766-770 */
size_t phastb_h8_damage_residual_workspace_bytes(const phastb_voxel_grid* g);
int phastb_h8_damage_residual_norm(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                   const uint8_t* slot, const double* H, double scale, const double* d,
                                   double* norm_host, void* workspace, size_t workspace_bytes,
                                   void* stream);

/* out = factor * x, then out[index] = value (index < 0: none); n FP64 entries.  The
 * staggered predictor x * (target / previous) with E[c] = target,
 * StaggeredSolver._predictor, solid3d/staggered.py:1207-1213 */
int phastb_scale_set(int n, const double* x, double factor, int index, double value, double* out,
                     void* stream);

/* 1 when the elastic action on this grid and word size stages its node layers with TMA tensor
 * copies (rx a multiple of 16 bytes' worth of words, the driver's tensor-map encoder present,
 * PHASTB_TMA not 0), 0 when it stages them through registers, -1 on bad arguments.  No reference
 * counterpart: it reports how this backend's kernel loads the operator's halo tiles. */
int phastb_h8_tma_staging(const phastb_voxel_grid* g, int dtype);

/* Self-test of the bounded grid barrier that the persistent damage CG uses (no counterpart in
 * the reference).  A cooperative launch of `blocks` blocks passes two barriers; block
 * `skip_block` (< 0: none) never arrives, so the other blocks' first wait runs out after
 * limit_s seconds (at most 10) of GPU time and the kernel ends with the error flag set.
 * Returns PHASTB_ERR_CUDA with *grid_error_host = 1 in that case, PHASTB_OK with 0 otherwise;
 * *passed_host counts the blocks that passed both barriers. */
int phastb_test_grid_barrier(int blocks, int skip_block, double limit_s, int* grid_error_host,
                             int* passed_host);

/* ---- Packed batches of periodic voxel cells --------------------------------------------
 * PhAST runs one cell per Problem.run (solid3d/api.py:191-233); these entry points advance
 * many cells of different sizes together.  A batch plan fixes the cells' grids, phase-field
 * lengths and damage-system scales (operator.py:238) and the packed layout: cell c's reduced
 * nodes, mechanics unknowns [u~ (3 n_red), E (6)] and elements follow those of cells
 * 0..c-1.  Each Krylov iteration is one launch per operator apply and per vector step over
 * every cell (one block per brick of a cell, one per chunk of a cell's vector), with every
 * cell's solver state and stopping rule on the device, as the single-cell solves above. */
typedef struct phastb_batch phastb_batch;

/* Host plan of n_cells cells (NULL on bad arguments): bricks of ox x oy nodes (16 x 8 or
 * 8 x 8) and kz node layers, at most 1184 bricks per cell.  ell and dscale: per cell. */
phastb_batch* phastb_batch_create(int n_cells, const phastb_voxel_grid* grids, const double* ell,
                                  const double* dscale, int ox, int oy, int kz);
void phastb_batch_destroy(phastb_batch* batch);

/* out[0..6] = packed nodes, mechanics unknowns, elements, brick blocks, bytes of the device
 * tables (phastb_batch_bind), mechanics chunks, node chunks; then per cell c
 * out[7 + 3c .. 9 + 3c] = its node, mechanics and element offsets. */
int phastb_batch_sizes(const phastb_batch* batch, long long* out);

/* Copies the plan's tables into the caller's device buffer (out[4] bytes), which must stay
 * allocated while the plan is used; synchronises `stream`. */
int phastb_batch_bind(phastb_batch* batch, void* tables, size_t bytes, void* stream);

/* Batched elastic action y = A(d) x of every cell (mech_action, operator.py:1108-1194);
 * rE_out (host, 6 per cell, may be NULL) receives each cell's macro-stress row sums. */
size_t phastb_batch_apply_workspace_bytes(const phastb_batch* batch);
int phastb_batch_mech_apply(const phastb_batch* batch, const phastb_voxel_material* m, const uint8_t* slot,
                            int dtype, const void* x, const void* d, const uint8_t* mask, void* y,
                            double* rE_out, void* workspace, size_t workspace_bytes, void* stream);

/* Batched damage action of every cell, scaled by each cell's dscale when `scaled`
 * (damage_action, operator.py:1450-1466). */
int phastb_batch_damage_apply(const phastb_batch* batch, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* d, const double* H, int scaled, const uint8_t* mask, double* y,
                              void* workspace, size_t workspace_bytes, void* stream);

/* Constrained mechanics solve of every cell (solve_constrained, solid3d/linalg.py:223-287):
 * Jacobi PCG in FP64 (mixed = 0) or FP32 inner PCG with FP64 dot products under FP64
 * iterative refinement (mixed = 1, after mixed_precision_cg.py:18-95), each cell stopped on
 * its FP64 residual ||r|| <= max(rtol ||b_f||, atol).  info[2c] iterations, info[2c+1]
 * converged; rinfo[2c] ||b_f||, rinfo[2c+1] final ||r||.  live_host (host, one int per cell,
 * NULL: every cell) selects the cells solved; the others keep x0 in x_out.  Returns the first
 * failing cell's status (PHASTB_OK when every cell converged). */
size_t phastb_batch_mech_solve_workspace_bytes(const phastb_batch* batch, int mixed);
int phastb_batch_mech_solve(const phastb_batch* batch, const phastb_voxel_material* m, const uint8_t* slot,
                            const double* d, const uint8_t* fixed, const double* fixed_values, const double* x0,
                            double rtol, double atol, int maxiter, int check_every, int mixed, double inner_rtol,
                            int max_refine, const int* live_host, double* x_out, int* info, double* rinfo,
                            void* workspace, size_t workspace_bytes, void* stream);

/* phastb_batch_mech_solve with the options of phastb_h8_mech_solve_ex: precond = 1 (with mixed = 1
 * and levels = 3) preconditions every cell's FP32 inner PCG with the voxel multigrid V-cycle of
 * phastb_h8_mech_solve_ex, all cells in the same launches (every cell's edges divisible by 4 and at
 * least 32, periodic).  reuse_lmax = 1 keeps the per-cell lambda_max estimates of the previous
 * call with the same workspace.  The voxel multigrid has no counterpart in PhAST's 3D code (its 2D
 * GMG semantics: multigrid.py:534-576, 996-1089). */
size_t phastb_batch_mech_solve_ex_workspace_bytes(const phastb_batch* batch, const phastb_mech_opts* o);
int phastb_batch_mech_solve_ex(const phastb_batch* batch, const phastb_voxel_material* m, const uint8_t* slot,
                               const double* d, const uint8_t* fixed, const double* fixed_values, const double* x0,
                               double rtol, double atol, int maxiter, int check_every, const phastb_mech_opts* o,
                               int reuse_lmax, const int* live_host, double* x_out, int* info, double* rinfo,
                               void* workspace, size_t workspace_bytes, void* stream);

/* Box-constrained damage solve of every cell's scaled system (solve_h8_scalar_box_kkt,
 * solvers/box_kkt_h8.py:256-778).  tol_rule = 1 sets each cell's linear tolerance as the
 * staggered solver does, max(min(lin_tol, 0.1 kkt_tol / max(r0, 1)), min_tol) with r0 the
 * residual of `initial` (StaggeredSolver._damage, solid3d/staggered.py:753-800); 0 uses
 * lin_tol.  info[4c..4c+3] = PCG iterations, active-set iterations, kkt_ok, status;
 * rinfo[2c], rinfo[2c+1] = r0 and the tolerance used (rinfo may be NULL).  live_host as for
 * phastb_batch_mech_solve; cells not solved return `initial` in d_out. */
size_t phastb_batch_box_kkt_workspace_bytes(const phastb_batch* batch);
int phastb_batch_damage_box_kkt(const phastb_batch* batch, const phastb_voxel_material* m, const uint8_t* slot,
                                const double* H, const double* lower, double upper, const double* initial,
                                double lin_tol, double kkt_tol, double min_tol, int tol_rule, int max_lin,
                                int max_active, const int* live_host, double* d_out, int* info, double* rinfo,
                                void* workspace, size_t workspace_bytes, void* stream);

/* Predictor of the next increment of every cell: x_out = factor * x with each cell's
 * E[component] = value, and values_out (may be NULL) = 0 except each cell's E[component] =
 * value (StaggeredSolver._predictor and mech_fixed_values, solid3d/staggered.py:1207-1213). */
int phastb_batch_predictor(const phastb_batch* batch, const double* x, double factor, int component,
                           double value, double* x_out, double* values_out, void* stream);

/* Staggered change parts of every cell, out_host[5c..5c+4] = ||du~||, ||u~||, max|dE|,
 * max|E|, max|dd| (StaggeredSolver._change, solid3d/staggered.py:1097-1124). */
size_t phastb_batch_change_workspace_bytes(const phastb_batch* batch);
int phastb_batch_stagger_change(const phastb_batch* batch, const double* x_new, const double* x_old,
                                const double* d_new, const double* d_old, double* out_host, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Library version string (host pointer). */
const char* phastb_version(void);

/* Number of kernel launches this library has issued in the process (host counter). */
long long phastb_launch_count(void);
void phastb_launch_count_reset(void);

#ifdef __cplusplus
}
#endif
#endif /* PHASTB_H */
