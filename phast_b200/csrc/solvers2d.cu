// 2D solver drivers over the structured-Q4 operators: the bound-projected
// PCG damage solve and the quasi-static Newton / matrix-free CG mechanics.
#include "engine.cuh"

#include <cstddef>
#include <cstring>
#include "q4_kernels.cuh"

#include <cmath>
#include <vector>

namespace phastb {

int q4_damage_apply_launch(const phastb_q4_grid* g, const double* d, const double* Hq, double rs, double rsh,
                           const double* rsh_e, double gcl0, const double* gcl0_e, double* y, const int* guard,
                           cudaStream_t s, const uint8_t* mask);
int q4_damage_adjoint_launch(const phastb_q4_grid* g, const double* lam, const double* d, double l0, double* g_gc,
                             double* g_h, double* lkd, double* lmd, cudaStream_t s);
int q4_force_launch(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* d,
                    double* f, const uint8_t* mask, const int* guard, cudaStream_t s);

struct Q4DamageCtx {
  phastb_q4_grid g;
  const double* Hq;
  double rsh;
  const double* rsh_e;
  double gcl0;
  const double* gcl0_e;
  const uint8_t* mask;  // rows held fixed (zero output), may be null
};

static int q4_damage_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const Q4DamageCtx* k = static_cast<const Q4DamageCtx*>(c);
  return q4_damage_apply_launch(&k->g, x, k->Hq, 2.0, k->rsh, k->rsh_e, k->gcl0, k->gcl0_e, y, guard, s, k->mask);
}

// Dirichlet-eliminated linear system set-up: bf = rhs on free rows (0 on fixed),
// x = vals on fixed rows (x0 or 0 elsewhere), Jacobi inverse zero on fixed rows.
__global__ void lin_setup_kernel(int n, const double* __restrict__ rhs, const uint8_t* __restrict__ fixed,
                                 const double* __restrict__ vals, const double* __restrict__ x0,
                                 double* __restrict__ bf, double* __restrict__ x, double* __restrict__ minv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool f = fixed && fixed[i];
    bf[i] = f ? 0.0 : rhs[i];
    x[i] = f ? (vals ? vals[i] : 0.0) : (x0 ? x0[i] : 0.0);
    if (f) minv[i] = 0.0;
  }
}

struct Q4ForceCtx {
  phastb_q4_grid g;
  phastb_q4_material m;
  const double* d;
  const uint8_t* mask;
};

static int q4_force_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const Q4ForceCtx* k = static_cast<const Q4ForceCtx*>(c);
  return q4_force_launch(&k->g, &k->m, x, k->d, y, k->mask, guard, s);
}

int q4_tangent_launch(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* du,
                      const double* d, double* f, const uint8_t* mask, const int* guard, cudaStream_t s);

// The consistent tangent at the Newton iterate `u` (read at every apply, so one
// context serves every Newton step of a solve).
struct Q4TangentCtx {
  phastb_q4_grid g;
  phastb_q4_material m;
  const double* d;
  const uint8_t* mask;
  const double* u;
};

static int q4_tangent_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const Q4TangentCtx* k = static_cast<const Q4TangentCtx*>(c);
  return q4_tangent_launch(&k->g, &k->m, k->u, x, k->d, y, k->mask, guard, s);
}

// residual r = (f_ext - f) * free, and u[bc] = bc_vals helpers
__global__ void qs_residual_kernel(int n2, const double* __restrict__ fext, const double* __restrict__ f,
                                   const uint8_t* __restrict__ bcm, double* __restrict__ r, RedWs ws) {
  double acc[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    const double v = bcm[i] ? 0.0 : (fext ? fext[i] : 0.0) - f[i];
    r[i] = v;
    acc[0] += v * v;
    acc[1] += isfinite(v) ? 0.0 : 1.0;
  }
  reduce_multi<2>(acc, ws);
}

__global__ void qs_axpy_bc_kernel(int n2, const double* __restrict__ u, double alpha, const double* __restrict__ du,
                                  const uint8_t* __restrict__ bcm, const double* __restrict__ bcv,
                                  double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x)
    out[i] = bcm[i] ? bcv[i] : (du ? u[i] + alpha * du[i] : u[i]);
}

__global__ void copy_kernel(int n, const double* __restrict__ a, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

__global__ void zero_kernel(int n, double* __restrict__ a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 0.0;
}

bool t3_valid_mesh(const phastb_t3_mesh* m);
int t3_force_launch(const phastb_t3_mesh& mesh, const phastb_q4_material& m, const double* u, const double* d,
                    double* f, const uint8_t* mask, const int* guard, cudaStream_t s);
int t3_damage_apply_launch(const phastb_t3_mesh& mesh, const double* d, const double* H, double gco,
                           const double* gco_e, double gcl0, const double* gcl0_e, double* y, const int* guard,
                           cudaStream_t s, const uint8_t* mask);

// T3 operator contexts for the Krylov engines (hashed as bytes: zeroed before filling).
struct T3ForceCtx {
  phastb_t3_mesh mesh;
  phastb_q4_material m;
  const double* d;
  const uint8_t* mask;
};

static int t3_force_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const T3ForceCtx* k = static_cast<const T3ForceCtx*>(c);
  return t3_force_launch(k->mesh, k->m, x, k->d, y, k->mask, guard, s);
}

int t3_tangent_launch(const phastb_t3_mesh& mesh, const phastb_q4_material& m, const double* u, const double* du,
                      const double* d, double* f, const uint8_t* mask, const int* guard, cudaStream_t s);

// The consistent tangent at the Newton iterate `u` on T3 (as Q4TangentCtx).
struct T3TangentCtx {
  phastb_t3_mesh mesh;
  phastb_q4_material m;
  const double* d;
  const uint8_t* mask;
  const double* u;
};

static int t3_tangent_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const T3TangentCtx* k = static_cast<const T3TangentCtx*>(c);
  return t3_tangent_launch(k->mesh, k->m, k->u, x, k->d, y, k->mask, guard, s);
}

static int t3_force_eval(const void* c, const double* u, double* f, cudaStream_t s) {
  const T3ForceCtx* k = static_cast<const T3ForceCtx*>(c);
  return t3_force_launch(k->mesh, k->m, u, k->d, f, nullptr, nullptr, s);
}

struct T3DamageMaskCtx {
  phastb_t3_mesh mesh;
  const double* H;
  double gco;
  const double* gco_e;
  double gcl0;
  const double* gcl0_e;
  const uint8_t* mask;
};

static int t3_damage_mask_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const T3DamageMaskCtx* k = static_cast<const T3DamageMaskCtx*>(c);
  return t3_damage_apply_launch(k->mesh, x, k->H, k->gco, k->gco_e, k->gcl0, k->gcl0_e, y, guard, s, k->mask);
}

static bool valid_grid(const phastb_q4_grid* g) {
  return g && g->nx >= 1 && g->ny >= 1 && g->hx > 0 && g->hy > 0 &&
         (long long)(g->nx + 1) * (g->ny + 1) < (1LL << 30);
}

// Newton-Raphson on f_int(u) = f_ext over the free dofs with K (the masked force operator)
// solved by plain CG per step and the residual-backtracking line search of _accept_newton_step
// (mechanics_solver.py:1597-1831).  ``force`` evaluates the unmasked f_int for the residual.
using ForceEval = int (*)(const void* ctx, const double* u, double* f, cudaStream_t s);

static int qs_newton(int n2, const LinOp<double>& K, ForceEval force, const void* fctx, const double* f_ext,
                     const uint8_t* bc_mask, const double* bc_vals, double* u, double tol, double cg_tol,
                     int cg_max_iter, int max_iter, int line_search, int ls_max_steps, double ls_min_alpha,
                     double ls_c, int* info, void* workspace, cudaStream_t s) {
  char* p = static_cast<char*>(workspace);
  PcgWs<double> w = pcg_ws<double>(p, n2);
  p += pcg_ws_bytes<double>(n2);
  const size_t v = align_up(sizeof(double) * (size_t)n2);
  double* du = reinterpret_cast<double*>(p);
  double* res = reinterpret_cast<double*>(p + v);
  double* ut = reinterpret_cast<double*>(p + 2 * v);
  double* ub = reinterpret_cast<double*>(p + 3 * v);
  void* redbase = p + 4 * v;
  RedWs rw = red_ws(redbase);
  const int G = grid_for(n2);
  int st;
  if ((st = red_ws_reset(rw, s))) return st;

  // u[bc] = bc_vals
  { note_launch(); qs_axpy_bc_kernel<<<G, kThreads, 0, s>>>(n2, u, 0.0, nullptr, bc_mask, bc_vals, u); }

  auto residual_norm = [&](const double* uu, double* r, double* nrm, bool* finite) -> int {
    int e = force(fctx, uu, w.Ap, s);
    if (e) return e;
    { note_launch(); qs_residual_kernel<<<G, kThreads, 0, s>>>(n2, f_ext, w.Ap, bc_mask, r, rw); }
    if ((e = last_launch_status())) return e;
    double o[2];
    if ((e = red_ws_fetch(rw, o, 2, s))) return e;
    *nrm = std::sqrt(o[0]);
    *finite = o[1] == 0.0 && std::isfinite(o[0]);
    return PHASTB_OK;
  };

  int total_cg = 0;
  for (int it = 0; it < max_iter; ++it) {
    double rn;
    bool fin;
    if ((st = residual_norm(u, res, &rn, &fin))) return st;
    if (!std::isnan(rn) && rn <= tol) {
      if (info) { info[0] = it; info[1] = 1; info[2] = total_cg; }
      return PHASTB_OK;
    }
    if (!fin) {
      if (info) { info[0] = max_iter; info[1] = 0; info[2] = total_cg; }
      return PHASTB_NONFINITE;
    }
    // du = CG(K(d) restricted to free dofs, res)
    { note_launch(); zero_kernel<<<G, kThreads, 0, s>>>(n2, du); }
    PcgResult pr{};
    if ((st = pcg_run<double>(K, n2, w, res, nullptr, nullptr, du, cg_tol, cg_max_iter, 50, PCG_PERIODIC, 0.0,
                              &pr, s)))
      return st;
    total_cg += pr.iterations;
    if (pr.breakdown || pr.nonfinite) {
      if (info) { info[0] = it + 1; info[1] = 0; info[2] = total_cg; }
      return PHASTB_BREAKDOWN;
    }
    // accept the Newton step (_accept_newton_step)
    if (!line_search) {
      { note_launch(); qs_axpy_bc_kernel<<<G, kThreads, 0, s>>>(n2, u, 1.0, du, bc_mask, bc_vals, u); }
      continue;
    }
    double alpha = 1.0, best = INFINITY;
    bool have_best = false, accepted = false;
    const double baseline = std::max(rn, 1e-30);
    const int n_ls = std::max(1, ls_max_steps + 1);
    for (int ls = 0; ls < n_ls; ++ls) {
      { note_launch(); qs_axpy_bc_kernel<<<G, kThreads, 0, s>>>(n2, u, alpha, du, bc_mask, bc_vals, ut); }
      double tn;
      bool tf;
      if ((st = residual_norm(ut, w.z, &tn, &tf))) return st;
      if (tn < best) {
        best = tn;
        have_best = true;
        { note_launch(); copy_kernel<<<G, kThreads, 0, s>>>(n2, ut, ub); }
      }
      if (tf && tn <= (1.0 - ls_c * alpha) * baseline) {
        { note_launch(); copy_kernel<<<G, kThreads, 0, s>>>(n2, ut, u); }
        accepted = true;
        break;
      }
      alpha *= 0.5;
      if (alpha < ls_min_alpha) break;
    }
    if (!accepted) {
      if (have_best && best < baseline)
        { note_launch(); copy_kernel<<<G, kThreads, 0, s>>>(n2, ub, u); }
      else
        { note_launch(); qs_axpy_bc_kernel<<<G, kThreads, 0, s>>>(n2, u, 1.0, du, bc_mask, bc_vals, u); }
    }
    if ((st = last_launch_status())) return st;
  }
  if (info) { info[0] = max_iter; info[1] = 0; info[2] = total_cg; }
  return PHASTB_NONCONVERGED;
}

}  // namespace phastb

using namespace phastb;

extern "C" {

size_t phastb_q4_damage_solve_workspace_bytes(int n_nodes) { return ppcg_ws_bytes(n_nodes); }

int phastb_q4_damage_solve(const phastb_q4_grid* g, const double* Hq, double gc_over_l0, const double* gc_over_l0_e,
                           double gcl0, const double* gcl0_e, const double* d_prev, const double* d_init,
                           const uint8_t* fixed, const double* fixed_vals, double tol, int max_iter, int check_every,
                           double* d_out, int* info, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_grid(g) || !Hq || !d_prev || !d_out || max_iter < 0 || check_every < 1) return PHASTB_ERR_ARG;
  if (fixed && !fixed_vals) return PHASTB_ERR_ARG;
  const int n = (g->nx + 1) * (g->ny + 1);
  if (!workspace || workspace_bytes < ppcg_ws_bytes(n)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  PpcgWs w = ppcg_ws(workspace, n);
  int st = phastb_q4_damage_prepare(g, Hq, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, w.b, w.minv, (void*)s);
  if (st) return st;
  Q4DamageCtx ctx{*g, Hq, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, nullptr};
  LinOp<double> A{q4_damage_op, &ctx, sizeof(ctx)};
  int inf[2] = {0, 0};
  st = ppcg_solve(A, n, w, d_prev, d_init, fixed, fixed_vals, tol, max_iter, check_every, d_out, inf, s);
  if (info) {
    info[0] = inf[0];
    info[1] = inf[1];
  }
  return st;
}

size_t phastb_q4_damage_linear_workspace_bytes(int n_nodes) {
  return pcg_ws_bytes<double>(n_nodes) + 2 * align_up(sizeof(double) * (size_t)n_nodes) + red_ws_bytes();
}

int phastb_q4_damage_linear_solve(const phastb_q4_grid* g, const double* Hq, double gc_over_l0,
                                  const double* gc_over_l0_e, double gcl0, const double* gcl0_e, const double* rhs,
                                  const uint8_t* fixed, const double* fixed_vals, const double* x0, double rtol,
                                  int max_iter, int check_every, double* x_out, int* info, double* rinfo,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_grid(g) || !Hq || !rhs || !x_out || max_iter < 1 || check_every < 1 || !(rtol >= 0)) return PHASTB_ERR_ARG;
  const int n = (g->nx + 1) * (g->ny + 1);
  if (!workspace || workspace_bytes < phastb_q4_damage_linear_workspace_bytes(n)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  char* p = static_cast<char*>(workspace);
  PcgWs<double> w = pcg_ws<double>(p, n);
  p += pcg_ws_bytes<double>(n);
  const size_t vb = align_up(sizeof(double) * (size_t)n);
  double* bf = reinterpret_cast<double*>(p);
  double* minv = reinterpret_cast<double*>(p + vb);
  RedWs rw = red_ws(p + 2 * vb);
  int st;
  if ((st = red_ws_reset(rw, s))) return st;
  // Jacobi inverse of the full operator (the b output of prepare is not needed)
  if ((st = phastb_q4_damage_prepare(g, Hq, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, w.z, minv, (void*)s))) return st;
  { note_launch(); lin_setup_kernel<<<grid_for(n), kThreads, 0, s>>>(n, rhs, fixed, fixed_vals, x0, bf, x_out, minv); }
  if ((st = last_launch_status())) return st;
  double bn = 0.0;
  if ((st = vec_norm2<double>(bf, n, &bn, p + 2 * vb, s))) return st;
  if (rinfo) rinfo[0] = bn;
  Q4DamageCtx ctx{*g, Hq, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, fixed};
  LinOp<double> A{q4_damage_op, &ctx, sizeof(ctx)};
  PcgResult pr{};
  if (bn == 0.0) {
    pr.converged = 1;
  } else if ((st = pcg_run<double>(A, n, w, bf, minv, nullptr, x_out, rtol * bn, max_iter, check_every, PCG_FREEZE,
                                   0.0, &pr, s))) {
    return st;
  }
  if (info) {
    info[0] = pr.iterations;
    info[1] = pr.converged ? 0 : (pr.breakdown ? 2 : (pr.nonfinite ? 3 : 1));
  }
  if (rinfo) rinfo[1] = pr.rnorm;
  return cuda_status(cudaStreamSynchronize(s));
}

int phastb_q4_damage_adjoint_grads(const phastb_q4_grid* g, const double* lam, const double* d, double l0,
                                   double* grad_gc_e, double* grad_H, double* lam_K_d_e, double* lam_M_d_e,
                                   void* stream) {
  if (!valid_grid(g) || !lam || !d || !(l0 > 0)) return PHASTB_ERR_ARG;
  return q4_damage_adjoint_launch(g, lam, d, l0, grad_gc_e, grad_H, lam_K_d_e, lam_M_d_e, (cudaStream_t)stream);
}

size_t phastb_q4_qs_workspace_bytes(int n_nodes) {
  const int n2 = 2 * n_nodes;
  return pcg_ws_bytes<double>(n2) + 4 * align_up(sizeof(double) * (size_t)n2) + red_ws_bytes();
}

static int q4_force_eval(const void* c, const double* u, double* f, cudaStream_t s) {
  const Q4ForceCtx* k = static_cast<const Q4ForceCtx*>(c);
  return q4_force_launch(&k->g, &k->m, u, k->d, f, nullptr, nullptr, s);
}

int phastb_q4_qs_solve(const phastb_q4_grid* g, const phastb_q4_material* m, const double* d, const double* f_ext,
                       const uint8_t* bc_mask, const double* bc_vals, double* u, double tol, double cg_tol,
                       int cg_max_iter, int max_iter, int line_search, int ls_max_steps, double ls_min_alpha,
                       double ls_c, int* info, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_grid(g) || !m || !d || !bc_mask || !bc_vals || !u || cg_max_iter < 1 || max_iter < 0)
    return PHASTB_ERR_ARG;
  const int nn = (g->nx + 1) * (g->ny + 1), n2 = 2 * nn;
  if (!workspace || workspace_bytes < phastb_q4_qs_workspace_bytes(nn)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  // The context is hashed as bytes (graph cache): zero it, then copy the material's
  // fields without its trailing padding.
  Q4ForceCtx kctx;
  std::memset(&kctx, 0, sizeof(kctx));
  kctx.g = *g;
  std::memcpy(&kctx.m, m, offsetof(phastb_q4_material, psi_split) + sizeof(int));
  kctx.d = d;
  kctx.mask = bc_mask;
  // Splits whose stress is not linear in the strain take the consistent tangent at the
  // iterate, as the reference's autograd JVP does for the spectral, Amor and star-convex
  // splits (mechanics_solver.py:1705-1733); linear stresses and the stress-spectral split
  // (which the reference linearises by evaluating the force at the increment) use the force.
  const int sp = m->stress_split;
  const bool tangent = sp == PHASTB_SPLIT_AMOR || sp == PHASTB_SPLIT_SPECTRAL || sp == PHASTB_SPLIT_STAR_CONVEX;
  Q4TangentCtx tctx;
  std::memset(&tctx, 0, sizeof(tctx));
  tctx.g = *g;
  std::memcpy(&tctx.m, m, offsetof(phastb_q4_material, psi_split) + sizeof(int));
  tctx.d = d;
  tctx.mask = bc_mask;
  tctx.u = u;
  LinOp<double> K = tangent ? LinOp<double>{q4_tangent_op, &tctx, sizeof(tctx)}
                            : LinOp<double>{q4_force_op, &kctx, sizeof(kctx)};
  return qs_newton(n2, K, q4_force_eval, &kctx, f_ext, bc_mask, bc_vals, u, tol, cg_tol, cg_max_iter, max_iter,
                   line_search, ls_max_steps, ls_min_alpha, ls_c, info, workspace, scope.get());
}

size_t phastb_t3_qs_workspace_bytes(int n_nodes) { return phastb_q4_qs_workspace_bytes(n_nodes); }

int phastb_t3_qs_solve(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* d, const double* f_ext,
                       const uint8_t* bc_mask, const double* bc_vals, double* u, double tol, double cg_tol,
                       int cg_max_iter, int max_iter, int line_search, int ls_max_steps, double ls_min_alpha,
                       double ls_c, int* info, void* workspace, size_t workspace_bytes, void* stream) {
  if (!t3_valid_mesh(mesh) || !m || !d || !bc_mask || !bc_vals || !u || cg_max_iter < 1 || max_iter < 0)
    return PHASTB_ERR_ARG;
  const int n2 = 2 * mesh->n_nodes;
  if (!workspace || workspace_bytes < phastb_t3_qs_workspace_bytes(mesh->n_nodes)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  T3ForceCtx kctx;
  std::memset(&kctx, 0, sizeof(kctx));
  kctx.mesh = *mesh;
  std::memcpy(&kctx.m, m, offsetof(phastb_q4_material, psi_split) + sizeof(int));
  kctx.d = d;
  kctx.mask = bc_mask;
  // the splits whose stress is not linear in the strain take the consistent tangent (as on Q4)
  const int sp = m->stress_split;
  const bool tangent = sp == PHASTB_SPLIT_AMOR || sp == PHASTB_SPLIT_SPECTRAL || sp == PHASTB_SPLIT_STAR_CONVEX;
  T3TangentCtx tctx;
  std::memset(&tctx, 0, sizeof(tctx));
  tctx.mesh = *mesh;
  std::memcpy(&tctx.m, m, offsetof(phastb_q4_material, psi_split) + sizeof(int));
  tctx.d = d;
  tctx.mask = bc_mask;
  tctx.u = u;
  LinOp<double> K = tangent ? LinOp<double>{t3_tangent_op, &tctx, sizeof(tctx)}
                            : LinOp<double>{t3_force_op, &kctx, sizeof(kctx)};
  return qs_newton(n2, K, t3_force_eval, &kctx, f_ext, bc_mask, bc_vals, u, tol, cg_tol, cg_max_iter, max_iter,
                   line_search, ls_max_steps, ls_min_alpha, ls_c, info, workspace, scope.get());
}

size_t phastb_t3_damage_linear_workspace_bytes(int n_nodes) { return phastb_q4_damage_linear_workspace_bytes(n_nodes); }

int phastb_t3_damage_linear_solve(const phastb_t3_mesh* mesh, const double* H, double gc_over_l0,
                                  const double* gc_over_l0_e, double gcl0, const double* gcl0_e, const double* rhs,
                                  const uint8_t* fixed, const double* fixed_vals, const double* x0, double rtol,
                                  int max_iter, int check_every, double* x_out, int* info, double* rinfo,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  if (!t3_valid_mesh(mesh) || !H || !rhs || !x_out || max_iter < 1 || check_every < 1 || !(rtol >= 0))
    return PHASTB_ERR_ARG;
  const int n = mesh->n_nodes;
  if (!workspace || workspace_bytes < phastb_t3_damage_linear_workspace_bytes(n)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  char* p = static_cast<char*>(workspace);
  PcgWs<double> w = pcg_ws<double>(p, n);
  p += pcg_ws_bytes<double>(n);
  const size_t vb = align_up(sizeof(double) * (size_t)n);
  double* bf = reinterpret_cast<double*>(p);
  double* minv = reinterpret_cast<double*>(p + vb);
  RedWs rw = red_ws(p + 2 * vb);
  int st;
  if ((st = red_ws_reset(rw, s))) return st;
  if ((st = phastb_t3_damage_prepare(mesh, H, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, w.z, minv, (void*)s))) return st;
  { note_launch(); lin_setup_kernel<<<grid_for(n), kThreads, 0, s>>>(n, rhs, fixed, fixed_vals, x0, bf, x_out, minv); }
  if ((st = last_launch_status())) return st;
  double bn = 0.0;
  if ((st = vec_norm2<double>(bf, n, &bn, p + 2 * vb, s))) return st;
  if (rinfo) rinfo[0] = bn;
  T3DamageMaskCtx ctx;
  std::memset(&ctx, 0, sizeof(ctx));
  ctx.mesh = *mesh;
  ctx.H = H;
  ctx.gco = gc_over_l0;
  ctx.gco_e = gc_over_l0_e;
  ctx.gcl0 = gcl0;
  ctx.gcl0_e = gcl0_e;
  ctx.mask = fixed;
  LinOp<double> A{t3_damage_mask_op, &ctx, sizeof(ctx)};
  PcgResult pr{};
  if (bn == 0.0) {
    pr.converged = 1;
  } else if ((st = pcg_run<double>(A, n, w, bf, minv, nullptr, x_out, rtol * bn, max_iter, check_every, PCG_FREEZE,
                                   0.0, &pr, s))) {
    return st;
  }
  if (info) {
    info[0] = pr.iterations;
    info[1] = pr.converged ? 0 : (pr.breakdown ? 2 : (pr.nonfinite ? 3 : 1));
  }
  if (rinfo) rinfo[1] = pr.rnorm;
  return cuda_status(cudaStreamSynchronize(s));
}

}  // extern "C"
