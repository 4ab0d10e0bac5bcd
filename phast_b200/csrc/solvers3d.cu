// 3D solver drivers over the periodic-voxel operators: constrained Jacobi-PCG
// mechanics (solid3d/linalg.py), box-KKT damage (solvers/box_kkt_h8.py) and the
// staggered-change measure (solid3d/staggered.py:1097-1124).
#include "engine.cuh"
#include "h8_kernels.cuh"
#include "h8_tile.cuh"

#include <cmath>

namespace phastb {

bool valid_vox(const phastb_voxel_grid* g);
bool valid_mat(const phastb_voxel_material* m);
size_t h8_scratch_bytes(const VoxGeom& v, int dtype);
template <typename T>
int h8_mech_apply_dot_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* x, const T* gq,
                        const T* d, const uint8_t* mask, T* y, void* scratch, const int* guard, cudaStream_t s);
const double* h8_apply_dot_slot(const VoxGeom& v, int word, void* scratch);
template <typename T>
int h8_mech_apply_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* x, const T* gq,
                    const T* d, const uint8_t* mask, T* y, void* scratch, const int* guard, cudaStream_t s);
template <typename T>
int h8_mech_diag_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* gq, const T* d, T* diag,
                   void* scratch, cudaStream_t s);
int h8_damage_launch(const VoxGeom& v, const VoxMat<double>& mm, const uint8_t* slot, int mode, const double* d,
                     const double* H, double scale, double* y, const uint8_t* mask, void* scratch,
                     const int* guard, cudaStream_t s);

int closure_add_launch(const VoxGeom& v, const VoxMat<double>& m, const uint8_t* slot, const double* x,
                       const double* gq, const uint8_t* pattern, const uint8_t* mask, double* y, void* sc,
                       cudaStream_t s);
int closure_diag_launch(const VoxGeom& v, const VoxMat<double>& m, const uint8_t* slot, const double* gq,
                        const uint8_t* pattern, double* diag, void* sc, cudaStream_t s);
int closure_reset(void* sc, const VoxGeom& v, cudaStream_t s);
size_t closure_scratch_bytes(const VoxGeom& v);

struct MechCtx {
  VoxGeom v;
  VoxMat<double> m;
  const uint8_t* slot;
  const double* gq;
  const double* d;
  const uint8_t* mask;
  void* scratch;
  // crack closure with a fixed sign pattern (closure != 0): the add-back joins the action
  const uint8_t* pattern;
  void* clsc;
  long long closure;  // 64-bit: no tail padding in the bytes that key a captured graph
};

static int mech_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const MechCtx* k = static_cast<const MechCtx*>(c);
  int st = h8_mech_apply_t<double>(k->v, k->m, k->slot, x, k->gq, k->d, k->mask, y, k->scratch, guard, s);
  if (st || !k->closure) return st;
  return closure_add_launch(k->v, k->m, k->slot, x, k->gq, k->pattern, k->mask, y, k->clsc, s);
}

static int mech_op_dot(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const MechCtx* k = static_cast<const MechCtx*>(c);
  return h8_mech_apply_dot_t<double>(k->v, k->m, k->slot, x, k->gq, k->d, k->mask, y, k->scratch, guard, s);
}

struct DamageCtx {
  VoxGeom v;
  VoxMat<double> m;
  const uint8_t* slot;
  const double* H;
  double scale;
  const uint8_t* mask;
  void* scratch;
};

static int damage_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const DamageCtx* k = static_cast<const DamageCtx*>(c);
  return h8_damage_launch(k->v, k->m, k->slot, 0, x, k->H, k->scale, y, k->mask, k->scratch, guard, s);
}

// the action plus x . y (mode 3 of h8_damage_launch)
static int damage_op_dot(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const DamageCtx* k = static_cast<const DamageCtx*>(c);
  return h8_damage_launch(k->v, k->m, k->slot, 3, x, k->H, k->scale, y, k->mask, k->scratch, guard, s);
}

// The damage action in FP32 (the inner solves of the mixed-precision box-KKT CG).
struct DamageCtx32 {
  VoxGeom v;
  VoxMat<float> m;
  const uint8_t* slot;
  const float* H;
  double scale;
  const uint8_t* mask;
  RedWs ws;
};

static int damage_op32(const void* c, const float* x, float* y, const int* guard, cudaStream_t s) {
  const DamageCtx32* k = static_cast<const DamageCtx32*>(c);
  return h8_damage_tile_launch<float>(k->v, k->m, k->slot, x, k->H, k->scale, k->mask, y, k->ws, guard, false, s);
}

static int damage_op_dot32(const void* c, const float* x, float* y, const int* guard, cudaStream_t s) {
  const DamageCtx32* k = static_cast<const DamageCtx32*>(c);
  return h8_damage_tile_launch<float>(k->v, k->m, k->slot, x, k->H, k->scale, k->mask, y, k->ws, guard, true, s);
}

// PHASTB_DAMAGE_MIXED=1: the box-KKT's Dirichlet CG runs in FP32 (FP64 dot
// products) under FP64 iterative refinement on the true FP64 residual, to the
// same FP64 threshold.
static bool damage_mixed_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PHASTB_DAMAGE_MIXED");
    return e && e[0] == '1';
  }();
  return on;
}

// xc = where(fixed, vals, 0); x0f = where(free, x0, 0); invd = 1/where(free, diag, 1)
__global__ void constrained_setup_kernel(int n, const uint8_t* __restrict__ fixed, const double* __restrict__ vals,
                                         const double* __restrict__ x0, double* __restrict__ xc,
                                         double* __restrict__ x0f, double* __restrict__ diag_inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool f = fixed[i];
    xc[i] = f ? vals[i] : 0.0;
    x0f[i] = f ? 0.0 : (x0 ? x0[i] : 0.0);
    diag_inv[i] = 1.0 / (f ? 1.0 : diag_inv[i]);
  }
}

// b_f = where(free, rhs - image, 0) with ||b_f||^2
__global__ void __launch_bounds__(kThreads) constrained_rhs_kernel(int n, const uint8_t* __restrict__ fixed,
                                                                   const double* __restrict__ rhs,
                                                                   const double* __restrict__ image,
                                                                   double* __restrict__ bf, RedWs ws) {
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = fixed[i] ? 0.0 : (rhs ? rhs[i] : 0.0) - image[i];
    bf[i] = v;
    acc[0] += v * v;
  }
  reduce_multi<1>(acc, ws);
}

__global__ void to_f32_kernel(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = float(a[i]);
}

__global__ void add_f32_kernel(int n, const float* __restrict__ dx, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += double(dx[i]);
}

__global__ void where_kernel(int n, const uint8_t* __restrict__ fixed, const double* __restrict__ a,
                             const double* __restrict__ b, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = fixed[i] ? b[i] : a[i];
}

// box-KKT helpers -----------------------------------------------------------

// fixed = la | ua | peq; known = where(fixed, (ua ? upper : lower), 0);
// x0f = where(free, initial, 0); invd = 1/where(free, diag, 1)
__global__ void kkt_setup_kernel(int n, const uint8_t* __restrict__ la, const uint8_t* __restrict__ ua,
                                 const double* __restrict__ lower, const double* __restrict__ upv, double upper,
                                 const double* __restrict__ initial, const double* __restrict__ diag,
                                 uint8_t* __restrict__ fixed, double* __restrict__ known, double* __restrict__ x0f,
                                 double* __restrict__ invd) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ub = upv ? upv[i] : upper;
    const bool peq = lower[i] == ub;
    const bool f = la[i] || ua[i] || peq;
    fixed[i] = f;
    known[i] = f ? (ua[i] ? ub : lower[i]) : 0.0;
    x0f[i] = f ? 0.0 : (initial ? initial[i] : 0.0);
    invd[i] = 1.0 / (f ? 1.0 : diag[i]);
  }
}

// grad = A cand - rhs; add/release sets; la/ua updated in place; counts OR'd.
__global__ void __launch_bounds__(kThreads) kkt_update_kernel(int n, const uint8_t* __restrict__ fixed,
                                                              const double* __restrict__ cand,
                                                              const double* __restrict__ Acand,
                                                              const double* __restrict__ rhs,
                                                              const double* __restrict__ lower,
                                                              const double* __restrict__ upv, double upper,
                                                              double kkt_tol, uint8_t* __restrict__ la,
                                                              uint8_t* __restrict__ ua, double* __restrict__ grad,
                                                              RedWs ws) {
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double gr = Acand[i] - rhs[i];
    grad[i] = gr;
    const bool fr = !fixed[i];
    const bool add_l = fr && (cand[i] < lower[i]);
    const bool add_u = fr && (cand[i] > (upv ? upv[i] : upper));
    const bool rel_l = la[i] && (gr < -kkt_tol);
    const bool rel_u = ua[i] && (gr > kkt_tol);
    if (add_l || add_u || rel_l || rel_u) acc[0] += 1.0;
    la[i] = (la[i] || add_l) && !rel_l;
    ua[i] = (ua[i] || add_u) && !rel_u;
  }
  reduce_multi<1>(acc, ws);
}

// KKT audit (box_kkt_h8._kkt_diagnostics): returns violation count and maxima.
__global__ void __launch_bounds__(kThreads) kkt_audit_kernel(int n, const double* __restrict__ sol,
                                                             const double* __restrict__ grad,
                                                             const double* __restrict__ lower,
                                                             const double* __restrict__ upv, double upper,
                                                             const uint8_t* __restrict__ la,
                                                             const uint8_t* __restrict__ ua, double tol, RedWs ws) {
  // acc: [violations count, max|free grad|, max|projected grad|, max|complementarity|]
  double cnt = 0, fs = 0, pg = 0, cm = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double s = sol[i], g = grad[i], lo = lower[i], up = upv ? upv[i] : upper;
    const bool peq = lo == up;
    const bool l = la[i], u = ua[i];
    const bool fixed = l || u || peq;
    if (s < lo || s > up) cnt += 1.0;
    if (l && g < -tol) cnt += 1.0;
    if (u && -g < -tol) cnt += 1.0;
    if (!fixed) {
      fs = fmax(fs, fabs(g));
      pg = fmax(pg, fabs(g));
    }
    if (l) {
      pg = fmax(pg, fabs(fmin(g, 0.0)));
      cm = fmax(cm, fabs(fmax(g, 0.0) * (s - lo)));
    }
    if (u) {
      pg = fmax(pg, fabs(fmax(g, 0.0)));
      cm = fmax(cm, fabs(fmax(-g, 0.0) * (up - s)));
    }
  }
  __shared__ double sh[32];
  double v = block_sum(cnt, sh);
  if (threadIdx.x == 0) ws.part[blockIdx.x] = v;
  double mx[3] = {fs, pg, cm};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v = block_max(mx[k], sh);
    if (threadIdx.x == 0) ws.part[(k + 1) * kMaxPartials + blockIdx.x] = v;
  }
  if (arrive_last(ws.counter)) {
    const double c = fold_sum(ws.part, gridDim.x, sh);
    if (threadIdx.x == 0) ws.out[0] = c;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double t = fold_max(ws.part + (k + 1) * kMaxPartials, gridDim.x, sh);
      if (threadIdx.x == 0) ws.out[k + 1] = t;
    }
    if (threadIdx.x == 0) *ws.counter = 0u;
  }
}

// staggered change parts: ||du||, ||u||, max|dE|, max|E|, max|dd| (staggered.py:1097-1124)
__global__ void __launch_bounds__(kThreads) change_kernel(int nu, const double* __restrict__ xn,
                                                          const double* __restrict__ xo, int nd,
                                                          const double* __restrict__ dn,
                                                          const double* __restrict__ dol, RedWs ws) {
  double du = 0, un = 0, dd = 0, dE = 0, Ei = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nu; i += gridDim.x * blockDim.x) {
    const double a = xn[i], b = a - xo[i];
    du += b * b;
    un += a * a;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x)
    dd = fmax(dd, fabs(dn[i] - dol[i]));
  if (blockIdx.x == 0 && threadIdx.x < 6) {
    dE = fabs(xn[nu + threadIdx.x] - xo[nu + threadIdx.x]);
    Ei = fabs(xn[nu + threadIdx.x]);
  }
  __shared__ double sh[32];
  double v = block_sum(du, sh);
  if (threadIdx.x == 0) ws.part[blockIdx.x] = v;
  v = block_sum(un, sh);
  if (threadIdx.x == 0) ws.part[kMaxPartials + blockIdx.x] = v;
  double mx[3] = {dE, Ei, dd};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v = block_max(mx[k], sh);
    if (threadIdx.x == 0) ws.part[(k + 2) * kMaxPartials + blockIdx.x] = v;
  }
  if (arrive_last(ws.counter)) {
    double t = fold_sum(ws.part, gridDim.x, sh);
    if (threadIdx.x == 0) ws.out[0] = sqrt(t);
    t = fold_sum(ws.part + kMaxPartials, gridDim.x, sh);
    if (threadIdx.x == 0) ws.out[1] = sqrt(t);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      t = fold_max(ws.part + (k + 2) * kMaxPartials, gridDim.x, sh);
      if (threadIdx.x == 0) ws.out[k + 2] = t;
    }
    if (threadIdx.x == 0) *ws.counter = 0u;
  }
}

}  // namespace phastb

using namespace phastb;

extern "C" {

size_t phastb_h8_mech_solve_workspace_bytes(const phastb_voxel_grid* g, int dtype) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  const int n = 3 * v.n_red + 6;
  return pcg_ws_bytes<double>(n) + 3 * align_up(sizeof(double) * (size_t)n) + h8_scratch_bytes(v, PHASTB_F64) +
         red_ws_bytes() + align_up(sizeof(double) * (size_t)n) + align_up(sizeof(double) * (size_t)v.n_red) +
         align_up(sizeof(double) * 8 * (size_t)v.n_elem);
}

// The constrained Jacobi PCG of phastb_h8_mech_solve; with closure != 0 the operator and its
// diagonal carry the crack-closure add-back of the sign pattern (copied into cl_ws, which
// holds closure_scratch_bytes + 8 E bytes).
static int mech_solve_impl(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                           const double* gq, const double* d, const uint8_t* pattern, int closure, void* cl_ws,
                           const uint8_t* fixed, const double* fixed_values, const double* x0, double rtol,
                           double atol, int maxiter, int check_every, double* x_out, int* info, double* rinfo,
                           void* workspace, void* stream) {
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  const VoxGeom v = make_vox_geom(*g);
  const VoxMat<double> mm = make_vox_mat<double>(*m);
  const int n = 3 * v.n_red + 6;
  char* p = static_cast<char*>(workspace);
  PcgWs<double> w = pcg_ws<double>(p, n);
  p += pcg_ws_bytes<double>(n);
  const size_t vb = align_up(sizeof(double) * (size_t)n);
  double* xc = reinterpret_cast<double*>(p);
  double* bf = reinterpret_cast<double*>(p + vb);
  double* invd = reinterpret_cast<double*>(p + 2 * vb);
  void* scratch = p + 3 * vb;
  void* redb = p + 3 * vb + h8_scratch_bytes(v, PHASTB_F64);
  RedWs rw = red_ws(redb);
  RedWs sw = red_ws(static_cast<char*>(scratch) + align_up(24 * sizeof(double) * (size_t)v.n_elem));
  const int G = grid_for(n);
  int st;
  if ((st = red_ws_reset(rw, s))) return st;
  if ((st = red_ws_reset(sw, s))) return st;
  // the captured PCG chunks read the iterate, d and g(d) from the workspace, so
  // repeated solves replay one graph however the caller allocates its tensors
  char* q = static_cast<char*>(redb) + red_ws_bytes();
  double* xw = reinterpret_cast<double*>(q);
  double* dw = reinterpret_cast<double*>(q + vb);
  double* gw = reinterpret_cast<double*>(q + vb + align_up(sizeof(double) * (size_t)v.n_red));
  if (d && (st = cuda_status(cudaMemcpyAsync(dw, d, sizeof(double) * v.n_red, cudaMemcpyDeviceToDevice, s))))
    return st;
  if (gq && (st = cuda_status(cudaMemcpyAsync(gw, gq, sizeof(double) * 8 * (size_t)v.n_elem,
                                               cudaMemcpyDeviceToDevice, s))))
    return st;
  d = d ? dw : nullptr;
  gq = gq ? gw : nullptr;
  const uint8_t* patw = nullptr;
  if (closure) {
    if ((st = closure_reset(cl_ws, v, s))) return st;
    if (pattern) {
      uint8_t* pw = static_cast<uint8_t*>(cl_ws) + closure_scratch_bytes(v);
      if ((st = cuda_status(cudaMemcpyAsync(pw, pattern, 8 * (size_t)v.n_elem, cudaMemcpyDeviceToDevice, s))))
        return st;
      patw = pw;
    }
  }
  // diagonal of A(g) into invd, then the constrained setup
  if ((st = h8_mech_diag_t<double>(v, mm, slot, gq, d, invd, scratch, s))) return st;
  if (closure && (st = closure_diag_launch(v, mm, slot, gq, patw, invd, cl_ws, s))) return st;
  { note_launch(); constrained_setup_kernel<<<G, kThreads, 0, s>>>(n, fixed, fixed_values, x0, xc, x_out, invd); }
  MechCtx full{v, mm, slot, gq, d, nullptr, scratch, patw, cl_ws, closure};
  if ((st = mech_op(&full, xc, w.Ap, nullptr, s))) return st;
  { note_launch(); constrained_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, nullptr, w.Ap, bf, rw); }
  if ((st = last_launch_status())) return st;
  double bn2;
  if ((st = red_ws_fetch(rw, &bn2, 1, s))) return st;
  const double bn = std::sqrt(bn2);
  if (rinfo) rinfo[0] = bn;
  if (!std::isfinite(bn)) return PHASTB_NONFINITE;
  if (bn == 0.0) {
    { note_launch(); where_kernel<<<G, kThreads, 0, s>>>(n, fixed, x_out, xc, x_out); }
    if (info) { info[0] = 0; info[1] = 1; }
    if (rinfo) rinfo[1] = 0.0;
    return last_launch_status();
  }
  const double thr = std::max(rtol * bn, atol);
  MechCtx free_ctx{v, mm, slot, gq, d, fixed, scratch, patw, cl_ws, closure};
  LinOp<double> A{mech_op, &free_ctx, sizeof(free_ctx), closure ? nullptr : mech_op_dot,
                  closure ? nullptr : h8_apply_dot_slot(v, 8, scratch)};
  PcgResult pr{};
  if ((st = cuda_status(cudaMemcpyAsync(xw, x_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)))) return st;
  if ((st = pcg_run<double>(A, n, w, bf, invd, nullptr, xw, thr, maxiter, check_every, PCG_FREEZE, 0.0, &pr, s)))
    return st;
  { note_launch(); where_kernel<<<G, kThreads, 0, s>>>(n, fixed, xw, xc, x_out); }
  if ((st = last_launch_status())) return st;
  if (info) { info[0] = pr.iterations; info[1] = pr.converged; }
  if (rinfo) rinfo[1] = pr.rnorm;
  if (pr.nonfinite) return PHASTB_NONFINITE;
  if (pr.breakdown) return PHASTB_BREAKDOWN;
  return pr.converged ? PHASTB_OK : PHASTB_NONCONVERGED;
}

int phastb_h8_mech_solve(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                         const double* gq, const double* d, const uint8_t* fixed, const double* fixed_values,
                         const double* x0, double rtol, double atol, int maxiter, int check_every, double* x_out,
                         int* info, double* rinfo, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !fixed || !fixed_values || !x_out || maxiter < 1 ||
      check_every < 1 || !(rtol >= 0) || !(atol >= 0) || (rtol == 0 && atol == 0))
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_mech_solve_workspace_bytes(g, PHASTB_F64))
    return PHASTB_ERR_WORKSPACE;
  return mech_solve_impl(g, m, slot, gq, d, nullptr, 0, nullptr, fixed, fixed_values, x0, rtol, atol, maxiter,
                         check_every, x_out, info, rinfo, workspace, stream);
}

size_t phastb_h8_mech_solve_closure_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  return phastb_h8_mech_solve_workspace_bytes(g, PHASTB_F64) + closure_scratch_bytes(v) +
         align_up(8 * (size_t)v.n_elem);
}

int phastb_h8_mech_solve_closure(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                 const double* gq, const uint8_t* pattern, const uint8_t* fixed,
                                 const double* fixed_values, const double* x0, double rtol, double atol,
                                 int maxiter, int check_every, double* x_out, int* info, double* rinfo,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !gq || !pattern || !fixed || !fixed_values || !x_out ||
      maxiter < 1 || check_every < 1 || !(rtol >= 0) || !(atol >= 0) || (rtol == 0 && atol == 0))
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_mech_solve_closure_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  void* cl_ws = static_cast<char*>(workspace) + phastb_h8_mech_solve_workspace_bytes(g, PHASTB_F64);
  return mech_solve_impl(g, m, slot, gq, nullptr, pattern, 1, cl_ws, fixed, fixed_values, x0, rtol, atol, maxiter,
                         check_every, x_out, info, rinfo, workspace, stream);
}

size_t phastb_h8_box_kkt_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  const int n = v.n_red;
  return pcg_ws_bytes<double>(n) + 6 * align_up(sizeof(double) * (size_t)n) + 4 * align_up((size_t)n) +
         h8_scratch_bytes(v, PHASTB_F64) + red_ws_bytes() + align_up(sizeof(double) * (size_t)n) +
         align_up(sizeof(double) * 8 * (size_t)v.n_elem) + red_ws_bytes() + align_up(sizeof(double) * (size_t)n) +
         // FP32 inner solves: CG workspace, right-hand side, correction, 1/diag, second direction, H, dot
         pcg_ws_bytes<float>(n) + 4 * align_up(sizeof(float) * (size_t)n) +
         align_up(sizeof(float) * 8 * (size_t)v.n_elem) + red_ws_bytes();
}

}  // extern "C"

namespace phastb {

// The primal active-set box solve behind phastb_h8_damage_box_kkt.  With rhs_in / diag_in
// NULL the system is the AT2 damage system of history H (its right-hand side and Jacobi
// diagonal formed here); otherwise the caller gives them and H holds the Gauss-point
// weights of the operator mm describes (the PF-CZM Newton tangent).  upper_v (NULL: the
// scalar upper) is the upper bound per node.  The workspace is
// phastb_h8_box_kkt_workspace_bytes.
int box_kkt_run(const VoxGeom& v, const VoxMat<double>& mm, const uint8_t* slot, const double* H, double scale,
                const double* rhs_in, const double* diag_in, const double* lower, const double* upper_v,
                double upper, const double* initial, double lin_tol, double kkt_tol, int max_lin, int max_active,
                bool allow_mixed, double* d_out, int* info, void* workspace, cudaStream_t s) {
  const int n = v.n_red;
  char* p = static_cast<char*>(workspace);
  PcgWs<double> w = pcg_ws<double>(p, n);
  p += pcg_ws_bytes<double>(n);
  const size_t vb = align_up(sizeof(double) * (size_t)n), ub = align_up((size_t)n);
  double* rhs = reinterpret_cast<double*>(p);
  double* diag = reinterpret_cast<double*>(p + vb);
  double* invd = reinterpret_cast<double*>(p + 2 * vb);
  double* known = reinterpret_cast<double*>(p + 3 * vb);
  double* bf = reinterpret_cast<double*>(p + 4 * vb);
  double* grad = reinterpret_cast<double*>(p + 5 * vb);
  uint8_t* la = reinterpret_cast<uint8_t*>(p + 6 * vb);
  uint8_t* ua = la + ub;
  uint8_t* fixed = la + 2 * ub;
  char* scratch = p + 6 * vb + 4 * ub;
  RedWs rw = red_ws(scratch + h8_scratch_bytes(v, PHASTB_F64));
  // the action's own reduction ticket (x . y of the fused CG) lives inside the scratch
  RedWs aw = red_ws(scratch + align_up(24 * sizeof(double) * (size_t)v.n_elem));
  // the iterate and the history live in the workspace, so the captured PCG
  // chunks see the same pointers on every call (one graph per workspace)
  char* q = scratch + h8_scratch_bytes(v, PHASTB_F64) + red_ws_bytes();
  double* xd = reinterpret_cast<double*>(q);
  double* Hw = H ? reinterpret_cast<double*>(q + vb) : nullptr;
  // the KKT audit reduces into its own workspace so one host read serves both checks
  RedWs kw = red_ws(q + vb + align_up(sizeof(double) * 8 * (size_t)v.n_elem));
  // second CG direction buffer of the persistent damage PCG
  double* p_alt = reinterpret_cast<double*>(q + vb + align_up(sizeof(double) * 8 * (size_t)v.n_elem) + red_ws_bytes());
  // FP32 buffers of the mixed-precision inner solves
  char* q32 = reinterpret_cast<char*>(p_alt) + vb;
  PcgWs<float> w32 = pcg_ws<float>(q32, n);
  q32 += pcg_ws_bytes<float>(n);
  const size_t fb = align_up(sizeof(float) * (size_t)n);
  float* r32 = reinterpret_cast<float*>(q32);
  float* dx32 = reinterpret_cast<float*>(q32 + fb);
  float* invd32 = reinterpret_cast<float*>(q32 + 2 * fb);
  float* palt32 = reinterpret_cast<float*>(q32 + 3 * fb);
  float* H32 = H ? reinterpret_cast<float*>(q32 + 4 * fb) : nullptr;
  RedWs dw32 = red_ws(q32 + 4 * fb + align_up(sizeof(float) * 8 * (size_t)v.n_elem));
  const bool mixed = allow_mixed && damage_mixed_enabled();
  const int G = grid_for(n);
  int st;
  if ((st = red_ws_reset(rw, s))) return st;
  if ((st = red_ws_reset(aw, s))) return st;
  if ((st = red_ws_reset(kw, s))) return st;
  if (mixed && (st = red_ws_reset(dw32, s))) return st;
  if (H && (st = cuda_status(cudaMemcpyAsync(Hw, H, sizeof(double) * 8 * (size_t)v.n_elem,
                                              cudaMemcpyDeviceToDevice, s))))
    return st;
  const VoxMat<float> m32 = vox_mat_cast<float>(mm);
  if (mixed && H) {
    const size_t ne = 8 * (size_t)v.n_elem;
    { note_launch(); to_f32_kernel<<<grid_for((long long)ne), kThreads, 0, s>>>(ne, Hw, H32); }
    if ((st = last_launch_status())) return st;
  }
  auto finish = [&](int code) -> int {
    const int e = cuda_status(cudaMemcpyAsync(d_out, xd, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return e ? e : code;
  };
  if (rhs_in) {
    if ((st = cuda_status(cudaMemcpyAsync(rhs, rhs_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)))) return st;
  } else {
    if ((st = h8_damage_launch(v, mm, slot, 1, nullptr, Hw, scale, rhs, nullptr, scratch, nullptr, s))) return st;
    if (!H && (st = cuda_status(cudaMemsetAsync(rhs, 0, sizeof(double) * n, s)))) return st;
  }
  if (diag_in) {
    if ((st = cuda_status(cudaMemcpyAsync(diag, diag_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, s))))
      return st;
  } else if ((st = h8_damage_launch(v, mm, slot, 2, nullptr, Hw, scale, diag, nullptr, scratch, nullptr, s))) {
    return st;
  }
  if ((st = cuda_status(cudaMemsetAsync(la, 0, 2 * ub, s)))) return st;
  DamageCtx full{v, mm, slot, Hw, scale, nullptr, scratch};
  int total = 0;
  const double* cinit = initial;
  for (int ai = 1; ai <= max_active; ++ai) {
    { note_launch(); kkt_setup_kernel<<<G, kThreads, 0, s>>>(n, la, ua, lower, upper_v, upper, cinit, diag, fixed, known, xd, invd); }
    // b_f = where(free, rhs - A known, 0)
    if ((st = damage_op(&full, known, w.Ap, nullptr, s))) return st;
    { note_launch(); constrained_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, rhs, w.Ap, bf, rw); }
    if ((st = last_launch_status())) return st;
    // Dirichlet PCG on the free set: tolerance relative to max(||r0||, 1)
    DamageCtx fctx{v, mm, slot, Hw, scale, fixed, scratch};
    LinOp<double> A{damage_op, &fctx, sizeof(fctx), damage_op_dot, h8_apply_dot_slot(v, 8, scratch)};
    PcgResult pr{};
    if (!mixed) {
      // all iterations in one persistent launch where the device allows it
      const PcgLoop loop = [&](int mi) {
        return h8_damage_pcg_launch<double>(v, mm, slot, Hw, scale, fixed, w, p_alt, xd, invd, mi, PCG_STRICT, s);
      };
      if ((st = pcg_run<double>(A, n, w, bf, invd, nullptr, xd, -lin_tol, max_lin, 10, PCG_STRICT, 0.0, &pr, s,
                                &loop)))
        return st;
    } else {
      // FP64 residual of the start iterate on the free set; the threshold is
      // lin_tol * max(||r0||, 1) as in the FP64 solve
      if ((st = damage_op(&fctx, xd, w.Ap, nullptr, s))) return st;
      { note_launch(); constrained_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, bf, w.Ap, w.r, rw); }
      { note_launch(); to_f32_kernel<<<G, kThreads, 0, s>>>((size_t)n, invd, invd32); }
      if ((st = last_launch_status())) return st;
      double rr0;
      if ((st = red_ws_fetch(rw, &rr0, 1, s))) return st;
      const double thr = lin_tol * std::max(std::sqrt(rr0), 1.0);
      DamageCtx32 c32{v, m32, slot, H32, scale, fixed, dw32};
      LinOp<float> A32{damage_op32, &c32, sizeof(c32), damage_op_dot32, dw32.out + kOutDot};
      const PcgLoop loop32 = [&](int mi) {
        return h8_damage_pcg_launch<float>(v, m32, slot, H32, scale, fixed, w32, palt32, dx32, invd32, mi,
                                           PCG_STRICT, s);
      };
      int inner = 0, conv = 0;
      for (int k = 0; k < 30 && inner < max_lin; ++k) {
        // correction equation in FP32; the start kernel checks the FP64 residual
        // norm (rw.out) against thr first and does nothing once it holds
        { note_launch(); to_f32_kernel<<<G, kThreads, 0, s>>>((size_t)n, w.r, r32); }
        if ((st = cuda_status(cudaMemsetAsync(dx32, 0, sizeof(float) * n, s)))) return st;
        PcgThreshold tin;
        tin.abs = 0.5 * thr;
        tin.rel = 1e-5;
        tin.outer_rr = rw.out;
        tin.outer_thr = thr;
        PcgResult pi{};
        if ((st = pcg_run_thr<float>(A32, n, w32, r32, invd32, nullptr, dx32, tin, max_lin - inner, 10, PCG_STRICT,
                                     &pi, s, &loop32)))
          return st;
        if (pi.outer_done) {
          conv = 1;
          break;
        }
        inner += pi.iterations;
        if (pi.nonfinite) pr.nonfinite = 1;
        if (pi.breakdown) pr.breakdown = 1;
        if (pr.nonfinite || pr.breakdown) break;
        { note_launch(); add_f32_kernel<<<G, kThreads, 0, s>>>(n, dx32, xd); }
        if ((st = damage_op(&fctx, xd, w.Ap, nullptr, s))) return st;
        { note_launch(); constrained_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, bf, w.Ap, w.r, rw); }
        if ((st = last_launch_status())) return st;
      }
      if (!conv && !pr.nonfinite && !pr.breakdown) {
        double rr;
        if ((st = red_ws_fetch(rw, &rr, 1, s))) return st;
        conv = std::sqrt(rr) <= thr;
      }
      pr.iterations = inner;
      pr.converged = conv;
    }
    // candidate = where(fixed, known, x)
    { note_launch(); where_kernel<<<G, kThreads, 0, s>>>(n, fixed, xd, known, xd); }
    total += pr.iterations;
    if (pr.nonfinite) return finish(PHASTB_NONFINITE);
    if (pr.breakdown) return finish(PHASTB_BREAKDOWN);
    // gradient, active-set change
    if ((st = damage_op(&full, xd, w.Ap, nullptr, s))) return st;
    { note_launch(); kkt_update_kernel<<<G, kThreads, 0, s>>>(n, fixed, xd, w.Ap, rhs, lower, upper_v, upper, kkt_tol, la, ua, grad, rw); }
    // the audit of the updated sets is only read when nothing changed, but running
    // it now lets one synchronisation fetch both results
    { note_launch(); kkt_audit_kernel<<<G, kThreads, 0, s>>>(n, xd, grad, lower, upper_v, upper, la, ua, kkt_tol, kw); }
    if ((st = last_launch_status())) return st;
    double changes, a[4];
    if ((st = cuda_status(cudaMemcpyAsync(&changes, rw.out, sizeof(double), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(a, kw.out, sizeof(a), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    if (info) { info[0] = total; info[1] = ai; info[2] = 0; }
    if (!pr.converged) return finish(PHASTB_NONCONVERGED);
    if (changes == 0.0) {
      const int ok = a[0] == 0.0 && a[1] <= kkt_tol && a[2] <= kkt_tol && a[3] <= kkt_tol;
      if (info) info[2] = ok;
      return finish(ok ? PHASTB_OK : PHASTB_NONCONVERGED);
    }
    // next set starts from this candidate (copy so the solve can overwrite the iterate)
    if ((st = cuda_status(cudaMemcpyAsync(grad, xd, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)))) return st;
    cinit = grad;
  }
  return finish(PHASTB_NONCONVERGED);
}

}  // namespace phastb

extern "C" {

int phastb_h8_damage_box_kkt(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                             const double* H, double scale, const double* lower, double upper,
                             const double* initial, double lin_tol, double kkt_tol, int max_lin, int max_active,
                             double* d_out, int* info, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !lower || !d_out || max_lin < 1 || max_active < 1 ||
      !(lin_tol > 0) || !(kkt_tol >= 0))
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_box_kkt_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  return box_kkt_run(make_vox_geom(*g), make_vox_mat<double>(*m), slot, H, scale, nullptr, nullptr, lower, nullptr,
                     upper, initial, lin_tol, kkt_tol, max_lin, max_active, true, d_out, info, workspace,
                     scope.get());
}

int phastb_h8_stagger_change(int n_u, const double* x_new, const double* x_old, int n_d, const double* d_new,
                             const double* d_old, double* out_host, void* workspace, size_t workspace_bytes,
                             void* stream) {
  if (!x_new || !x_old || !d_new || !d_old || !out_host || n_u < 0 || n_d < 0) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < red_ws_bytes()) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  RedWs rw = red_ws(workspace);
  int st = red_ws_reset(rw, s);
  if (st) return st;
  { note_launch(); change_kernel<<<grid_for(std::max(n_u, n_d)), kThreads, 0, s>>>(n_u, x_new, x_old, n_d, d_new, d_old, rw); }
  if ((st = last_launch_status())) return st;
  return red_ws_fetch(rw, out_host, 5, s);
}

}  // extern "C"
