// PF-CZM damage law of the periodic voxel cell (SolverConfig.damage_law = 'pfczm'):
// Wu's rational degradation g = (1 - kappa) A/(A + Q) + kappa, A = (1 - d)^p,
// Q = a1 d (1 + a2 d + a2 a3 d^2) with g' and g'' (physics/pfczm.py:79-125); the damage
// energy, its gradient and the Newton tangent of PeriodicVoxelPhaseFieldOperator
// (solid3d/operator.py:465-606); and the projected Newton damage solve of
// StaggeredSolver._damage_pfczm (solid3d/staggered.py:843-1096).
//
// Every element quantity is one thread per element: the eight corner values are
// interpolated to the Gauss points (interp_sf), the law is evaluated per Gauss point and
// the nodal contributions go to an element scratch that a node-centric gather sums in a
// fixed order (no atomics, the same bits on every run).  The tangent action reuses the
// tiled damage action (h8_dtile) with the tangent's coefficients (VoxMat::dform = 1) and
// the curvature weights in place of the history, so the box-QP of each Newton step runs
// on the persistent damage CG of the AT2 solve.
#include "h8_kernels.cuh"
#include "h8_tile.cuh"
#include "reduce.cuh"
#include <cmath>
#include <utility>

namespace phastb {

bool valid_vox(const phastb_voxel_grid* g);
bool valid_mat(const phastb_voxel_material* m);
int box_kkt_run(const VoxGeom& v, const VoxMat<double>& mm, const uint8_t* slot, const double* H, double scale,
                const double* rhs_in, const double* diag_in, const double* lower, const double* upper_v,
                double upper, const double* initial, double lin_tol, double kkt_tol, int max_lin, int max_active,
                bool allow_mixed, double* d_out, int* info, void* workspace, cudaStream_t s);

namespace {

constexpr double kPi = 3.14159265358979323846;  // PFCZM_C_ALPHA, pfczm.py:6
constexpr double kTangentFloor = 0.25;          // PFCZM_TANGENT_FLOOR, operator.py:125
constexpr double kArmijo = 1.0e-4;              // staggered.py:118
constexpr double kEnergyRtol = 1.0e-12;         // staggered.py:121
constexpr int kMaxHalvings = 30;                // staggered.py:124
constexpr int kMaxDoublings = 6;                // staggered.py:127
constexpr double kInnerFraction = 0.1;          // staggered.py:130
constexpr double kMinLinTol = 4.0 * 2.220446049250313080847e-16;  // staggered.py:97
constexpr int kEnergyWords = PHASTB_PFCZM_ENERGY_WORDS;

struct PfLaw {
  double a1[PHASTB_MAX_SLOTS];
  double a2, a3, p, eta;
};

PfLaw make_law(const phastb_pfczm_law& l, double kappa) {
  PfLaw r{};
  for (int s = 0; s < PHASTB_MAX_SLOTS; ++s) r.a1[s] = l.a1[s];
  r.a2 = l.a2;
  r.a3 = l.a3;
  r.p = l.p;
  r.eta = kappa;
  return r;
}

bool valid_law(const phastb_pfczm_law* l, const phastb_voxel_material* m) {
  if (!l || !(l->p >= 2.0) || !std::isfinite(l->a2) || !std::isfinite(l->a3)) return false;
  for (int s = 0; s < m->n_slots; ++s)
    if (!(l->a1[s] > 0.0) || !std::isfinite(l->a1[s])) return false;
  return true;
}

__device__ __forceinline__ void elem_ijk(const VoxGeom& g, int e, int& ie, int& je, int& ke) {
  ie = e % g.nx;
  const int r = e / g.nx;
  je = r % g.ny;
  ke = r / g.ny;
}

// g, g', g'' of the law at one Gauss point (pfczm_degradation_derivatives, pfczm.py:79-125).
// An integral p = 2 uses products as the reference does; g'' = 2 there.
template <int NDER>
__device__ __forceinline__ void pf_derivs(double d, double a1, const PfLaw& L, double& g, double& gp,
                                          double& gpp) {
  const double p = L.p;
  const double omd = fmax(1.0 - d, 0.0);
  double A, Ap, App;
  if (p == 2.0) {
    A = omd * omd;
    Ap = -2.0 * omd;
    App = 2.0;
  } else {
    A = pow(omd, p);
    Ap = -p * pow(omd, p - 1.0);
    App = p * (p - 1.0) * pow(omd, p - 2.0);
  }
  const double a2 = L.a2, a23 = L.a2 * L.a3;
  const double Q = a1 * d * (1.0 + a2 * d + a23 * d * d);
  const double S = fmax(A + Q, 1.0e-30);
  const double s = 1.0 - L.eta;
  g = s * (A / S) + L.eta;
  if (NDER >= 1) {
    const double Qp = a1 * (1.0 + 2.0 * a2 * d + 3.0 * a23 * d * d);
    const double N = Ap * Q - A * Qp;
    gp = s * (N / (S * S));
    if (NDER >= 2) {
      const double Qpp = a1 * (2.0 * a2 + 6.0 * a23 * d);
      const double Np = App * Q - A * Qpp;
      gpp = s * (Np / (S * S) - 2.0 * N * (Ap + Qp) / (S * S * S));
    }
  }
}

// Shape value N_L at Gauss point q of the unit 2-point rule (corner and point bits x, y, z).
__device__ __forceinline__ double shape_at(int L, int q) {
  return ((q & 1) == (L & 1) ? kC1 : kC2) * (((q >> 1) & 1) == ((L >> 1) & 1) ? kC1 : kC2) *
         ((q >> 2) == (L >> 2) ? kC1 : kC2);
}

enum PfMode { kPfG = 0, kPfEnergy = 1, kPfGrad = 2, kPfNewton = 3, kPfWeights = 4 };

// One thread per element.
//   kPfG:       gq[8e + q] = g(d_q)
//   kPfEnergy:  sums [history, local, gradient, by slot] into ws
//   kPfGrad:    sc[L E + e] = scale * element gradient at corner L
//   kPfNewton:  W (E,8) curvature weights, the scaled gradient in sc[0:8E) and the scaled
//               tangent diagonal in sc[8E:16E)
//   kPfWeights: W only
// kdl = diag of (2 ell/pi) L at one corner (the same at every corner).
template <int MODE>
__global__ void __launch_bounds__(kThreads) pf_elem_kernel(VoxGeom g, VoxMat<double> m, PfLaw law,
                                                           const uint8_t* __restrict__ slot,
                                                           const double* __restrict__ d,
                                                           const double* __restrict__ H, double scale, double kdl,
                                                           double* __restrict__ out_q, double* __restrict__ sc,
                                                           RedWs ws) {
  const double ihx = 1.0 / g.hx, ihy = 1.0 / g.hy, ihz = 1.0 / g.hz, w = g.w, ell = m.ell;
  const double c_loc = 1.0 / (kPi * ell), c_grad = ell / kPi;            // energy
  const double c_loc2 = 2.0 / (kPi * ell), c_grad2 = 2.0 * ell / kPi;    // gradient
  const size_t E = (size_t)g.n_elem;
  double acc[3 + PHASTB_MAX_SLOTS];
#pragma unroll
  for (int k = 0; k < 3 + PHASTB_MAX_SLOTS; ++k) acc[k] = 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    double dd[8], dq[8];
#pragma unroll
    for (int L = 0; L < 8; ++L) dd[L] = __ldg(d + nd[L]);
    interp_sf(dd, dq);
    const int s = slot[e];
    const double a1 = law.a1[s], Gc = m.Gc[s];
    double Hq[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) Hq[q] = H ? __ldg(H + 8 * (size_t)e + q) : 0.0;
    if (MODE == kPfG) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        double gv, u1, u2;
        pf_derivs<0>(dq[q], a1, law, gv, u1, u2);
        out_q[8 * (size_t)e + q] = gv;
      }
      continue;
    }
    if (MODE == kPfWeights || MODE == kPfNewton) {
      const double concave = c_loc2 * Gc, floor = kTangentFloor * concave;
      double wq[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        double gv, gp, gpp;
        pf_derivs<2>(dq[q], a1, law, gv, gp, gpp);
        wq[q] = H ? fmax(Hq[q] * gpp - concave, floor) : floor;
        out_q[8 * (size_t)e + q] = wq[q];
      }
      if (MODE == kPfNewton) {
#pragma unroll
        for (int L = 0; L < 8; ++L) {
          double a = 0.0;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const double n = shape_at(L, q);
            a += (wq[q] * w) * (n * n);
          }
          sc[(size_t)(8 + L) * E + e] = scale * (Gc * kdl + a);
        }
      }
      if (MODE == kPfWeights) continue;
    }
    double Dx[2][2], Dy[2][2], Dz[2][2];
    grad_sf(dd, ihx, ihy, ihz, Dx, Dy, Dz);
    if (MODE == kPfEnergy) {
      double hist = 0.0, loc = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (H) {
          double gv, u1, u2;
          pf_derivs<0>(dq[q], a1, law, gv, u1, u2);
          hist += (Hq[q] * w) * gv;
        }
        loc += 2.0 * dq[q] - dq[q] * dq[q];
      }
      double gl = 0.0;
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) gl += Dx[i][j] * Dx[i][j] + Dy[i][j] * Dy[i][j] + Dz[i][j] * Dz[i][j];
      // each face-difference gradient value holds at the two Gauss points along its own axis
      const double local = Gc * c_loc * (w * loc);
      const double grd = Gc * c_grad * (2.0 * w * gl);
      acc[0] += hist;
      acc[1] += local;
      acc[2] += grd;
#pragma unroll
      for (int k = 0; k < PHASTB_MAX_SLOTS; ++k) acc[3 + k] += (k == s) ? local + grd : 0.0;
      continue;
    }
    // gradient: sum_q w N_q [Gc 2/(pi ell) (1 - d_q) + H_q g'(d_q)] + Gc (2 ell/pi) L d_e
    double vq[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      double t = Gc * c_loc2 * (1.0 - dq[q]);
      if (H) {
        double gv, gp, u2;
        pf_derivs<1>(dq[q], a1, law, gv, gp, u2);
        t += Hq[q] * gp;
      }
      vq[q] = w * t;
    }
    double o[8], og[8];
    interp_sf_t(vq, o);
    const double k2 = 2.0 * w * Gc * c_grad2;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        Dx[i][j] *= k2;
        Dy[i][j] *= k2;
        Dz[i][j] *= k2;
      }
    grad_sf_t(Dx, Dy, Dz, ihx, ihy, ihz, og);
#pragma unroll
    for (int L = 0; L < 8; ++L) sc[(size_t)L * E + e] = scale * (o[L] + og[L]);
  }
  if (MODE == kPfEnergy) reduce_multi<3 + PHASTB_MAX_SLOTS>(acc, ws);
}

// y_f[n] = sum over the (up to) 8 elements of node n of sc[(f 8 + L) E + e], f < NF.
template <int NF>
__global__ void __launch_bounds__(kThreads) pf_gather_kernel(VoxGeom g, const double* __restrict__ sc,
                                                             double* __restrict__ y0, double* __restrict__ y1) {
  const size_t E = (size_t)g.n_elem;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n_red; n += gridDim.x * blockDim.x) {
    const int ir = n % g.rx;
    const int rem = n / g.rx;
    const int jr = rem % g.ry, kr = rem / g.ry;
    double acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0;
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      int ie = ir - (L & 1), je = jr - ((L >> 1) & 1), ke = kr - ((L >> 2) & 1);
      if (g.px) { if (ie < 0) ie += g.nx; } else if (ie < 0 || ie >= g.nx) continue;
      if (g.py) { if (je < 0) je += g.ny; } else if (je < 0 || je >= g.ny) continue;
      if (g.pz) { if (ke < 0) ke += g.nz; } else if (ke < 0 || ke >= g.nz) continue;
      const size_t e = (size_t)ie + (size_t)g.nx * ((size_t)je + (size_t)g.ny * ke);
#pragma unroll
      for (int f = 0; f < NF; ++f) acc[f] += __ldg(sc + (size_t)(f * 8 + L) * E + e);
    }
    y0[n] = acc[0];
    if (NF > 1) y1[n] = acc[NF - 1];
  }
}

// Jacobi diagonal of the tangent from the weights: sc[L E + e] = scale (Gc kdl + sum_q w W_q N_L(q)^2).
__global__ void __launch_bounds__(kThreads) pf_wdiag_kernel(VoxGeom g, VoxMat<double> m,
                                                            const uint8_t* __restrict__ slot,
                                                            const double* __restrict__ W, double scale, double kdl,
                                                            double* __restrict__ sc) {
  const size_t E = (size_t)g.n_elem;
  const double w = g.w;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    const double Gc = m.Gc[slot[e]];
    double wq[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) wq[q] = __ldg(W + 8 * (size_t)e + q);
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      double a = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double n = shape_at(L, q);
        a += (wq[q] * w) * (n * n);
      }
      sc[(size_t)L * E + e] = scale * (Gc * kdl + a);
    }
  }
}

// out[0] = sum grad^2, out[1] = max |projected grad| with the outward part removed at an
// active bound (d <= lower: grad clamped above by 0; d >= 1: clamped below by 0).
__global__ void __launch_bounds__(kThreads) pf_resid_kernel(int n, const double* __restrict__ grad,
                                                            const double* __restrict__ d,
                                                            const double* __restrict__ lower, RedWs ws) {
  double ss = 0.0, mx = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double gr = grad[i], di = d[i];
    double pg = di <= lower[i] ? fmin(gr, 0.0) : gr;
    if (di >= 1.0) pg = fmax(pg, 0.0);
    ss += gr * gr;
    // NaN propagates into the maximum (fmax would drop it)
    const double a = fabs(pg);
    mx = (a > mx || a != a) ? a : mx;
  }
  __shared__ double sh[32];
  const double bs = block_sum(ss, sh);
  const double bm = block_max(mx, sh);
  if (threadIdx.x == 0) {
    ws.part[blockIdx.x] = bs;
    ws.part[kMaxPartials + blockIdx.x] = bm;
  }
  if (arrive_last(ws.counter)) {
    const double t = fold_sum(ws.part, gridDim.x, sh);
    const double u = fold_max(ws.part + kMaxPartials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      ws.out[0] = t;
      ws.out[1] = u;
      *ws.counter = 0u;
    }
  }
}

// Bounds of the Newton box-QP: nodes on a bound with an outward gradient above tol are held.
__global__ void pf_bounds_kernel(int n, const double* __restrict__ d, const double* __restrict__ lower,
                                 const double* __restrict__ grad, double tol, double* __restrict__ lower_k,
                                 double* __restrict__ upper_k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double di = d[i], lo = lower[i], gr = grad[i];
    const bool hold_lower = di <= lo && gr > tol;
    const bool hold_upper = di >= 1.0 && gr < -tol;
    upper_k[i] = hold_lower ? lo : 1.0;
    lower_k[i] = hold_upper ? 1.0 : lo;
  }
}

__global__ void pf_sub_kernel(int n, double* __restrict__ a, const double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] -= b[i];
}

// out[0] = sum grad (target - d)
__global__ void __launch_bounds__(kThreads) pf_slope_kernel(int n, const double* __restrict__ grad,
                                                            const double* __restrict__ target,
                                                            const double* __restrict__ d, RedWs ws) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[0] += grad[i] * (target[i] - d[i]);
  reduce_multi<1>(v, ws);
}

// out = min(max(d + t (target - d), lower), 1); with cmp, ws.out[0] = entries where out != cmp.
__global__ void __launch_bounds__(kThreads) pf_trial_kernel(int n, const double* __restrict__ d,
                                                            const double* __restrict__ target, double t,
                                                            const double* __restrict__ lower,
                                                            double* __restrict__ out,
                                                            const double* __restrict__ cmp, RedWs ws) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double di = d[i];
    const double x = fmin(fmax(di + t * (target[i] - di), lower[i]), 1.0);
    out[i] = x;
    if (cmp && x != cmp[i]) v[0] += 1.0;
  }
  if (cmp) reduce_multi<1>(v, ws);
}

// diag of (2 ell/pi) L at one corner (the same at every corner by symmetry)
double tangent_kdl(const VoxGeom& v, double ell) {
  const double c[2] = {kC1, kC2};
  double acc = 0.0;
  for (int q = 0; q < 8; ++q) {
    const int qx = q & 1, qy = (q >> 1) & 1, qz = q >> 2;
    const double nx = c[qx != 0], ny = c[qy != 0], nz = c[qz != 0];
    const double gx = -ny * nz / v.hx, gy = -nx * nz / v.hy, gz = -nx * ny / v.hz;
    acc += v.w * (gx * gx + gy * gy + gz * gz);
  }
  return 2.0 * ell / kPi * acc;
}

// The tangent's VoxMat: the tiled damage action then computes Gc (2 ell/pi) L f plus the
// mass of the Gauss-point weights passed as its history (2 (1 - kappa) = 1).
VoxMat<double> tangent_mat(const VoxMat<double>& m) {
  VoxMat<double> t = m;
  t.dform = 1;
  t.kappa = 0.5;
  return t;
}

size_t elem_scratch_bytes(const VoxGeom& v) { return align_up(sizeof(double) * 16 * (size_t)v.n_elem); }

struct PfCtx {
  VoxGeom v;
  VoxMat<double> m;
  PfLaw law;
  const uint8_t* slot;
  double kdl;
  double* sc;  // 16 E doubles
  cudaStream_t s;
};

int pf_energy(const PfCtx& c, const double* d, const double* H, RedWs ws, double* out) {
  { note_launch(); pf_elem_kernel<kPfEnergy><<<grid_for(c.v.n_elem), kThreads, 0, c.s>>>(
        c.v, c.m, c.law, c.slot, d, H, 1.0, c.kdl, nullptr, nullptr, ws); }
  int st = last_launch_status();
  if (st) return st;
  double r[3 + PHASTB_MAX_SLOTS];
  if ((st = red_ws_fetch(ws, r, 3 + PHASTB_MAX_SLOTS, c.s))) return st;
  out[0] = r[1] + r[2] + r[0];
  for (int k = 0; k < 3 + PHASTB_MAX_SLOTS; ++k) out[1 + k] = r[k];
  return PHASTB_OK;
}

int pf_gradient(const PfCtx& c, const double* d, const double* H, double scale, double* grad) {
  { note_launch(); pf_elem_kernel<kPfGrad><<<grid_for(c.v.n_elem), kThreads, 0, c.s>>>(
        c.v, c.m, c.law, c.slot, d, H, scale, c.kdl, nullptr, c.sc, RedWs{}); }
  { note_launch(); pf_gather_kernel<1><<<grid_for(c.v.n_red), kThreads, 0, c.s>>>(c.v, c.sc, grad, nullptr); }
  return last_launch_status();
}

}  // namespace
}  // namespace phastb

using namespace phastb;

extern "C" {

int phastb_h8_pfczm_degradation(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                const phastb_pfczm_law* law, const uint8_t* slot, const double* d, double* gq,
                                void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !valid_law(law, m) || !slot || !d || !gq) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  { note_launch(); pf_elem_kernel<kPfG><<<grid_for(v.n_elem), kThreads, 0, s>>>(
        v, make_vox_mat<double>(*m), make_law(*law, m->kappa), slot, d, nullptr, 1.0, 0.0, gq, nullptr, RedWs{}); }
  return last_launch_status();
}

size_t phastb_h8_pfczm_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  return elem_scratch_bytes(make_vox_geom(*g)) + red_ws_bytes();
}

int phastb_h8_pfczm_energy(const phastb_voxel_grid* g, const phastb_voxel_material* m, const phastb_pfczm_law* law,
                           const uint8_t* slot, const double* d, const double* H, double* out_host, void* workspace,
                           size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !valid_law(law, m) || !slot || !d || !out_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_pfczm_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  char* p = static_cast<char*>(workspace);
  PfCtx c{v, make_vox_mat<double>(*m), make_law(*law, m->kappa), slot, 0.0, reinterpret_cast<double*>(p),
          (cudaStream_t)stream};
  RedWs ws = red_ws(p + elem_scratch_bytes(v));
  int st = red_ws_reset(ws, c.s);
  if (st) return st;
  double r[1 + 3 + PHASTB_MAX_SLOTS];
  if ((st = pf_energy(c, d, H, ws, r))) return st;
  // [0] total, [1] history, [2] local, [3] gradient, [4..] by slot
  for (int k = 0; k < kEnergyWords; ++k) out_host[k] = r[k];
  return PHASTB_OK;
}

int phastb_h8_pfczm_gradient(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                             const phastb_pfczm_law* law, const uint8_t* slot, const double* d, const double* H,
                             double scale, double* grad, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !valid_law(law, m) || !slot || !d || !grad) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_pfczm_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  PfCtx c{v, make_vox_mat<double>(*m), make_law(*law, m->kappa), slot, 0.0, static_cast<double*>(workspace),
          (cudaStream_t)stream};
  return pf_gradient(c, d, H, scale, grad);
}

int phastb_h8_pfczm_tangent_weights(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                    const phastb_pfczm_law* law, const uint8_t* slot, const double* d,
                                    const double* H, double* W, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !valid_law(law, m) || !slot || !d || !W) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  { note_launch(); pf_elem_kernel<kPfWeights><<<grid_for(v.n_elem), kThreads, 0, s>>>(
        v, make_vox_mat<double>(*m), make_law(*law, m->kappa), slot, d, H, 1.0, 0.0, W, nullptr, RedWs{}); }
  return last_launch_status();
}

int phastb_h8_pfczm_tangent_apply(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                  const double* W, const double* f, double scale, double* y, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !W || !f || !y) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_pfczm_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(static_cast<char*>(workspace) + elem_scratch_bytes(v));
  int st = red_ws_reset(ws, s);
  if (st) return st;
  return h8_damage_tile_launch<double>(v, tangent_mat(make_vox_mat<double>(*m)), slot, f, W, scale, nullptr, y, ws,
                                       nullptr, false, s);
}

int phastb_h8_pfczm_tangent_diagonal(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                     const uint8_t* slot, const double* W, double scale, double* diag,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !W || !diag) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_pfczm_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  double* sc = static_cast<double*>(workspace);
  { note_launch(); pf_wdiag_kernel<<<grid_for(v.n_elem), kThreads, 0, s>>>(
        v, make_vox_mat<double>(*m), slot, W, scale, tangent_kdl(v, m->ell), sc); }
  { note_launch(); pf_gather_kernel<1><<<grid_for(v.n_red), kThreads, 0, s>>>(v, sc, diag, nullptr); }
  return last_launch_status();
}

size_t phastb_h8_pfczm_solve_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  const size_t vb = align_up(sizeof(double) * (size_t)v.n_red);
  return phastb_h8_box_kkt_workspace_bytes(g) + elem_scratch_bytes(v) + align_up(sizeof(double) * 8 * (size_t)v.n_elem) +
         11 * vb + 3 * red_ws_bytes();
}

int phastb_h8_pfczm_damage_solve(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                 const phastb_pfczm_law* law, const uint8_t* slot, const double* H, double scale,
                                 const double* lower, const double* initial, double kkt_tol, double lin_tol,
                                 int max_lin, int max_active, int max_newton, double* d_out, int* info,
                                 double* rinfo, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !valid_law(law, m) || !slot || !lower || !initial || !d_out ||
      !(kkt_tol > 0) || !(lin_tol > 0) || max_lin < 1 || max_active < 1 || max_newton < 0 || !(scale > 0))
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_pfczm_solve_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  const VoxGeom v = make_vox_geom(*g);
  const int n = v.n_red;
  const VoxMat<double> mm = make_vox_mat<double>(*m);
  const VoxMat<double> mt = tangent_mat(mm);
  char* p = static_cast<char*>(workspace);
  void* kws = p;
  p += phastb_h8_box_kkt_workspace_bytes(g);
  PfCtx c{v, mm, make_law(*law, m->kappa), slot, tangent_kdl(v, m->ell), reinterpret_cast<double*>(p), s};
  p += elem_scratch_bytes(v);
  double* W = reinterpret_cast<double*>(p);
  p += align_up(sizeof(double) * 8 * (size_t)v.n_elem);
  const size_t vb = align_up(sizeof(double) * (size_t)n);
  double* vec[11];
  for (int k = 0; k < 11; ++k) vec[k] = reinterpret_cast<double*>(p + k * vb);
  p += 11 * vb;
  double *dc = vec[0], *target = vec[1], *bufA = vec[2], *bufB = vec[3], *grad = vec[4], *diag = vec[5];
  double *rhs = vec[6], *lower_k = vec[7], *upper_k = vec[8], *gtmp = vec[9];
  RedWs ew = red_ws(p), rw = red_ws(p + red_ws_bytes()), sw = red_ws(p + 2 * red_ws_bytes());
  int st;
  if ((st = red_ws_reset(ew, s)) || (st = red_ws_reset(rw, s)) || (st = red_ws_reset(sw, s))) return st;
  const int G = grid_for(n);
  const double tol = kkt_tol, inner = kInnerFraction * kkt_tol;
  int pcg = 0, sets = 0, iters = 0, reason = 0;
  double res = NAN, energy = NAN;
  auto report = [&](int code) -> int {
    if (info) {
      info[0] = pcg;
      info[1] = sets;
      info[2] = iters;
      info[3] = reason;
    }
    if (rinfo) {
      rinfo[0] = res;
      rinfo[1] = energy;
    }
    const int e = cuda_status(cudaMemcpyAsync(d_out, dc, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return e ? e : code;
  };
  auto energy_of = [&](const double* x, double* out) -> int {
    double r[1 + 3 + PHASTB_MAX_SLOTS];
    const int e = pf_energy(c, x, H, ew, r);
    *out = r[0];
    return e;
  };
  // projected gradient of the (scaled) gradient field gr at x: res_out = max norm, gg = sum gr^2
  auto residual_of = [&](const double* gr, const double* x, double* res_out, double* gg) -> int {
    { note_launch(); pf_resid_kernel<<<G, kThreads, 0, s>>>(n, gr, x, lower, rw); }
    int e = last_launch_status();
    if (e) return e;
    double r2[2];
    if ((e = red_ws_fetch(rw, r2, 2, s))) return e;
    if (gg) *gg = r2[0];
    *res_out = r2[1];
    return PHASTB_OK;
  };
  if ((st = cuda_status(cudaMemcpyAsync(dc, initial, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)))) return st;
  if ((st = energy_of(dc, &energy))) return st;
  if (!std::isfinite(energy)) {
    reason = 1;
    return report(PHASTB_NONFINITE);
  }
  for (int it = 0; it <= max_newton; ++it) {
    iters = it;
    // Newton system at dc: weights, scaled gradient and tangent diagonal
    { note_launch(); pf_elem_kernel<kPfNewton><<<grid_for(v.n_elem), kThreads, 0, s>>>(
          v, mm, c.law, slot, dc, H, scale, c.kdl, W, c.sc, RedWs{}); }
    { note_launch(); pf_gather_kernel<2><<<G, kThreads, 0, s>>>(v, c.sc, grad, diag); }
    if ((st = last_launch_status())) return st;
    double gg;
    if ((st = residual_of(grad, dc, &res, &gg))) return st;
    if (!std::isfinite(res) || !std::isfinite(gg)) {
      reason = 2;
      return report(PHASTB_NONFINITE);
    }
    if (res <= tol) return report(PHASTB_OK);
    if (it == max_newton) break;
    // box-QP min 1/2 (x - d).K (x - d) + grad.(x - d) over the held bounds: rhs = K d - grad
    { note_launch(); pf_bounds_kernel<<<G, kThreads, 0, s>>>(n, dc, lower, grad, tol, lower_k, upper_k); }
    if ((st = h8_damage_tile_launch<double>(v, mt, slot, dc, W, scale, nullptr, rhs, sw, nullptr, false, s))) return st;
    { note_launch(); pf_sub_kernel<<<G, kThreads, 0, s>>>(n, rhs, grad); }
    if ((st = last_launch_status())) return st;
    const double r0 = std::sqrt(gg);
    const double lt = std::max(std::min(lin_tol, 0.1 * inner / std::max(r0, 1.0)), kMinLinTol);
    int kinfo[3] = {0, 0, 0};
    st = box_kkt_run(v, mt, slot, W, scale, rhs, diag, lower_k, upper_k, 1.0, dc, lt, inner, max_lin, max_active,
                     false, target, kinfo, kws, s);
    pcg += kinfo[0];
    sets += kinfo[1];
    if (st) {
      reason = 3;
      return report(st);
    }
    // Armijo line search along dc -> target with step halving
    { note_launch(); pf_slope_kernel<<<G, kThreads, 0, s>>>(n, grad, target, dc, sw); }
    if ((st = last_launch_status())) return st;
    double slope;
    if ((st = red_ws_fetch(sw, &slope, 1, s))) return st;
    slope /= scale;
    double t = 1.0, te = NAN;
    const double* cur = target;
    bool accepted = false;
    for (int h = 0; h <= kMaxHalvings; ++h) {
      if (t == 1.0) {
        cur = target;
      } else {
        { note_launch(); pf_trial_kernel<<<G, kThreads, 0, s>>>(n, dc, target, t, lower, bufA, nullptr, RedWs{}); }
        if ((st = last_launch_status())) return st;
        cur = bufA;
      }
      if ((st = energy_of(cur, &te))) return st;
      if (std::isfinite(te) && te <= energy + kArmijo * t * slope + kEnergyRtol * std::fabs(energy)) {
        accepted = true;
        break;
      }
      t *= 0.5;
    }
    if (!accepted) {
      reason = 4;
      return report(PHASTB_NONCONVERGED);
    }
    if (t == 1.0) {
      // the full step may already solve the nonlinear KKT system; otherwise extrapolate
      // along the projected path while the energy keeps decreasing
      double tr;
      if ((st = pf_gradient(c, target, H, scale, gtmp))) return st;
      if ((st = residual_of(gtmp, target, &tr, nullptr))) return st;
      if (!(tr <= tol)) {
        double* spare = bufA;
        for (int k = 0; k < kMaxDoublings; ++k) {
          t *= 2.0;
          { note_launch(); pf_trial_kernel<<<G, kThreads, 0, s>>>(n, dc, target, t, lower, spare, cur, sw); }
          if ((st = last_launch_status())) return st;
          double differ;
          if ((st = red_ws_fetch(sw, &differ, 1, s))) return st;
          if (differ == 0.0) break;
          double fe;
          if ((st = energy_of(spare, &fe))) return st;
          if (!(std::isfinite(fe) && fe < te)) break;
          te = fe;
          double* prev = const_cast<double*>(cur);
          cur = spare;
          spare = (prev == target) ? bufB : prev;
        }
      }
    }
    // accept: the iterate becomes the buffer `cur` points at
    double* nd = const_cast<double*>(cur);
    for (int k = 0; k < 4; ++k) {
      if (vec[k] == nd) {
        std::swap(vec[0], vec[k]);
        break;
      }
    }
    dc = vec[0];
    target = vec[1];
    bufA = vec[2];
    bufB = vec[3];
    energy = te;
  }
  reason = 5;
  return report(PHASTB_NONCONVERGED);
}

}  // extern "C"
