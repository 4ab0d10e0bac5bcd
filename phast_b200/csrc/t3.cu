// Unstructured linear-triangle (T3) operators with a coloured element scatter.
//
// The elements are greedily coloured on the host so that no two elements of
// one colour share a node; each colour is one launch in which every element
// adds its three nodal contributions with plain read-modify-writes -- no
// atomics, and the per-node summation order (colour by colour) is fixed, so
// results are deterministic.  One Gauss point per element (centroid), the
// stress splits of q4_kernels.cuh, and the element-H AT2 damage system with
// the consistent T3 mass.  C ABI in include/phastb.h.
#include "engine.cuh"

#include <vector>
#include "q4_kernels.cuh"

#include <cstring>

namespace phastb {

namespace {

struct T3Dev {
  const int* elem;     // (E, 3)
  const int* order;    // (E,) element ids sorted by colour
  const double* grad;  // (E, 3, 2)
  const double* areas; // (E,)
};

inline T3Dev t3_dev(const phastb_t3_mesh& m) { return T3Dev{m.elem, m.order, m.grad, m.areas}; }

__device__ __forceinline__ void t3_strain(const T3Dev& t, int e, const double* __restrict__ u, double& exx,
                                          double& eyy, double& gxy, int* n, double (*gp)[2]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    n[a] = __ldg(t.elem + 3 * e + a);
    gp[a][0] = __ldg(t.grad + 6 * e + 2 * a);
    gp[a][1] = __ldg(t.grad + 6 * e + 2 * a + 1);
  }
  exx = eyy = gxy = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double ux = __ldg(u + 2 * n[a]), uy = __ldg(u + 2 * n[a] + 1);
    exx += gp[a][0] * ux;
    eyy += gp[a][1] * uy;
    gxy += gp[a][1] * ux + gp[a][0] * uy;
  }
}

// f_a += A (sigma . grad phi_a) for the elements order[k0 .. k1) of one colour.
__global__ void __launch_bounds__(kThreads) t3_force_colour(T3Dev t, Mat2<double> m, int split,
                                                            const double* __restrict__ u,
                                                            const double* __restrict__ d, double* f, int k0,
                                                            int k1, const int* guard) {
  if (guard && *guard == 0) return;
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  int n[3];
  double gp[3][2], exx, eyy, gxy;
  t3_strain(t, e, u, exx, eyy, gxy, n, gp);
  double sxx, syy, sxy;
  if (d) {
    const double de = (__ldg(d + n[0]) + __ldg(d + n[1]) + __ldg(d + n[2])) / 3.0;
    stress2(m, split, exx, eyy, gxy, degr(m, de), sxx, syy, sxy);
  } else {
    stress2(m, PHASTB_SPLIT_LINEAR, exx, eyy, gxy, 1.0, sxx, syy, sxy);
  }
  const double A = __ldg(t.areas + e);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    f[2 * n[a]] += A * (sxx * gp[a][0] + sxy * gp[a][1]);
    f[2 * n[a] + 1] += A * (sxy * gp[a][0] + syy * gp[a][1]);
  }
}

// Consistent tangent: f_a += A (dsigma(eps(u); eps(du)) . grad phi_a) for the elements of one
// colour, the directional derivative of the split stress at the iterate u (dstress2), at the
// element-mean degradation of the force kernel.  The autograd JVP of internal_force that
// QuasiStaticSolver takes as its CG operator (mechanics_solver.py:1705-1733), on T3.
__global__ void __launch_bounds__(kThreads) t3_tangent_colour(T3Dev t, Mat2<double> m, int split,
                                                              const double* __restrict__ u,
                                                              const double* __restrict__ du,
                                                              const double* __restrict__ d, double* f, int k0,
                                                              int k1, const int* guard) {
  if (guard && *guard == 0) return;
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  int n[3];
  double gp[3][2], exx, eyy, gxy;
  t3_strain(t, e, u, exx, eyy, gxy, n, gp);
  double vxx = 0.0, vyy = 0.0, vxy = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double vx = du[2 * n[a]], vy = du[2 * n[a] + 1];
    vxx += gp[a][0] * vx;
    vyy += gp[a][1] * vy;
    vxy += gp[a][1] * vx + gp[a][0] * vy;
  }
  const double g = d ? degr(m, (__ldg(d + n[0]) + __ldg(d + n[1]) + __ldg(d + n[2])) / 3.0) : 1.0;
  double sxx, syy, sxy;
  dstress2(m, split, exx, eyy, gxy, vxx, vyy, vxy, g, sxx, syy, sxy);
  const double A = __ldg(t.areas + e);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    f[2 * n[a]] += A * (sxx * gp[a][0] + sxy * gp[a][1]);
    f[2 * n[a] + 1] += A * (sxy * gp[a][0] + syy * gp[a][1]);
  }
}

__global__ void __launch_bounds__(kThreads) t3_psi_kernel(T3Dev t, Mat2<double> m, const double* __restrict__ u,
                                                          const double* __restrict__ Hin, double* __restrict__ Hout,
                                                          double* __restrict__ psi, int ne) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int n[3];
  double gp[3][2], exx, eyy, gxy;
  t3_strain(t, e, u, exx, eyy, gxy, n, gp);
  const double p = psi2(m, m.psplit, exx, eyy, gxy);
  if (psi) psi[e] = p;
  if (Hout) {
    const double h = Hin ? Hin[e] : 0.0;
    Hout[e] = p > h ? p : h;
  }
}

// y_a += gcl0_e A (grad phi_a . grad d) + rc_e (d_a + d_sum),  rc_e = (2 H_e + gco_e) A / 12
__global__ void __launch_bounds__(kThreads) t3_damage_colour(T3Dev t, const double* __restrict__ d,
                                                             const double* __restrict__ H, double gco,
                                                             const double* __restrict__ gco_e, double gcl0,
                                                             const double* __restrict__ gcl0_e, double* y, int k0,
                                                             int k1, const int* guard) {
  if (guard && *guard == 0) return;
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  int n[3];
  double gp[3][2], dd[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    n[a] = __ldg(t.elem + 3 * e + a);
    gp[a][0] = __ldg(t.grad + 6 * e + 2 * a);
    gp[a][1] = __ldg(t.grad + 6 * e + 2 * a + 1);
    dd[a] = __ldg(d + n[a]);
  }
  const double A = __ldg(t.areas + e);
  const double gx = gp[0][0] * dd[0] + gp[1][0] * dd[1] + gp[2][0] * dd[2];
  const double gy = gp[0][1] * dd[0] + gp[1][1] * dd[1] + gp[2][1] * dd[2];
  const double rc = (2.0 * (H ? __ldg(H + e) : 0.0) + (gco_e ? __ldg(gco_e + e) : gco)) * A / 12.0;
  const double kl = gcl0_e ? __ldg(gcl0_e + e) : gcl0;
  const double ds = dd[0] + dd[1] + dd[2];
#pragma unroll
  for (int a = 0; a < 3; ++a) y[n[a]] += kl * (A * (gp[a][0] * gx + gp[a][1] * gy)) + rc * (dd[a] + ds);
}

// b_a += (2 H_e - src_e) A / 3;  diag_a += gcl0_e A |grad phi_a|^2 + 2 rc_e  (src: the AT1 source
// 3 Gc / (8 l0), zero for AT2; damage_solver.py:2060-2080)
__global__ void __launch_bounds__(kThreads) t3_prepare_colour(T3Dev t, const double* __restrict__ H, double gco,
                                                              const double* __restrict__ gco_e, double gcl0,
                                                              const double* __restrict__ gcl0_e, double src,
                                                              const double* __restrict__ src_e, double* b,
                                                              double* diag, int k0, int k1) {
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  const double A = __ldg(t.areas + e);
  const double He = H ? __ldg(H + e) : 0.0;
  const double rc = (2.0 * He + (gco_e ? __ldg(gco_e + e) : gco)) * A / 12.0;
  const double kl = gcl0_e ? __ldg(gcl0_e + e) : gcl0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int n = __ldg(t.elem + 3 * e + a);
    const double gx = __ldg(t.grad + 6 * e + 2 * a), gy = __ldg(t.grad + 6 * e + 2 * a + 1);
    b[n] += (2.0 * He - (src_e ? __ldg(src_e + e) : src)) * A / 3.0;
    diag[n] += kl * (A * (gx * gx + gy * gy)) + 2.0 * rc;
  }
}

// Nodal history (PhaseFieldX convention, damage_solver.py:1840-1912): the reaction mass is
// int 2 H N_a N_b with H interpolated from the nodes, i.e. with the triple products
// int N_i N_j N_k = A/10, A/30, A/60 (all, two, no indices equal):
//   y_a += kl A grad phi_a . grad d + A/30 [(2 H_a + S_H) d_a + (H_a + S_H) S_d + H.d]
//          + gco A/12 (d_a + S_d),   S_H, S_d, H.d the element sums.
__global__ void __launch_bounds__(kThreads) t3_damage_nodal_colour(T3Dev t, const double* __restrict__ d,
                                                                   const double* __restrict__ Hn, double gco,
                                                                   const double* __restrict__ gco_e, double gcl0,
                                                                   const double* __restrict__ gcl0_e, double* y,
                                                                   int k0, int k1, const int* guard) {
  if (guard && *guard == 0) return;
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  int n[3];
  double gp[3][2], dd[3], hh[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    n[a] = __ldg(t.elem + 3 * e + a);
    gp[a][0] = __ldg(t.grad + 6 * e + 2 * a);
    gp[a][1] = __ldg(t.grad + 6 * e + 2 * a + 1);
    dd[a] = __ldg(d + n[a]);
    hh[a] = Hn ? __ldg(Hn + n[a]) : 0.0;
  }
  const double A = __ldg(t.areas + e);
  const double gx = gp[0][0] * dd[0] + gp[1][0] * dd[1] + gp[2][0] * dd[2];
  const double gy = gp[0][1] * dd[0] + gp[1][1] * dd[1] + gp[2][1] * dd[2];
  const double kl = gcl0_e ? __ldg(gcl0_e + e) : gcl0;
  const double rg = (gco_e ? __ldg(gco_e + e) : gco) * A / 12.0;
  const double sh = hh[0] + hh[1] + hh[2], sd = dd[0] + dd[1] + dd[2];
  const double hd = hh[0] * dd[0] + hh[1] * dd[1] + hh[2] * dd[2];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double mh = A / 30.0 * ((2.0 * hh[a] + sh) * dd[a] + (hh[a] + sh) * sd + hd);
    y[n[a]] += kl * (A * (gp[a][0] * gx + gp[a][1] * gy)) + (mh + rg * (dd[a] + sd));
  }
}

// Nodal history: b_a += A/6 (H_a + S_H);  diag_a += kl A |grad phi_a|^2 + (2 H_a + S_H) A/15 + gco A/6
// (_prepare_cg_nodal, damage_solver.py:2303-2348)
__global__ void __launch_bounds__(kThreads) t3_prepare_nodal_colour(T3Dev t, const double* __restrict__ Hn,
                                                                    double gco, const double* __restrict__ gco_e,
                                                                    double gcl0, const double* __restrict__ gcl0_e,
                                                                    double* b, double* diag, int k0, int k1) {
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  const double A = __ldg(t.areas + e);
  const double kl = gcl0_e ? __ldg(gcl0_e + e) : gcl0;
  const double go = gco_e ? __ldg(gco_e + e) : gco;
  int n[3];
  double hh[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    n[a] = __ldg(t.elem + 3 * e + a);
    hh[a] = Hn ? __ldg(Hn + n[a]) : 0.0;
  }
  const double sh = hh[0] + hh[1] + hh[2];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double gx = __ldg(t.grad + 6 * e + 2 * a), gy = __ldg(t.grad + 6 * e + 2 * a + 1);
    b[n[a]] += A / 6.0 * (hh[a] + sh);
    diag[n[a]] += kl * (A * (gx * gx + gy * gy)) + ((2.0 * hh[a] + sh) * A / 15.0 + go * A / 6.0);
  }
}

__global__ void t3_invert_kernel(int n, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = 1.0 / (x[i] + 1e-30);
}

__global__ void t3_zero_kernel(int n, double* __restrict__ y, const int* guard) {
  if (guard && *guard == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = 0.0;
}

// y[i] = 0 on the rows a mask holds fixed (Dirichlet-eliminated operators of the Krylov engines)
__global__ void t3_mask_rows_kernel(int n, const uint8_t* __restrict__ mask, double* __restrict__ y,
                                    const int* guard) {
  if (guard && *guard == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (mask[i]) y[i] = 0.0;
}

// f_a += w_e B_a^T sigma0(u_e): the transpose of u -> psi_e (isotropic split, full energy
// 0.5 eps : C : eps at the centroid), weighted per element.
__global__ void __launch_bounds__(kThreads) t3_psi_grad_t_colour(T3Dev t, Mat2<double> m,
                                                                 const double* __restrict__ u,
                                                                 const double* __restrict__ w, double* f, int k0,
                                                                 int k1) {
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  int n[3];
  double gp[3][2], exx, eyy, gxy;
  t3_strain(t, e, u, exx, eyy, gxy, n, gp);
  double sxx, syy, sxy;
  stress2(m, PHASTB_SPLIT_LINEAR, exx, eyy, gxy, 1.0, sxx, syy, sxy);
  const double we = __ldg(w + e);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    f[2 * n[a]] += we * (sxx * gp[a][0] + sxy * gp[a][1]);
    f[2 * n[a] + 1] += we * (sxy * gp[a][0] + syy * gp[a][1]);
  }
}

// out_a += A_e g'(d_e) / 3 eps(z_e) . sigma0(u_e): the derivative of z . f_int(u, d) with
// respect to the nodal damage, d_e the element mean, g(d) = (1-d)^2 (1-eta) + eta.
__global__ void __launch_bounds__(kThreads) t3_force_dd_t_colour(T3Dev t, Mat2<double> m,
                                                                 const double* __restrict__ u,
                                                                 const double* __restrict__ z,
                                                                 const double* __restrict__ d, double* out, int k0,
                                                                 int k1) {
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  const int e = __ldg(t.order + k);
  int n[3];
  double gp[3][2], exx, eyy, gxy;
  t3_strain(t, e, u, exx, eyy, gxy, n, gp);
  double zxx = 0, zyy = 0, zxy = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double zx = __ldg(z + 2 * n[a]), zy = __ldg(z + 2 * n[a] + 1);
    zxx += gp[a][0] * zx;
    zyy += gp[a][1] * zy;
    zxy += gp[a][1] * zx + gp[a][0] * zy;
  }
  double sxx, syy, sxy;
  stress2(m, PHASTB_SPLIT_LINEAR, exx, eyy, gxy, 1.0, sxx, syy, sxy);
  const double de = (__ldg(d + n[0]) + __ldg(d + n[1]) + __ldg(d + n[2])) / 3.0;
  const double dg = -2.0 * (1.0 - de) * (1.0 - m.eta);
  const double v = __ldg(t.areas + e) * dg * (zxx * sxx + zyy * syy + zxy * sxy) / 3.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) out[n[a]] += v;
}

// Per-element adjoint quadratic forms of the AT2 system and the Gc-field / history gradients:
//   lkd_e = A (grad lam . grad d),  lmd_e = A/12 (sum lam sum d + lam . d),
//   dJ/dGc_e = -(l0 lkd_e + lmd_e / l0),  dJ/dH_e = 2 A sum_a lam_a (1/3 - (d_a + sum d) / 12)
// (_adjoint_quadratic_forms_perelem and the history pullback, damage_solver.py:284-336, 1017-1027).
__global__ void __launch_bounds__(kThreads) t3_damage_adjoint_kernel(T3Dev t, const double* __restrict__ lam,
                                                                     const double* __restrict__ d, double l0,
                                                                     double* __restrict__ g_gc,
                                                                     double* __restrict__ g_h,
                                                                     double* __restrict__ lkd,
                                                                     double* __restrict__ lmd, int ne) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double l[3], dd[3], glx = 0, gly = 0, gdx = 0, gdy = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int n = __ldg(t.elem + 3 * e + a);
    const double gx = __ldg(t.grad + 6 * e + 2 * a), gy = __ldg(t.grad + 6 * e + 2 * a + 1);
    l[a] = __ldg(lam + n);
    dd[a] = __ldg(d + n);
    glx += gx * l[a];
    gly += gy * l[a];
    gdx += gx * dd[a];
    gdy += gy * dd[a];
  }
  const double A = __ldg(t.areas + e);
  const double ls = l[0] + l[1] + l[2], ds = dd[0] + dd[1] + dd[2];
  const double kd = A * (glx * gdx + gly * gdy);
  const double md = A / 12.0 * (ls * ds + l[0] * dd[0] + l[1] * dd[1] + l[2] * dd[2]);
  if (g_gc) g_gc[e] = -(l0 * kd + md / l0);
  if (g_h) {
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) acc += l[a] * (1.0 / 3.0 - (dd[a] + ds) / 12.0);
    g_h[e] = 2.0 * A * acc;
  }
  if (lkd) lkd[e] = kd;
  if (lmd) lmd[e] = md;
}

}  // namespace

bool t3_valid_mesh(const phastb_t3_mesh* m) {
  if (!m || m->n_nodes < 1 || m->n_elems < 1 || m->n_colors < 1 || !m->elem || !m->order || !m->color_off ||
      !m->grad || !m->areas)
    return false;
  if (m->color_off[0] != 0 || m->color_off[m->n_colors] != m->n_elems) return false;
  for (int c = 0; c < m->n_colors; ++c)
    if (m->color_off[c + 1] < m->color_off[c]) return false;
  return true;
}

// Host check of a colouring (host arrays): node ids in range, `order` a permutation of the
// elements, colour offsets non-decreasing from 0 to n_elems, and no node touched twice by
// the elements of one colour (the condition of the atomic-free scatter).
int t3_check_mesh_host(int n_nodes, int n_elems, const int* elem, const int* order, int n_colors,
                       const int* color_off) {
  if (n_nodes < 1 || n_elems < 1 || n_colors < 1 || !elem || !order || !color_off) return PHASTB_ERR_ARG;
  if (color_off[0] != 0 || color_off[n_colors] != n_elems) return PHASTB_ERR_ARG;
  for (int c = 0; c < n_colors; ++c)
    if (color_off[c + 1] < color_off[c]) return PHASTB_ERR_ARG;
  for (long long i = 0; i < 3LL * n_elems; ++i)
    if (elem[i] < 0 || elem[i] >= n_nodes) return PHASTB_ERR_ARG;
  std::vector<int> seen_elem(n_elems, 0), last(n_nodes, -1);
  for (int i = 0; i < n_elems; ++i) {
    const int e = order[i];
    if (e < 0 || e >= n_elems || seen_elem[e]) return PHASTB_ERR_ARG;
    seen_elem[e] = 1;
  }
  for (int c = 0; c < n_colors; ++c) {
    for (int i = color_off[c]; i < color_off[c + 1]; ++i) {
      const int e = order[i];
      for (int k = 0; k < 3; ++k) {
        const int v = elem[3 * (size_t)e + k];
        if (last[v] == c) return PHASTB_ERR_ARG;  // two elements of colour c share node v
        last[v] = c;
      }
    }
  }
  return PHASTB_OK;
}

// y = A(H, Gc) d of the AT2 system; rows that ``mask`` holds fixed give 0.
int t3_damage_apply_launch(const phastb_t3_mesh& mesh, const double* d, const double* H, double gco,
                           const double* gco_e, double gcl0, const double* gcl0_e, double* y, const int* guard,
                           cudaStream_t s, const uint8_t* mask) {
  int st = cuda_status(cudaMemsetAsync(y, 0, sizeof(double) * (size_t)mesh.n_nodes, s));
  if (st) return st;
  const T3Dev t = t3_dev(mesh);
  for (int c = 0; c < mesh.n_colors; ++c) {
    const int k0 = mesh.color_off[c], k1 = mesh.color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_damage_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, d, H, gco, gco_e, gcl0, gcl0_e, y, k0, k1, guard); }
  }
  if (mask) { note_launch(); t3_mask_rows_kernel<<<grid_for(mesh.n_nodes), kThreads, 0, s>>>(mesh.n_nodes, mask, y, guard); }
  return last_launch_status();
}

// y = A d of a damage model (element or nodal history, AT2 or AT1 coefficients); masked rows 0.
int t3_damage_model_launch(const phastb_t3_mesh& mesh, const phastb_t3_damage_model& md, const double* d,
                           const double* H, double* y, const int* guard, cudaStream_t s, const uint8_t* mask) {
  if (!md.nodal_h)
    return t3_damage_apply_launch(mesh, d, H, md.gc_over_l0, md.gc_over_l0_e, md.gcl0, md.gcl0_e, y, guard, s,
                                  mask);
  int st = cuda_status(cudaMemsetAsync(y, 0, sizeof(double) * (size_t)mesh.n_nodes, s));
  if (st) return st;
  const T3Dev t = t3_dev(mesh);
  for (int c = 0; c < mesh.n_colors; ++c) {
    const int k0 = mesh.color_off[c], k1 = mesh.color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_damage_nodal_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, d, H, md.gc_over_l0, md.gc_over_l0_e, md.gcl0, md.gcl0_e, y, k0, k1, guard); }
  }
  if (mask) { note_launch(); t3_mask_rows_kernel<<<grid_for(mesh.n_nodes), kThreads, 0, s>>>(mesh.n_nodes, mask, y, guard); }
  return last_launch_status();
}

// f = f_int(u, d) (d NULL: undegraded linear); rows that ``mask`` holds fixed (2 per node) give 0.
int t3_force_launch(const phastb_t3_mesh& mesh, const phastb_q4_material& m, const double* u, const double* d,
                    double* f, const uint8_t* mask, const int* guard, cudaStream_t s) {
  const int n2 = 2 * mesh.n_nodes;
  { note_launch(); t3_zero_kernel<<<grid_for(n2), kThreads, 0, s>>>(n2, f, guard); }
  const T3Dev t = t3_dev(mesh);
  const Mat2<double> mm = make_mat2<double>(m);
  for (int c = 0; c < mesh.n_colors; ++c) {
    const int k0 = mesh.color_off[c], k1 = mesh.color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_force_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, mm, m.stress_split, u, d, f, k0, k1, guard); }
  }
  if (mask) { note_launch(); t3_mask_rows_kernel<<<grid_for(n2), kThreads, 0, s>>>(n2, mask, f, guard); }
  return last_launch_status();
}

int t3_tangent_launch(const phastb_t3_mesh& mesh, const phastb_q4_material& m, const double* u, const double* du,
                      const double* d, double* f, const uint8_t* mask, const int* guard, cudaStream_t s) {
  const int n2 = 2 * mesh.n_nodes;
  { note_launch(); t3_zero_kernel<<<grid_for(n2), kThreads, 0, s>>>(n2, f, guard); }
  const T3Dev t = t3_dev(mesh);
  const Mat2<double> mm = make_mat2<double>(m);
  for (int c = 0; c < mesh.n_colors; ++c) {
    const int k0 = mesh.color_off[c], k1 = mesh.color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_tangent_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, mm, m.stress_split, u, du, d, f, k0, k1, guard); }
  }
  if (mask) { note_launch(); t3_mask_rows_kernel<<<grid_for(n2), kThreads, 0, s>>>(n2, mask, f, guard); }
  return last_launch_status();
}

namespace {

// Damage operator context for the Krylov engines.  The mesh is held by value;
// color_off points into caller memory that must outlive the solve.
struct T3DamageCtx {
  phastb_t3_mesh mesh;
  const double* H;
  double gco;
  const double* gco_e;
  double gcl0;
  const double* gcl0_e;
};

int t3_damage_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const T3DamageCtx* k = static_cast<const T3DamageCtx*>(c);
  return t3_damage_apply_launch(k->mesh, x, k->H, k->gco, k->gco_e, k->gcl0, k->gcl0_e, y, guard, s, nullptr);
}

// A damage model's operator for the Krylov engines (hashed as bytes: zeroed before filling).
struct T3ModelCtx {
  phastb_t3_mesh mesh;
  phastb_t3_damage_model model;
  const double* H;
};

int t3_model_op(const void* c, const double* x, double* y, const int* guard, cudaStream_t s) {
  const T3ModelCtx* k = static_cast<const T3ModelCtx*>(c);
  return t3_damage_model_launch(k->mesh, k->model, x, k->H, y, guard, s, nullptr);
}

bool valid_model(const phastb_t3_damage_model* m) {
  return m && (m->nodal_h == 0 || m->nodal_h == 1) && !(m->nodal_h && (m->source != 0.0 || m->source_e)) &&
         m->reserved == 0;
}

}  // namespace

}  // namespace phastb

using namespace phastb;

extern "C" {

int phastb_t3_internal_force(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                             const double* d, double* f, void* stream) {
  if (!t3_valid_mesh(mesh) || !m || !u || !f) return PHASTB_ERR_ARG;
  return t3_force_launch(*mesh, *m, u, d, f, nullptr, nullptr, (cudaStream_t)stream);
}

int phastb_t3_check_mesh(int n_nodes, int n_elems, const int* elem, const int* order, int n_colors,
                         const int* color_off) {
  return t3_check_mesh_host(n_nodes, n_elems, elem, order, n_colors, color_off);
}

int phastb_t3_psi_history(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                          const double* H_in, double* H_out, double* psi, void* stream) {
  if (!t3_valid_mesh(mesh) || !m || !u || (!H_out && !psi)) return PHASTB_ERR_ARG;
  const int ne = mesh->n_elems;
  { note_launch(); t3_psi_kernel<<<grid_full(ne), kThreads, 0, (cudaStream_t)stream>>>(t3_dev(*mesh), make_mat2<double>(*m), u, H_in, H_out, psi, ne); }
  return last_launch_status();
}

int phastb_t3_damage_apply(const phastb_t3_mesh* mesh, const double* d, const double* H, double gc_over_l0,
                           const double* gc_over_l0_e, double gcl0, const double* gcl0_e, double* y, void* stream) {
  if (!t3_valid_mesh(mesh) || !d || !y) return PHASTB_ERR_ARG;
  return t3_damage_apply_launch(*mesh, d, H, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, y, nullptr,
                                (cudaStream_t)stream, nullptr);
}

int phastb_t3_damage_prepare(const phastb_t3_mesh* mesh, const double* H, double gc_over_l0,
                             const double* gc_over_l0_e, double gcl0, const double* gcl0_e, double* b,
                             double* m_inv, void* stream) {
  if (!t3_valid_mesh(mesh) || !b || !m_inv) return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nb = sizeof(double) * (size_t)mesh->n_nodes;
  int st;
  if ((st = cuda_status(cudaMemsetAsync(b, 0, nb, s)))) return st;
  if ((st = cuda_status(cudaMemsetAsync(m_inv, 0, nb, s)))) return st;
  const T3Dev t = t3_dev(*mesh);
  for (int c = 0; c < mesh->n_colors; ++c) {
    const int k0 = mesh->color_off[c], k1 = mesh->color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_prepare_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, H, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, 0.0, nullptr, b, m_inv, k0, k1); }
  }
  { note_launch(); t3_invert_kernel<<<grid_for(mesh->n_nodes), kThreads, 0, s>>>(mesh->n_nodes, m_inv); }
  return last_launch_status();
}

size_t phastb_t3_damage_solve_workspace_bytes(int n_nodes) { return ppcg_ws_bytes(n_nodes); }

int phastb_t3_damage_solve(const phastb_t3_mesh* mesh, const double* H, double gc_over_l0,
                           const double* gc_over_l0_e, double gcl0, const double* gcl0_e, const double* d_prev,
                           const double* d_init, const uint8_t* fixed, const double* fixed_vals, double tol,
                           int max_iter, int check_every, double* d_out, int* info, void* workspace,
                           size_t workspace_bytes, void* stream) {
  if (!t3_valid_mesh(mesh) || !d_prev || !d_out || max_iter < 0 || check_every < 1) return PHASTB_ERR_ARG;
  if (fixed && !fixed_vals) return PHASTB_ERR_ARG;
  const int n = mesh->n_nodes;
  if (!workspace || workspace_bytes < ppcg_ws_bytes(n)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  PpcgWs w = ppcg_ws(workspace, n);
  int st = phastb_t3_damage_prepare(mesh, H, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, w.b, w.minv, (void*)s);
  if (st) return st;
  T3DamageCtx ctx;
  std::memset(&ctx, 0, sizeof(ctx));
  ctx.mesh = *mesh;
  ctx.H = H;
  ctx.gco = gc_over_l0;
  ctx.gco_e = gc_over_l0_e;
  ctx.gcl0 = gcl0;
  ctx.gcl0_e = gcl0_e;
  LinOp<double> A{t3_damage_op, &ctx, sizeof(ctx)};
  int inf[2] = {0, 0};
  st = ppcg_solve(A, n, w, d_prev, d_init, fixed, fixed_vals, tol, max_iter, check_every, d_out, inf, s);
  if (info) {
    info[0] = inf[0];
    info[1] = inf[1];
  }
  return st;
}

int phastb_t3_damage_apply_ex(const phastb_t3_mesh* mesh, const phastb_t3_damage_model* model, const double* d,
                              const double* H, double* y, void* stream) {
  if (!t3_valid_mesh(mesh) || !valid_model(model) || !d || !y) return PHASTB_ERR_ARG;
  return t3_damage_model_launch(*mesh, *model, d, H, y, nullptr, (cudaStream_t)stream, nullptr);
}

int phastb_t3_damage_prepare_ex(const phastb_t3_mesh* mesh, const phastb_t3_damage_model* model, const double* H,
                                double* b, double* m_inv, void* stream) {
  if (!t3_valid_mesh(mesh) || !valid_model(model) || !b || !m_inv) return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nb = sizeof(double) * (size_t)mesh->n_nodes;
  int st;
  if ((st = cuda_status(cudaMemsetAsync(b, 0, nb, s)))) return st;
  if ((st = cuda_status(cudaMemsetAsync(m_inv, 0, nb, s)))) return st;
  const T3Dev t = t3_dev(*mesh);
  const phastb_t3_damage_model& md = *model;
  for (int c = 0; c < mesh->n_colors; ++c) {
    const int k0 = mesh->color_off[c], k1 = mesh->color_off[c + 1];
    if (k1 <= k0) continue;
    if (md.nodal_h)
      { note_launch(); t3_prepare_nodal_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, H, md.gc_over_l0, md.gc_over_l0_e, md.gcl0, md.gcl0_e, b, m_inv, k0, k1); }
    else
      { note_launch(); t3_prepare_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, H, md.gc_over_l0, md.gc_over_l0_e, md.gcl0, md.gcl0_e, md.source, md.source_e, b, m_inv, k0, k1); }
  }
  { note_launch(); t3_invert_kernel<<<grid_for(mesh->n_nodes), kThreads, 0, s>>>(mesh->n_nodes, m_inv); }
  return last_launch_status();
}

int phastb_t3_damage_solve_ex(const phastb_t3_mesh* mesh, const phastb_t3_damage_model* model, const double* H,
                              const double* d_prev, const double* d_init, const uint8_t* fixed,
                              const double* fixed_vals, double tol, int max_iter, int check_every, double* d_out,
                              int* info, void* workspace, size_t workspace_bytes, void* stream) {
  if (!t3_valid_mesh(mesh) || !valid_model(model) || !d_prev || !d_out || max_iter < 0 || check_every < 1)
    return PHASTB_ERR_ARG;
  if (fixed && !fixed_vals) return PHASTB_ERR_ARG;
  const int n = mesh->n_nodes;
  if (!workspace || workspace_bytes < ppcg_ws_bytes(n)) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  PpcgWs w = ppcg_ws(workspace, n);
  int st = phastb_t3_damage_prepare_ex(mesh, model, H, w.b, w.minv, (void*)s);
  if (st) return st;
  T3ModelCtx ctx;
  std::memset(&ctx, 0, sizeof(ctx));
  ctx.mesh = *mesh;
  ctx.model = *model;
  ctx.H = H;
  LinOp<double> A{t3_model_op, &ctx, sizeof(ctx)};
  int inf[2] = {0, 0};
  st = ppcg_solve(A, n, w, d_prev, d_init, fixed, fixed_vals, tol, max_iter, check_every, d_out, inf, s);
  if (info) {
    info[0] = inf[0];
    info[1] = inf[1];
  }
  return st;
}

int phastb_t3_psi_grad_t(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                         const double* w, double* f, void* stream) {
  if (!t3_valid_mesh(mesh) || !m || !u || !w || !f) return PHASTB_ERR_ARG;
  if (m->psi_split != PHASTB_SPLIT_ISOTROPIC && m->psi_split != PHASTB_SPLIT_LINEAR) return PHASTB_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  int st = cuda_status(cudaMemsetAsync(f, 0, sizeof(double) * 2 * (size_t)mesh->n_nodes, s));
  if (st) return st;
  const T3Dev t = t3_dev(*mesh);
  const Mat2<double> mm = make_mat2<double>(*m);
  for (int c = 0; c < mesh->n_colors; ++c) {
    const int k0 = mesh->color_off[c], k1 = mesh->color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_psi_grad_t_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, mm, u, w, f, k0, k1); }
  }
  return last_launch_status();
}

int phastb_t3_force_dd_t(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u, const double* z,
                         const double* d, double* out, void* stream) {
  if (!t3_valid_mesh(mesh) || !m || !u || !z || !d || !out) return PHASTB_ERR_ARG;
  if (m->stress_split != PHASTB_SPLIT_ISOTROPIC && m->stress_split != PHASTB_SPLIT_LINEAR) return PHASTB_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  int st = cuda_status(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)mesh->n_nodes, s));
  if (st) return st;
  const T3Dev t = t3_dev(*mesh);
  const Mat2<double> mm = make_mat2<double>(*m);
  for (int c = 0; c < mesh->n_colors; ++c) {
    const int k0 = mesh->color_off[c], k1 = mesh->color_off[c + 1];
    if (k1 <= k0) continue;
    { note_launch(); t3_force_dd_t_colour<<<grid_full(k1 - k0), kThreads, 0, s>>>(t, mm, u, z, d, out, k0, k1); }
  }
  return last_launch_status();
}

int phastb_t3_damage_adjoint_grads(const phastb_t3_mesh* mesh, const double* lam, const double* d, double l0,
                                   double* grad_gc_e, double* grad_H, double* lam_K_d_e, double* lam_M_d_e,
                                   void* stream) {
  if (!t3_valid_mesh(mesh) || !lam || !d || !(l0 > 0)) return PHASTB_ERR_ARG;
  const int ne = mesh->n_elems;
  { note_launch(); t3_damage_adjoint_kernel<<<grid_full(ne), kThreads, 0, (cudaStream_t)stream>>>(
      t3_dev(*mesh), lam, d, l0, grad_gc_e, grad_H, lam_K_d_e, lam_M_d_e, ne); }
  return last_launch_status();
}

int phastb_t3_tangent_apply(const phastb_t3_mesh* mesh, const phastb_q4_material* m, const double* u,
                            const double* du, const double* d, double* f, void* stream) {
  if (!t3_valid_mesh(mesh) || !m || !u || !du || !f) return PHASTB_ERR_ARG;
  return t3_tangent_launch(*mesh, *m, u, du, d, f, nullptr, nullptr, (cudaStream_t)stream);
}

}  // extern "C"
