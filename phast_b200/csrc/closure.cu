// Crack closure of the voxel cell (SolverConfig.crack_closure = 'axes'), isotropic group:
// damaged elements add back (1 - g) of the fixed-axis compressive energy
// psi_c = sum_k k_k/2 <v_k . eps>-^2 over the rows v = (trace, e_x, e_y, e_z) with moduli
// k = (lam, 2 mu, 2 mu, 2 mu) (closure_isotropic_rows / closure_isotropic_moduli,
// solid3d/splits.py:486-503), in every element with a damage driver.  For a fixed sign
// pattern s (4 bits per Gauss point) the stress add-back (1 - g) sum_k s_k k_k (v_k . eps) v_k
// is linear in the strain; without a pattern each point uses its own signs
// (solid3d/operator.py:770-877, 1039-1302).
//
// The rows touch only the normal strains, so the add-back is a diagonal stress
// (c0 + c1, c0 + c2, c0 + c3) with c_k = s_k k_k (v_k . eps): one thread per element forms
// the three normal strains at the eight Gauss points from the face differences of the
// corner displacements, writes the element's 24 nodal forces to a scratch that a
// node-centric gather adds to the elastic action in a fixed order, and reduces the macro
// rows.  The kinematic guard of the closure record (operator.py:1713-1770) is here too.
#include "h8_kernels.cuh"
#include "reduce.cuh"
#include <cmath>

namespace phastb {

bool valid_vox(const phastb_voxel_grid* g);
bool valid_mat(const phastb_voxel_material* m);

namespace {

__device__ __forceinline__ void elem_ijk(const VoxGeom& g, int e, int& ie, int& je, int& ke) {
  ie = e % g.nx;
  const int r = e / g.nx;
  je = r % g.ny;
  ke = r / g.ny;
}

__device__ __forceinline__ double shape1(int q, int a) { return q == a ? kC1 : kC2; }

// Displacement gradient of the element at its Gauss points (q = qx + 2 qy + 4 qz):
// G[c][j] = d u_c / d x_j, each derivative from the face differences (grad_sf).
struct ElemGrad {
  double Dx[3][2][2], Dy[3][2][2], Dz[3][2][2];
  __device__ __forceinline__ double at(int c, int j, int q) const {
    const int qx = q & 1, qy = (q >> 1) & 1, qz = q >> 2;
    return j == 0 ? Dx[c][qz][qy] : (j == 1 ? Dy[c][qz][qx] : Dz[c][qy][qx]);
  }
};

__device__ __forceinline__ void elem_grad(const VoxGeom& g, const double* __restrict__ x, const int* nd,
                                          ElemGrad& G) {
  const double ihx = 1.0 / g.hx, ihy = 1.0 / g.hy, ihz = 1.0 / g.hz;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double u[8];
#pragma unroll
    for (int L = 0; L < 8; ++L) u[L] = __ldg(x + 3 * (size_t)nd[L] + c);
    grad_sf(u, ihx, ihy, ihz, G.Dx[c], G.Dy[c], G.Dz[c]);
  }
}

enum ClMode { kClAdd = 0, kClEnergy = 1, kClDiag = 2, kClPattern = 3, kClChange = 4 };

// One thread per element.
//   kClAdd:     sc[(3 L + c) E + e] = the element's add-back forces; ws: the 3 macro rows
//   kClEnergy:  ws: [0.5 sum w (1-g) sigma_c . eps, r_E xx, yy, zz] (pattern NULL: own signs)
//   kClDiag:    sc = the element's Jacobi-diagonal terms; ws: the 3 macro diagonal rows
//               (bits of `pattern`, all bits without it)
//   kClPattern: pat[8 e + q] = own sign bits (bit k: v_k . eps < 0)
//   kClChange:  pat_new as kClPattern; ws: [max k |v.eps|, max (1-g) k |v.eps| over flipped bits]
template <int MODE>
__global__ void __launch_bounds__(kThreads) cl_elem_kernel(VoxGeom g, VoxMat<double> m,
                                                           const uint8_t* __restrict__ slot,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ gq,
                                                           const uint8_t* __restrict__ pattern,
                                                           uint8_t* __restrict__ pat_out, double* __restrict__ sc,
                                                           RedWs ws) {
  const size_t E = (size_t)g.n_elem;
  const double w = g.w, ihx = 1.0 / g.hx, ihy = 1.0 / g.hy, ihz = 1.0 / g.hz;
  double E3[3] = {0.0, 0.0, 0.0};
  if (MODE != kClDiag) {
    const double* Ex = x + 3 * (size_t)g.n_red;
    E3[0] = __ldg(Ex);
    E3[1] = __ldg(Ex + 1);
    E3[2] = __ldg(Ex + 2);
  }
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double mx0 = 0.0, mx1 = 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    const int s = slot[e];
    const bool on = m.driver[s] != PHASTB_DRIVER_NONE;
    const double kk[4] = {m.lam[s], 2.0 * m.mu[s], 2.0 * m.mu[s], 2.0 * m.mu[s]};
    if (MODE == kClDiag) {
      if (!on) {
#pragma unroll
        for (int r = 0; r < 24; ++r) sc[(size_t)r * E + e] = 0.0;
        continue;
      }
      double cx[8], cy[8], cz[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const unsigned bits = pattern ? pattern[8 * (size_t)e + q] : 0xFu;
        const double omg = (1.0 - __ldg(gq + 8 * (size_t)e + q)) * w;
        double c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k] = ((bits >> k) & 1u) ? omg * kk[k] : 0.0;
        cx[q] = c[0] + c[1];
        cy[q] = c[0] + c[2];
        cz[q] = c[0] + c[3];
        acc[0] += cx[q];
        acc[1] += cy[q];
        acc[2] += cz[q];
      }
#pragma unroll
      for (int L = 0; L < 8; ++L) {
        const int ax = L & 1, ay = (L >> 1) & 1, az = L >> 2;
        double dx = 0.0, dy = 0.0, dz = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int qx = q & 1, qy = (q >> 1) & 1, qz = q >> 2;
          const double nx = shape1(qx, ax), ny = shape1(qy, ay), nz = shape1(qz, az);
          const double gx = ny * nz * ihx, gy = nx * nz * ihy, gz = nx * ny * ihz;
          dx += cx[q] * (gx * gx);
          dy += cy[q] * (gy * gy);
          dz += cz[q] * (gz * gz);
        }
        sc[(size_t)(3 * L + 0) * E + e] = dx;
        sc[(size_t)(3 * L + 1) * E + e] = dy;
        sc[(size_t)(3 * L + 2) * E + e] = dz;
      }
      continue;
    }
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    ElemGrad G;
    elem_grad(g, x, nd, G);
    double sx[8], sy[8], sz[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double exx = G.at(0, 0, q) + E3[0], eyy = G.at(1, 1, q) + E3[1], ezz = G.at(2, 2, q) + E3[2];
      const double v[4] = {exx + eyy + ezz, exx, eyy, ezz};
      unsigned own = 0u;
#pragma unroll
      for (int k = 0; k < 4; ++k) own |= (v[k] < 0.0 ? 1u : 0u) << k;
      if (MODE == kClPattern || MODE == kClChange) {
        const unsigned nb = on ? own : 0u;
        pat_out[8 * (size_t)e + q] = (uint8_t)nb;
        if (MODE == kClChange) {
          const unsigned flip = nb ^ pattern[8 * (size_t)e + q];
          const double omg = 1.0 - __ldg(gq + 8 * (size_t)e + q);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double st = on ? kk[k] * fabs(v[k]) : 0.0;
            mx0 = fmax(mx0, st);
            if ((flip >> k) & 1u) mx1 = fmax(mx1, omg * st);
          }
        }
        continue;
      }
      const unsigned bits = pattern ? pattern[8 * (size_t)e + q] : own;
      double c[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) c[k] = (on && ((bits >> k) & 1u)) ? v[k] * kk[k] : 0.0;
      const double omg = 1.0 - __ldg(gq + 8 * (size_t)e + q);
      sx[q] = omg * (c[0] + c[1]);
      sy[q] = omg * (c[0] + c[2]);
      sz[q] = omg * (c[0] + c[3]);
      acc[1] += w * sx[q];
      acc[2] += w * sy[q];
      acc[3] += w * sz[q];
      if (MODE == kClEnergy) acc[0] += 0.5 * w * (sx[q] * exx + sy[q] * eyy + sz[q] * ezz);
    }
    if (MODE != kClAdd) continue;
    // nodal forces f_L = sum_q w sigma_c(q) . grad N_L(q): each normal stress meets the
    // derivative along its own axis, which is constant along that axis
    double Px[2][2], Py[2][2], Pz[2][2], Zr[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        Px[a][b] = w * (sx[2 * b + 4 * a] + sx[1 + 2 * b + 4 * a]);   // [qz][qy], summed over qx
        Py[a][b] = w * (sy[b + 4 * a] + sy[b + 2 + 4 * a]);           // [qz][qx], summed over qy
        Pz[a][b] = w * (sz[b + 2 * a] + sz[b + 2 * a + 4]);           // [qy][qx], summed over qz
      }
    double fx[8], fy[8], fz[8];
    grad_sf_t(Px, Zr, Zr, ihx, ihy, ihz, fx);
    grad_sf_t(Zr, Py, Zr, ihx, ihy, ihz, fy);
    grad_sf_t(Zr, Zr, Pz, ihx, ihy, ihz, fz);
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      sc[(size_t)(3 * L + 0) * E + e] = fx[L];
      sc[(size_t)(3 * L + 1) * E + e] = fy[L];
      sc[(size_t)(3 * L + 2) * E + e] = fz[L];
    }
  }
  if (MODE == kClAdd) {
    double r[3] = {acc[1], acc[2], acc[3]};
    reduce_multi<3>(r, ws);
  } else if (MODE == kClDiag) {
    double r[3] = {acc[0], acc[1], acc[2]};
    reduce_multi<3>(r, ws);
  } else if (MODE == kClEnergy) {
    reduce_multi<4>(acc, ws);
  } else if (MODE == kClChange) {
    __shared__ double sh[32];
    const double b0 = block_max(mx0, sh);
    const double b1 = block_max(mx1, sh);
    if (threadIdx.x == 0) {
      ws.part[blockIdx.x] = b0;
      ws.part[kMaxPartials + blockIdx.x] = b1;
    }
    if (arrive_last(ws.counter)) {
      const double t0 = fold_max(ws.part, gridDim.x, sh);
      const double t1 = fold_max(ws.part + kMaxPartials, gridDim.x, sh);
      if (threadIdx.x == 0) {
        ws.out[0] = t0;
        ws.out[1] = t1;
        *ws.counter = 0u;
      }
    }
  }
}

// y[3 n + c] += sum over the elements of node n of sc[(3 L + c) E + e] (rows with mask set are
// left alone); the first thread adds the three macro rows ws.out[0..2] to y[3 n_red + i].
__global__ void __launch_bounds__(kThreads) cl_gather_add_kernel(VoxGeom g, const double* __restrict__ sc,
                                                                 const uint8_t* __restrict__ mask,
                                                                 const double* __restrict__ macro,
                                                                 double* __restrict__ y) {
  const size_t E = (size_t)g.n_elem;
  if (blockIdx.x == 0 && threadIdx.x < 3) {
    const size_t idx = 3 * (size_t)g.n_red + threadIdx.x;
    if (!(mask && mask[idx])) y[idx] += macro[threadIdx.x];
  }
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n_red; n += gridDim.x * blockDim.x) {
    const int ir = n % g.rx;
    const int rem = n / g.rx;
    const int jr = rem % g.ry, kr = rem / g.ry;
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      int ie = ir - (L & 1), je = jr - ((L >> 1) & 1), ke = kr - ((L >> 2) & 1);
      if (g.px) { if (ie < 0) ie += g.nx; } else if (ie < 0 || ie >= g.nx) continue;
      if (g.py) { if (je < 0) je += g.ny; } else if (je < 0 || je >= g.ny) continue;
      if (g.pz) { if (ke < 0) ke += g.nz; } else if (ke < 0 || ke >= g.nz) continue;
      const size_t e = (size_t)ie + (size_t)g.nx * ((size_t)je + (size_t)g.ny * ke);
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] += __ldg(sc + (size_t)(3 * L + c) * E + e);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t idx = 3 * (size_t)n + c;
      if (!(mask && mask[idx])) y[idx] += acc[c];
    }
  }
}

// ws.out = [min element-mean normal strain, min principal value of the element-mean strain,
// min Gauss-point det(I + E + grad u~), the same three over the damaged elements (mean nodal
// damage > threshold; +inf when there are none)] (kinematic_guard, operator.py:1713-1770).
__global__ void __launch_bounds__(kThreads) kin_guard_kernel(VoxGeom g, const double* __restrict__ x,
                                                             const double* __restrict__ d, double threshold,
                                                             RedWs ws) {
  const double* Ex = x + 3 * (size_t)g.n_red;
  double E6[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) E6[i] = __ldg(Ex + i);
  // macro displacement gradient: the engineering strain as a symmetric tensor
  const double Em[3][3] = {{E6[0], 0.5 * E6[5], 0.5 * E6[4]},
                           {0.5 * E6[5], E6[1], 0.5 * E6[3]},
                           {0.5 * E6[4], 0.5 * E6[3], E6[2]}};
  double mn = INFINITY, mp = INFINITY, md = INFINITY, dn = INFINITY, dp = INFINITY, dd = INFINITY;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    ElemGrad G;
    elem_grad(g, x, nd, G);
    double eps[6] = {0, 0, 0, 0, 0, 0};
    double emin_det = INFINITY;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      double F[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) F[i][j] = (i == j ? 1.0 : 0.0) + Em[i][j] + G.at(i, j, q);
      const double det = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                         F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                         F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
      emin_det = fmin(emin_det, det);
      eps[0] += G.at(0, 0, q) + E6[0];
      eps[1] += G.at(1, 1, q) + E6[1];
      eps[2] += G.at(2, 2, q) + E6[2];
      eps[3] += G.at(1, 2, q) + G.at(2, 1, q) + E6[3];
      eps[4] += G.at(0, 2, q) + G.at(2, 0, q) + E6[4];
      eps[5] += G.at(0, 1, q) + G.at(1, 0, q) + E6[5];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) eps[i] *= 0.125;
    const double en = fmin(eps[0], fmin(eps[1], eps[2]));
    double ev[3];
    eig3(eps[0], eps[1], eps[2], 0.5 * eps[5], 0.5 * eps[4], 0.5 * eps[3], ev);
    mn = fmin(mn, en);
    mp = fmin(mp, ev[0]);
    md = fmin(md, emin_det);
    if (d) {
      double dm = 0.0;
#pragma unroll
      for (int L = 0; L < 8; ++L) dm += __ldg(d + nd[L]);
      if (dm / 8.0 > threshold) {
        dn = fmin(dn, en);
        dp = fmin(dp, ev[0]);
        dd = fmin(dd, emin_det);
      }
    }
  }
  __shared__ double sh[32];
  const double v[6] = {mn, mp, md, dn, dp, dd};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double b = block_min(v[k], sh);
    if (threadIdx.x == 0) ws.part[k * kMaxPartials + blockIdx.x] = b;
  }
  if (arrive_last(ws.counter)) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double t = fold_min(ws.part + k * kMaxPartials, gridDim.x, sh);
      if (threadIdx.x == 0) ws.out[k] = t;
    }
    if (threadIdx.x == 0) *ws.counter = 0u;
  }
}

}  // namespace

size_t closure_scratch_bytes(const VoxGeom& v) {
  return align_up(sizeof(double) * 24 * (size_t)v.n_elem) + red_ws_bytes();
}

// y += the closure add-back of x at the degradation gq (pattern NULL: own signs); rows with
// mask set are left alone.  sc: closure_scratch_bytes.
int closure_add_launch(const VoxGeom& v, const VoxMat<double>& m, const uint8_t* slot, const double* x,
                       const double* gq, const uint8_t* pattern, const uint8_t* mask, double* y, void* sc,
                       cudaStream_t s) {
  double* e = static_cast<double*>(sc);
  RedWs ws = red_ws(static_cast<char*>(sc) + align_up(sizeof(double) * 24 * (size_t)v.n_elem));
  { note_launch(); cl_elem_kernel<kClAdd><<<grid_for(v.n_elem), kThreads, 0, s>>>(v, m, slot, x, gq, pattern, nullptr,
                                                                                  e, ws); }
  { note_launch(); cl_gather_add_kernel<<<grid_for(v.n_red), kThreads, 0, s>>>(v, e, mask, ws.out, y); }
  return last_launch_status();
}

// diag += the closure terms of the Jacobi diagonal (pattern NULL: every bit).
int closure_diag_launch(const VoxGeom& v, const VoxMat<double>& m, const uint8_t* slot, const double* gq,
                        const uint8_t* pattern, double* diag, void* sc, cudaStream_t s) {
  double* e = static_cast<double*>(sc);
  RedWs ws = red_ws(static_cast<char*>(sc) + align_up(sizeof(double) * 24 * (size_t)v.n_elem));
  { note_launch(); cl_elem_kernel<kClDiag><<<grid_for(v.n_elem), kThreads, 0, s>>>(v, m, slot, nullptr, gq, pattern,
                                                                                   nullptr, e, ws); }
  { note_launch(); cl_gather_add_kernel<<<grid_for(v.n_red), kThreads, 0, s>>>(v, e, nullptr, ws.out, diag); }
  return last_launch_status();
}

int closure_reset(void* sc, const VoxGeom& v, cudaStream_t s) {
  return red_ws_reset(red_ws(static_cast<char*>(sc) + align_up(sizeof(double) * 24 * (size_t)v.n_elem)), s);
}

}  // namespace phastb

using namespace phastb;

extern "C" {

size_t phastb_h8_closure_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  return closure_scratch_bytes(make_vox_geom(*g));
}

int phastb_h8_closure_pattern(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* x, uint8_t* pattern, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !pattern) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  { note_launch(); cl_elem_kernel<kClPattern><<<grid_for(v.n_elem), kThreads, 0, (cudaStream_t)stream>>>(
        v, make_vox_mat<double>(*m), slot, x, nullptr, nullptr, pattern, nullptr, RedWs{}); }
  return last_launch_status();
}

int phastb_h8_closure_pattern_change(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                     const uint8_t* slot, const double* x, const double* gq,
                                     const uint8_t* pattern_old, double tolerance, uint8_t* pattern_new,
                                     int* changed_host, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !gq || !pattern_old || !pattern_new || !changed_host ||
      pattern_old == pattern_new)
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_closure_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(static_cast<char*>(workspace) + align_up(sizeof(double) * 24 * (size_t)v.n_elem));
  int st = red_ws_reset(ws, s);
  if (st) return st;
  { note_launch(); cl_elem_kernel<kClChange><<<grid_for(v.n_elem), kThreads, 0, s>>>(
        v, make_vox_mat<double>(*m), slot, x, gq, pattern_old, pattern_new, nullptr, ws); }
  if ((st = last_launch_status())) return st;
  double r[2];
  if ((st = red_ws_fetch(ws, r, 2, s))) return st;
  // a flip counts where its stress jump exceeds tolerance x the largest closure stress
  *changed_host = r[1] > tolerance * r[0] ? 1 : 0;
  return PHASTB_OK;
}

int phastb_h8_closure_apply_add(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                const double* x, const double* gq, const uint8_t* pattern, const uint8_t* mask,
                                double* y, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !gq || !y) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_closure_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  int st = closure_reset(workspace, v, s);
  if (st) return st;
  return closure_add_launch(v, make_vox_mat<double>(*m), slot, x, gq, pattern, mask, y, workspace, s);
}

int phastb_h8_closure_diagonal_add(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                   const uint8_t* slot, const double* gq, const uint8_t* pattern, double* diag,
                                   void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !gq || !diag) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_closure_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  int st = closure_reset(workspace, v, s);
  if (st) return st;
  return closure_diag_launch(v, make_vox_mat<double>(*m), slot, gq, pattern, diag, workspace, s);
}

int phastb_h8_closure_energy(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                             const double* x, const double* gq, const uint8_t* pattern, double* out_host,
                             void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !gq || !out_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_closure_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(static_cast<char*>(workspace) + align_up(sizeof(double) * 24 * (size_t)v.n_elem));
  int st = red_ws_reset(ws, s);
  if (st) return st;
  { note_launch(); cl_elem_kernel<kClEnergy><<<grid_for(v.n_elem), kThreads, 0, s>>>(
        v, make_vox_mat<double>(*m), slot, x, gq, pattern, nullptr, nullptr, ws); }
  if ((st = last_launch_status())) return st;
  return red_ws_fetch(ws, out_host, 4, s);
}

int phastb_h8_kinematic_guard(const phastb_voxel_grid* g, const double* x, const double* d, double threshold,
                              double* out_host, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !x || !out_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < red_ws_bytes()) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(workspace);
  int st = red_ws_reset(ws, s);
  if (st) return st;
  { note_launch(); kin_guard_kernel<<<grid_for(v.n_elem), kThreads, 0, s>>>(v, x, d, threshold, ws); }
  if ((st = last_launch_status())) return st;
  return red_ws_fetch(ws, out_host, 6, s);
}

}  // extern "C"
