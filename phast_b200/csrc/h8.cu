// Periodic voxel H8 operators: degradation, elastic action and diagonal,
// driving force + history, AT2 damage action / rhs / diagonal.
// C ABI in include/phastb.h.
#include "h8_kernels.cuh"
#include "h8_tile.cuh"
#include "reduce.cuh"

#include <cmath>
#include <mutex>

namespace phastb {

template <typename T>
__device__ __forceinline__ T g_of(T kappa, T d) {
  const T o = T(1) - d;
  return (T(1) - kappa) * o * o + kappa;
}

__device__ __forceinline__ void elem_ijk(const VoxGeom& g, int e, int& ie, int& je, int& ke) {
  ie = e % g.nx;
  const int r = e / g.nx;
  je = r % g.ny;
  ke = r / g.ny;
}

// Gauss-point degradation factors of one element from gq (E,8), from nodal d or 1.
template <typename T>
__device__ __forceinline__ void load_g(const VoxGeom& g, const T* __restrict__ gq, const T* __restrict__ d,
                                       T kappa, int e, const int* nd, T* gv) {
  if (gq) {
#pragma unroll
    for (int q = 0; q < 8; ++q) gv[q] = __ldg(gq + 8 * (size_t)e + q);
  } else if (d) {
    T dd[8], dq[8];
#pragma unroll
    for (int L = 0; L < 8; ++L) dd[L] = __ldg(d + nd[L]);
    interp_sf(dd, dq);
#pragma unroll
    for (int q = 0; q < 8; ++q) gv[q] = g_of(kappa, dq[q]);
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) gv[q] = T(1);
  }
}

// ------------------------------------------------------------ elastic action

template <typename T, bool ENERGY>
__global__ void __launch_bounds__(kThreads) h8_mech_elem_kernel(VoxGeom g, VoxMat<T> m,
                                                                const uint8_t* __restrict__ slot,
                                                                const T* __restrict__ x, const T* __restrict__ gq,
                                                                const T* __restrict__ d, T* __restrict__ scratch,
                                                                T* __restrict__ y, const uint8_t* __restrict__ mask,
                                                                RedWs ws, const int* guard) {
  if (guard && *guard == 0) return;
  const T ihx = T(1.0 / g.hx), ihy = T(1.0 / g.hy), ihz = T(1.0 / g.hz), w = T(g.w);
  const size_t E = (size_t)g.n_elem;
  const T* Ex = x + 3 * (size_t)g.n_red;
  const T E6[6] = {__ldg(Ex), __ldg(Ex + 1), __ldg(Ex + 2), __ldg(Ex + 3), __ldg(Ex + 4), __ldg(Ex + 5)};
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    T gv[8];
    load_g(g, gq, d, m.kappa, e, nd, gv);
    const int s = slot[e];
    T D[3][3][2][2];  // [component][axis][..][..]
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T u[8];
#pragma unroll
      for (int L = 0; L < 8; ++L) u[L] = __ldg(x + 3 * (size_t)nd[L] + c);
      grad_sf(u, ihx, ihy, ihz, D[c][0], D[c][1], D[c][2]);
    }
    T P[3][3][2][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) P[c][a][i][j] = T(0);
#pragma unroll
    for (int qz = 0; qz < 2; ++qz)
#pragma unroll
      for (int qy = 0; qy < 2; ++qy)
#pragma unroll
        for (int qx = 0; qx < 2; ++qx) {
          T ep[6];
          ep[0] = D[0][0][qz][qy] + E6[0];
          ep[1] = D[1][1][qz][qx] + E6[1];
          ep[2] = D[2][2][qy][qx] + E6[2];
          ep[3] = D[1][2][qy][qx] + D[2][1][qz][qx] + E6[3];
          ep[4] = D[0][2][qy][qx] + D[2][0][qz][qy] + E6[4];
          ep[5] = D[0][1][qz][qx] + D[1][0][qz][qy] + E6[5];
          T sg[6];
          voigt_stress(m, s, ep, sg);
          const T gw = gv[qx + 2 * qy + 4 * qz] * w;
#pragma unroll
          for (int k = 0; k < 6; ++k) sg[k] *= gw;
          if (ENERGY) {
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[6] += 0.5 * double(sg[k]) * double(ep[k]);
          }
          P[0][0][qz][qy] += sg[0];
          P[0][1][qz][qx] += sg[5];
          P[0][2][qy][qx] += sg[4];
          P[1][0][qz][qy] += sg[5];
          P[1][1][qz][qx] += sg[1];
          P[1][2][qy][qx] += sg[3];
          P[2][0][qz][qy] += sg[4];
          P[2][1][qz][qx] += sg[3];
          P[2][2][qy][qx] += sg[2];
        }
    // r_E = sum_q w g sigma: each stress component is summed by one P block
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        acc[0] += double(P[0][0][i][j]);
        acc[1] += double(P[1][1][i][j]);
        acc[2] += double(P[2][2][i][j]);
        acc[3] += double(P[1][2][i][j]);
        acc[4] += double(P[0][2][i][j]);
        acc[5] += double(P[0][1][i][j]);
      }
    if (scratch) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T out[8];
        grad_sf_t(P[c][0], P[c][1], P[c][2], ihx, ihy, ihz, out);
#pragma unroll
        for (int L = 0; L < 8; ++L) scratch[(size_t)(L * 3 + c) * E + e] = out[L];
      }
    }
  }
  constexpr int NK = ENERGY ? 7 : 6;
  __shared__ double sh[32 * NK];
  double v[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) v[k] = acc[k];
  block_sum_multi<NK>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NK; ++k) ws.part[k * kMaxPartials + blockIdx.x] = v[k];
  }
  if (arrive_last(ws.counter)) {
    double f[NK];
    fold_sum_multi<NK>(ws.part, kMaxPartials, gridDim.x, f, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NK; ++k) {
        ws.out[k] = f[k];
        if (y && k < 6) {
          const size_t idx = 3 * (size_t)g.n_red + k;
          y[idx] = (mask && mask[idx]) ? T(0) : T(f[k]);
        }
      }
      *ws.counter = 0u;
    }
  }
}

// Deterministic element->node gather of NC components per node.
template <typename T, int NC>
__global__ void __launch_bounds__(kThreads) h8_gather_kernel(VoxGeom g, const T* __restrict__ scratch,
                                                             T* __restrict__ y, const uint8_t* __restrict__ mask,
                                                             const int* guard) {
  if (guard && *guard == 0) return;
  const size_t E = (size_t)g.n_elem;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n_red; n += gridDim.x * blockDim.x) {
    const int ir = n % g.rx;
    const int rem = n / g.rx;
    const int jr = rem % g.ry, kr = rem / g.ry;
    T acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = T(0);
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      int ie = ir - (L & 1), je = jr - ((L >> 1) & 1), ke = kr - ((L >> 2) & 1);
      if (g.px) { if (ie < 0) ie += g.nx; } else if (ie < 0 || ie >= g.nx) continue;
      if (g.py) { if (je < 0) je += g.ny; } else if (je < 0 || je >= g.ny) continue;
      if (g.pz) { if (ke < 0) ke += g.nz; } else if (ke < 0 || ke >= g.nz) continue;
      const size_t e = (size_t)ie + (size_t)g.nx * ((size_t)je + (size_t)g.ny * ke);
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] += __ldg(scratch + (size_t)(L * NC + c) * E + e);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const size_t idx = (size_t)n * NC + c;
      y[idx] = (mask && mask[idx]) ? T(0) : acc[c];
    }
  }
}

// ------------------------------------------------------------ elastic diagonal

template <typename T>
__global__ void __launch_bounds__(kThreads) h8_mdiag_elem_kernel(VoxGeom g, VoxMat<T> m,
                                                                 const uint8_t* __restrict__ slot,
                                                                 const T* __restrict__ gq, const T* __restrict__ d,
                                                                 T* __restrict__ scratch, T* __restrict__ diag,
                                                                 RedWs ws) {
  const T ihx = T(1.0 / g.hx), ihy = T(1.0 / g.hy), ihz = T(1.0 / g.hz), w = T(g.w);
  const size_t E = (size_t)g.n_elem;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    T gv[8];
    load_g(g, gq, d, m.kappa, e, nd, gv);
    const int s = slot[e];
    T C[6][6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const int a = i < j ? i : j, b = i < j ? j : i;
        C[i][j] = m.C[s][a * 6 - a * (a - 1) / 2 + (b - a)];
      }
    T out[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int L = 0; L < 8; ++L) out[c][L] = T(0);
    T gsum = 0;
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      const int qx = q & 1, qy = (q >> 1) & 1, qz = q >> 2;
      const T gw = gv[q] * w;
      gsum += gw;
#pragma unroll
      for (int L = 0; L < 8; ++L) {
        const int ax = L & 1, ay = (L >> 1) & 1, az = L >> 2;
        const T nx_ = (qx == ax) ? T(kC1) : T(kC2);
        const T ny_ = (qy == ay) ? T(kC1) : T(kC2);
        const T nz_ = (qz == az) ? T(kC1) : T(kC2);
        const T gx = (ax ? ihx : -ihx) * ny_ * nz_;
        const T gy = (ay ? ihy : -ihy) * nx_ * nz_;
        const T gz = (az ? ihz : -ihz) * nx_ * ny_;
        out[0][L] += gw * (C[0][0] * gx * gx + C[4][4] * gz * gz + C[5][5] * gy * gy +
                           T(2) * (C[0][4] * gx * gz + C[0][5] * gx * gy + C[4][5] * gz * gy));
        out[1][L] += gw * (C[1][1] * gy * gy + C[3][3] * gz * gz + C[5][5] * gx * gx +
                           T(2) * (C[1][3] * gy * gz + C[1][5] * gy * gx + C[3][5] * gz * gx));
        out[2][L] += gw * (C[2][2] * gz * gz + C[3][3] * gy * gy + C[4][4] * gx * gx +
                           T(2) * (C[2][3] * gz * gy + C[2][4] * gz * gx + C[3][4] * gy * gx));
      }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] += double(gsum) * double(C[k][k]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int L = 0; L < 8; ++L) scratch[(size_t)(L * 3 + c) * E + e] = out[c][L];
  }
  __shared__ double sh[32 * 6];
  double v[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = acc[k];
  block_sum_multi<6>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) ws.part[k * kMaxPartials + blockIdx.x] = v[k];
  }
  if (arrive_last(ws.counter)) {
    double f[6];
    fold_sum_multi<6>(ws.part, kMaxPartials, gridDim.x, f, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < 6; ++k) diag[3 * (size_t)g.n_red + k] = T(f[k]);
      *ws.counter = 0u;
    }
  }
}

// ------------------------------------------------------------ degradation

template <typename T>
__global__ void h8_degradation_kernel(VoxGeom g, const T* __restrict__ d, T kappa, T* __restrict__ gout) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    T gv[8];
    load_g<T>(g, nullptr, d, kappa, e, nd, gv);
#pragma unroll
    for (int q = 0; q < 8; ++q) gout[8 * (size_t)e + q] = gv[q];
  }
}

// ------------------------------------------------------------ driving force

__global__ void __launch_bounds__(kThreads) h8_driving_kernel(VoxGeom g, VoxMat<double> m,
                                                              const uint8_t* __restrict__ slot,
                                                              const double* __restrict__ x,
                                                              const double* __restrict__ Hprev,
                                                              double* __restrict__ Y, double* __restrict__ Hout) {
  const double ihx = 1.0 / g.hx, ihy = 1.0 / g.hy, ihz = 1.0 / g.hz;
  const double* Ex = x + 3 * (size_t)g.n_red;
  const double E6[6] = {__ldg(Ex), __ldg(Ex + 1), __ldg(Ex + 2), __ldg(Ex + 3), __ldg(Ex + 4), __ldg(Ex + 5)};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    const int s = slot[e];
    const int drv = m.driver[s];
    double yq[8];
    if (drv == PHASTB_DRIVER_NONE) {
#pragma unroll
      for (int q = 0; q < 8; ++q) yq[q] = 0.0;
    } else {
      int ie, je, ke;
      elem_ijk(g, e, ie, je, ke);
      int nd[8];
      vox_corners(g, ie, je, ke, nd);
      double D[3][3][2][2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double u[8];
#pragma unroll
        for (int L = 0; L < 8; ++L) u[L] = __ldg(x + 3 * (size_t)nd[L] + c);
        grad_sf(u, ihx, ihy, ihz, D[c][0], D[c][1], D[c][2]);
      }
#pragma unroll
      for (int qz = 0; qz < 2; ++qz)
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx) {
            double ep[6];
            ep[0] = D[0][0][qz][qy] + E6[0];
            ep[1] = D[1][1][qz][qx] + E6[1];
            ep[2] = D[2][2][qy][qx] + E6[2];
            ep[3] = D[1][2][qy][qx] + D[2][1][qz][qx] + E6[3];
            ep[4] = D[0][2][qy][qx] + D[2][0][qz][qy] + E6[4];
            ep[5] = D[0][1][qz][qx] + D[1][0][qz][qy] + E6[5];
            double val;
            if (drv == PHASTB_DRIVER_FULL) {
              double sg[6];
              voigt_stress(m, s, ep, sg);
              val = 0.0;
#pragma unroll
              for (int k = 0; k < 6; ++k) val += ep[k] * sg[k];
              val *= 0.5;
            } else {
              double ev[3];
              eig3(ep[0], ep[1], ep[2], 0.5 * ep[5], 0.5 * ep[4], 0.5 * ep[3], ev);
              double trp = ep[0] + ep[1] + ep[2];
              trp = trp > 0.0 ? trp : 0.0;
              double sp = 0.0;
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                const double v = ev[k] > 0.0 ? ev[k] : 0.0;
                sp += v * v;
              }
              val = 0.5 * m.lam[s] * trp * trp + m.mu[s] * sp;
            }
            yq[qx + 2 * qy + 4 * qz] = val;
          }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const size_t k = 8 * (size_t)e + q;
      if (Y) Y[k] = yq[q];
      if (Hout) {
        const double h = Hprev ? Hprev[k] : 0.0;
        Hout[k] = yq[q] > h ? yq[q] : h;
      }
    }
  }
}

// ------------------------------------------------------------ damage

template <int MODE>  // 0 action, 1 rhs, 2 diagonal
__global__ void __launch_bounds__(kThreads) h8_damage_elem_kernel(VoxGeom g, VoxMat<double> m,
                                                                  const uint8_t* __restrict__ slot,
                                                                  const double* __restrict__ d,
                                                                  const double* __restrict__ H, double scale,
                                                                  double kdiag, double* __restrict__ scratch,
                                                                  const int* guard) {
  if (guard && *guard == 0) return;
  const double ihx = 1.0 / g.hx, ihy = 1.0 / g.hy, ihz = 1.0 / g.hz, w = g.w;
  const double ch = 2.0 * (1.0 - m.kappa);
  const double ell = m.ell;
  const size_t E = (size_t)g.n_elem;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    const double Gc = m.Gc[slot[e]];
    double Hq[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) Hq[q] = H ? __ldg(H + 8 * (size_t)e + q) : 0.0;
    double out[8];
    if (MODE == 0) {
      int ie, je, ke;
      elem_ijk(g, e, ie, je, ke);
      int nd[8];
      vox_corners(g, ie, je, ke, nd);
      double dd[8], dq[8];
#pragma unroll
      for (int L = 0; L < 8; ++L) dd[L] = __ldg(d + nd[L]);
      interp_sf(dd, dq);
      double mq[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) mq[q] = w * (Gc / ell + ch * Hq[q]) * dq[q];
      interp_sf_t(mq, out);
      double Dx[2][2], Dy[2][2], Dz[2][2];
      grad_sf(dd, ihx, ihy, ihz, Dx, Dy, Dz);
      const double k2 = 2.0 * w * Gc * ell;
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          Dx[i][j] *= k2;
          Dy[i][j] *= k2;
          Dz[i][j] *= k2;
        }
      double og[8];
      grad_sf_t(Dx, Dy, Dz, ihx, ihy, ihz, og);
#pragma unroll
      for (int L = 0; L < 8; ++L) out[L] += og[L];
    } else if (MODE == 1) {
      double hq[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) hq[q] = ch * (Hq[q] * w);
      interp_sf_t(hq, out);
    } else {
#pragma unroll
      for (int L = 0; L < 8; ++L) {
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const double n = ((q & 1) == (L & 1) ? kC1 : kC2) * (((q >> 1) & 1) == ((L >> 1) & 1) ? kC1 : kC2) *
                           ((q >> 2) == (L >> 2) ? kC1 : kC2);
          acc += (Hq[q] * w) * (n * n);
        }
        out[L] = Gc * kdiag + ch * acc;
      }
    }
#pragma unroll
    for (int L = 0; L < 8; ++L) scratch[(size_t)L * E + e] = scale * out[L];
  }
}

// ------------------------------------------------------------ host helpers

bool valid_vox(const phastb_voxel_grid* g) {
  return g && g->nx >= 1 && g->ny >= 1 && g->nz >= 1 && g->hx > 0 && g->hy > 0 && g->hz > 0 &&
         (long long)(g->nx + 1) * (g->ny + 1) * (g->nz + 1) < (1LL << 31) / 24;
}

bool valid_mat(const phastb_voxel_material* m) {
  return m && m->n_slots >= 1 && m->n_slots <= PHASTB_MAX_SLOTS && m->ell > 0;
}

size_t h8_scratch_bytes(const VoxGeom& v, int dtype) {
  const size_t w = dtype == PHASTB_F32 ? 4 : 8;
  return align_up(24 * w * (size_t)v.n_elem) + red_ws_bytes();
}

template <typename T>
int h8_mech_apply_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* x, const T* gq,
                    const T* d, const uint8_t* mask, T* y, void* scratch, const int* guard, cudaStream_t s) {
  RedWs ws = red_ws(static_cast<char*>(scratch) + align_up(24 * sizeof(T) * (size_t)v.n_elem));
  return h8_mech_tile_launch<T>(v, mm, slot, x, gq, d, mask, y, ws, guard, false, false, s);
}

template <typename T>
int h8_mech_apply_dot_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* x, const T* gq,
                        const T* d, const uint8_t* mask, T* y, void* scratch, const int* guard, cudaStream_t s) {
  RedWs ws = red_ws(static_cast<char*>(scratch) + align_up(24 * sizeof(T) * (size_t)v.n_elem));
  return h8_mech_tile_launch<T>(v, mm, slot, x, gq, d, mask, y, ws, guard, true, false, s);
}

// The reduction ticket inside an element scratch must start at zero: every
// entry point that hands a caller workspace to the actions resets it once.
int h8_scratch_reset(const VoxGeom& v, int word, void* scratch, cudaStream_t s) {
  return red_ws_reset(red_ws(static_cast<char*>(scratch) + align_up(24 * (size_t)word * (size_t)v.n_elem)), s);
}

const double* h8_apply_dot_slot(const VoxGeom& v, int word, void* scratch) {
  return red_ws(static_cast<char*>(scratch) + align_up(24 * (size_t)word * (size_t)v.n_elem)).out + kOutDot;
}

template int h8_mech_apply_dot_t<double>(const VoxGeom&, const VoxMat<double>&, const uint8_t*, const double*,
                                         const double*, const double*, const uint8_t*, double*, void*, const int*,
                                         cudaStream_t);
template int h8_mech_apply_dot_t<float>(const VoxGeom&, const VoxMat<float>&, const uint8_t*, const float*,
                                        const float*, const float*, const uint8_t*, float*, void*, const int*,
                                        cudaStream_t);

template int h8_mech_apply_t<double>(const VoxGeom&, const VoxMat<double>&, const uint8_t*, const double*,
                                     const double*, const double*, const uint8_t*, double*, void*, const int*,
                                     cudaStream_t);
template int h8_mech_apply_t<float>(const VoxGeom&, const VoxMat<float>&, const uint8_t*, const float*,
                                    const float*, const float*, const uint8_t*, float*, void*, const int*,
                                    cudaStream_t);

template <typename T>
int h8_mech_diag_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* gq, const T* d, T* diag,
                   void* scratch, cudaStream_t s) {
  T* sc = static_cast<T*>(scratch);
  RedWs ws = red_ws(static_cast<char*>(scratch) + align_up(24 * sizeof(T) * (size_t)v.n_elem));
  { note_launch(); h8_mdiag_elem_kernel<T><<<grid_for(v.n_elem), kThreads, 0, s>>>(v, mm, slot, gq, d, sc, diag, ws); }
  { note_launch(); h8_gather_kernel<T, 3><<<grid_for(v.n_red), kThreads, 0, s>>>(v, sc, diag, nullptr, nullptr); }
  return last_launch_status();
}

template int h8_mech_diag_t<double>(const VoxGeom&, const VoxMat<double>&, const uint8_t*, const double*,
                                    const double*, double*, void*, cudaStream_t);
template int h8_mech_diag_t<float>(const VoxGeom&, const VoxMat<float>&, const uint8_t*, const float*, const float*,
                                   float*, void*, cudaStream_t);

double damage_kdiag(const VoxGeom& v, double ell) {
  // diag of M/ell + ell L for one corner (the same at every corner by symmetry)
  const double c[2] = {kC1, kC2};
  double acc = 0.0;
  for (int q = 0; q < 8; ++q) {
    const int qx = q & 1, qy = (q >> 1) & 1, qz = q >> 2;
    const double nx = c[qx != 0], ny = c[qy != 0], nz = c[qz != 0];  // corner L = 0
    const double n = nx * ny * nz;
    const double gx = -ny * nz / v.hx, gy = -nx * nz / v.hy, gz = -nx * ny / v.hz;
    acc += v.w * (n * n / ell + ell * (gx * gx + gy * gy + gz * gz));
  }
  return acc;
}

int h8_damage_launch(const VoxGeom& v, const VoxMat<double>& mm, const uint8_t* slot, int mode, const double* d,
                     const double* H, double scale, double* y, const uint8_t* mask, void* scratch,
                     const int* guard, cudaStream_t s) {
  double* sc = static_cast<double*>(scratch);
  const int G = grid_for(v.n_elem);
  const double kd = damage_kdiag(v, double(mm.ell));
  if (mode == 0 || mode == 3) {
    RedWs ws = red_ws(static_cast<char*>(scratch) + align_up(24 * sizeof(double) * (size_t)v.n_elem));
    return h8_damage_tile_launch<double>(v, mm, slot, d, H, scale, mask, y, ws, guard, mode == 3, s);
  }
  if (mode == 1)
    { note_launch(); h8_damage_elem_kernel<1><<<G, kThreads, 0, s>>>(v, mm, slot, d, H, scale, kd, sc, guard); }
  else
    { note_launch(); h8_damage_elem_kernel<2><<<G, kThreads, 0, s>>>(v, mm, slot, d, H, scale, kd, sc, guard); }
  { note_launch(); h8_gather_kernel<double, 1><<<grid_for(v.n_red), kThreads, 0, s>>>(v, sc, y, mask, guard); }
  return last_launch_status();
}

}  // namespace phastb

using namespace phastb;

extern "C" {

size_t phastb_h8_scratch_bytes(const phastb_voxel_grid* g, int dtype) {
  if (!valid_vox(g)) return 0;
  return h8_scratch_bytes(make_vox_geom(*g), dtype);
}

int phastb_h8_degradation(const phastb_voxel_grid* g, int dtype, const void* d, double kappa, void* g_out,
                          void* stream) {
  if (!valid_vox(g) || !d || !g_out) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == PHASTB_F64)
    { note_launch(); h8_degradation_kernel<double><<<grid_for(v.n_elem), kThreads, 0, s>>>(v, (const double*)d, kappa,
                                                                         (double*)g_out); }
  else if (dtype == PHASTB_F32)
    { note_launch(); h8_degradation_kernel<float><<<grid_for(v.n_elem), kThreads, 0, s>>>(v, (const float*)d, (float)kappa,
                                                                        (float*)g_out); }
  else
    return PHASTB_ERR_ARG;
  return last_launch_status();
}

int phastb_h8_mech_apply(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot, int dtype,
                         const void* x, const void* gq, const void* d, const uint8_t* mask, void* y, void* scratch,
                         void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !y || !scratch) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(static_cast<char*>(scratch) +
                    align_up((dtype == PHASTB_F32 ? 4 : 8) * 24 * (size_t)v.n_elem));
  int st = red_ws_reset(ws, s);
  if (st) return st;
  if (dtype == PHASTB_F64)
    return h8_mech_apply_t<double>(v, make_vox_mat<double>(*m), slot, (const double*)x, (const double*)gq,
                                   (const double*)d, mask, (double*)y, scratch, nullptr, s);
  if (dtype == PHASTB_F32)
    return h8_mech_apply_t<float>(v, make_vox_mat<float>(*m), slot, (const float*)x, (const float*)gq,
                                  (const float*)d, mask, (float*)y, scratch, nullptr, s);
  return PHASTB_ERR_ARG;
}

int phastb_h8_mech_diagonal(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                            int dtype, const void* gq, const void* d, void* diag, void* scratch, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !diag || !scratch) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(static_cast<char*>(scratch) +
                    align_up((dtype == PHASTB_F32 ? 4 : 8) * 24 * (size_t)v.n_elem));
  int st = red_ws_reset(ws, s);
  if (st) return st;
  if (dtype == PHASTB_F64)
    return h8_mech_diag_t<double>(v, make_vox_mat<double>(*m), slot, (const double*)gq, (const double*)d,
                                  (double*)diag, scratch, s);
  if (dtype == PHASTB_F32)
    return h8_mech_diag_t<float>(v, make_vox_mat<float>(*m), slot, (const float*)gq, (const float*)d,
                                 (float*)diag, scratch, s);
  return PHASTB_ERR_ARG;
}

int phastb_h8_stress_energy(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                            const double* x, const double* gq, const double* d, double* rE_host,
                            double* energy_host, void* scratch, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !scratch) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(static_cast<char*>(scratch) + align_up(8 * 24 * (size_t)v.n_elem));
  int st = red_ws_reset(ws, s);
  if (st) return st;
  { note_launch(); h8_mech_elem_kernel<double, true><<<grid_for(v.n_elem), kThreads, 0, s>>>(
      v, make_vox_mat<double>(*m), slot, x, gq, d, nullptr, nullptr, nullptr, ws, nullptr); }
  if ((st = last_launch_status())) return st;
  double o[7];
  if ((st = red_ws_fetch(ws, o, 7, s))) return st;
  if (rE_host)
    for (int k = 0; k < 6; ++k) rE_host[k] = o[k];
  if (energy_host) *energy_host = o[6];
  return PHASTB_OK;
}

int phastb_h8_driving_history(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* x, const double* H_prev, double* Y, double* H_out, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || (!Y && !H_out)) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  { note_launch(); h8_driving_kernel<<<grid_for(v.n_elem), kThreads, 0, (cudaStream_t)stream>>>(v, make_vox_mat<double>(*m), slot,
                                                                               x, H_prev, Y, H_out); }
  return last_launch_status();
}

int phastb_h8_damage_apply(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                           const double* d, const double* H, double scale, double* y, void* scratch, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !d || !y || !scratch) return PHASTB_ERR_ARG;
  return h8_damage_launch(make_vox_geom(*g), make_vox_mat<double>(*m), slot, 0, d, H, scale, y, nullptr, scratch,
                          nullptr, (cudaStream_t)stream);
}

int phastb_h8_damage_rhs_diag(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* H, double scale, double* rhs, double* diag, void* scratch,
                              void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !scratch) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  const VoxMat<double> mm = make_vox_mat<double>(*m);
  cudaStream_t s = (cudaStream_t)stream;
  int st = PHASTB_OK;
  if (rhs) {
    if (H)
      st = h8_damage_launch(v, mm, slot, 1, nullptr, H, scale, rhs, nullptr, scratch, nullptr, s);
    else
      st = cuda_status(cudaMemsetAsync(rhs, 0, sizeof(double) * v.n_red, s));
  }
  if (st) return st;
  if (diag) st = h8_damage_launch(v, mm, slot, 2, nullptr, H, scale, diag, nullptr, scratch, nullptr, s);
  return st;
}

}  // extern "C"

// ------------------------------------------------------------ accepted-increment record

namespace phastb {

// Sums of the record kernel: fracture energy by material slot, its local and
// gradient parts, the sum of element-mean damage and the damaged-element count.
constexpr int kRecSums = PHASTB_MAX_SLOTS + 4;
constexpr int kRecMax = 2;  // max H, max d

// Per element (solid3d/operator.py:1511-1545, staggered.py:1440-1455):
//   local    = Gc / (2 ell) d_e^T M d_e,  M = sum_q w N_q N_q^T
//   gradient = Gc ell / 2 d_e^T L d_e,    L = sum_q w grad N_q . grad N_q
// (by sum factorisation: d at the Gauss points and its face-difference gradients),
// the element-mean damage of the 8 corners, and the maxima of H and d.
__global__ void __launch_bounds__(kThreads) h8_record_kernel(VoxGeom g, VoxMat<double> m,
                                                             const uint8_t* __restrict__ slot,
                                                             const double* __restrict__ d,
                                                             const double* __restrict__ H, double threshold,
                                                             int pfczm, RedWs ws) {
  const double ihx = 1.0 / g.hx, ihy = 1.0 / g.hy, ihz = 1.0 / g.hz, w = g.w, ell = m.ell;
  constexpr double kPi = 3.14159265358979323846;
  double acc[kRecSums];
#pragma unroll
  for (int k = 0; k < kRecSums; ++k) acc[k] = 0.0;
  double mxH = -INFINITY, mxd = -INFINITY;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    double dd[8], dq[8];
#pragma unroll
    for (int L = 0; L < 8; ++L) dd[L] = __ldg(d + nd[L]);
    interp_sf(dd, dq);
    // AT2: int d^2; PF-CZM: int alpha(d) = int (2 d - d^2)
    double mloc = 0.0;
    if (pfczm) {
#pragma unroll
      for (int q = 0; q < 8; ++q) mloc += 2.0 * dq[q] - dq[q] * dq[q];
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q) mloc += dq[q] * dq[q];
    }
    double Dx[2][2], Dy[2][2], Dz[2][2];
    grad_sf(dd, ihx, ihy, ihz, Dx, Dy, Dz);
    double gl = 0.0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) gl += Dx[i][j] * Dx[i][j] + Dy[i][j] * Dy[i][j] + Dz[i][j] * Dz[i][j];
    // each face-difference gradient value holds at the two Gauss points along its own axis
    const int s = slot[e];
    const double Gc = m.Gc[s];
    const double local = pfczm ? Gc / (kPi * ell) * (w * mloc) : Gc / (2.0 * ell) * (w * mloc);
    const double grad = pfczm ? Gc * ell / kPi * (2.0 * w * gl) : 0.5 * Gc * ell * (2.0 * w * gl);
#pragma unroll
    for (int k = 0; k < PHASTB_MAX_SLOTS; ++k) acc[k] += (k == s) ? local + grad : 0.0;
    acc[PHASTB_MAX_SLOTS] += local;
    acc[PHASTB_MAX_SLOTS + 1] += grad;
    double dbar = 0.0;
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      dbar += dd[L];
      mxd = fmax(mxd, dd[L]);
    }
    dbar *= 0.125;
    acc[PHASTB_MAX_SLOTS + 2] += dbar;
    acc[PHASTB_MAX_SLOTS + 3] += dbar >= threshold ? 1.0 : 0.0;
    if (H) {
#pragma unroll
      for (int q = 0; q < 8; ++q) mxH = fmax(mxH, __ldg(H + 8 * (size_t)e + q));
    }
  }
  __shared__ double sh[32 * kRecSums];
  block_sum_multi<kRecSums>(acc, sh);
  const double bH = block_max(mxH, sh);
  const double bd = block_max(mxd, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kRecSums; ++k) ws.part[k * kMaxPartials + blockIdx.x] = acc[k];
    ws.part[kRecSums * kMaxPartials + blockIdx.x] = bH;
    ws.part[(kRecSums + 1) * kMaxPartials + blockIdx.x] = bd;
  }
  if (arrive_last(ws.counter)) {
    double f[kRecSums];
    fold_sum_multi<kRecSums>(ws.part, kMaxPartials, gridDim.x, f, sh);
    const double fH = fold_max(ws.part + kRecSums * kMaxPartials, gridDim.x, sh);
    const double fd = fold_max(ws.part + (kRecSums + 1) * kMaxPartials, gridDim.x, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < kRecSums; ++k) ws.out[k] = f[k];
      ws.out[kRecSums] = H ? fH : 0.0;
      ws.out[kRecSums + 1] = fd;
      *ws.counter = 0u;
    }
  }
}
static_assert(kRecSums + kRecMax <= kRedMaxK, "record reduction exceeds the reduction workspace");

// ||a - b||^2 over n entries (deterministic partials and fold).
__global__ void __launch_bounds__(kThreads) diff_norm2_kernel(int n, const double* __restrict__ a,
                                                              const double* __restrict__ b, RedWs ws) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double r = a[i] - b[i];
    v[0] += r * r;
  }
  reduce_multi<1>(v, ws);
}

// out = factor * x with out[idx] = value (idx < 0: no override).
__global__ void scale_set_kernel(int n, const double* __restrict__ x, double factor, int idx, double value,
                                 double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = i == idx ? value : factor * x[i];
}

}  // namespace phastb

extern "C" {

size_t phastb_h8_record_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  return 2 * red_ws_bytes();
}

int phastb_h8_increment_record(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                               const double* x, const double* d, const double* H, double threshold,
                               double* out_host, void* workspace, size_t workspace_bytes, void* stream) {
  return phastb_h8_increment_record_ex(g, m, slot, x, nullptr, d, H, threshold, nullptr, out_host, workspace,
                                       workspace_bytes, stream);
}

int phastb_h8_increment_record_ex(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                  const double* x, const double* gq, const double* d, const double* H,
                                  double threshold, const phastb_pfczm_law* law, double* out_host,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !d || !out_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_record_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws_s = red_ws(workspace);
  RedWs ws_d = red_ws(static_cast<char*>(workspace) + red_ws_bytes());
  int st;
  if ((st = red_ws_reset(ws_s, s)) || (st = red_ws_reset(ws_d, s))) return st;
  if (x) {
    { note_launch(); h8_mech_elem_kernel<double, true><<<grid_for(v.n_elem), kThreads, 0, s>>>(
        v, make_vox_mat<double>(*m), slot, x, gq, d, nullptr, nullptr, nullptr, ws_s, nullptr); }
    if ((st = last_launch_status())) return st;
  }
  { note_launch(); h8_record_kernel<<<grid_for(v.n_elem), kThreads, 0, s>>>(v, make_vox_mat<double>(*m), slot, d, H,
                                                                             threshold, law ? 1 : 0, ws_d); }
  if ((st = last_launch_status())) return st;
  if (x) {
    if ((st = cuda_status(cudaMemcpyAsync(out_host, x + 3 * (size_t)v.n_red, 6 * sizeof(double),
                                          cudaMemcpyDeviceToHost, s))))
      return st;
    if ((st = cuda_status(cudaMemcpyAsync(out_host + 6, ws_s.out, 7 * sizeof(double), cudaMemcpyDeviceToHost, s))))
      return st;
  } else {
    for (int k = 0; k < 13; ++k) out_host[k] = 0.0;
  }
  if ((st = cuda_status(cudaMemcpyAsync(out_host + 13, ws_d.out, (kRecSums + kRecMax) * sizeof(double),
                                        cudaMemcpyDeviceToHost, s))))
    return st;
  return cuda_status(cudaStreamSynchronize(s));
}

size_t phastb_h8_damage_residual_workspace_bytes(const phastb_voxel_grid* g) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  return h8_scratch_bytes(v, PHASTB_F64) + 2 * align_up(sizeof(double) * (size_t)v.n_red) + red_ws_bytes();
}

int phastb_h8_damage_residual_norm(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                                   const double* H, double scale, const double* d, double* norm_host,
                                   void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !d || !norm_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_h8_damage_residual_workspace_bytes(g)) return PHASTB_ERR_WORKSPACE;
  const VoxGeom v = make_vox_geom(*g);
  const VoxMat<double> mm = make_vox_mat<double>(*m);
  cudaStream_t s = (cudaStream_t)stream;
  char* p = static_cast<char*>(workspace);
  void* scratch = p;
  p += h8_scratch_bytes(v, PHASTB_F64);
  double* rhs = reinterpret_cast<double*>(p);
  double* Ad = reinterpret_cast<double*>(p + align_up(sizeof(double) * (size_t)v.n_red));
  RedWs ws = red_ws(p + 2 * align_up(sizeof(double) * (size_t)v.n_red));
  int st;
  if ((st = red_ws_reset(ws, s))) return st;
  if (H) {
    if ((st = h8_damage_launch(v, mm, slot, 1, nullptr, H, scale, rhs, nullptr, scratch, nullptr, s))) return st;
  } else if ((st = cuda_status(cudaMemsetAsync(rhs, 0, sizeof(double) * v.n_red, s)))) {
    return st;
  }
  if ((st = h8_damage_launch(v, mm, slot, 0, d, H, scale, Ad, nullptr, scratch, nullptr, s))) return st;
  { note_launch(); diff_norm2_kernel<<<grid_for(v.n_red), kThreads, 0, s>>>(v.n_red, rhs, Ad, ws); }
  if ((st = last_launch_status())) return st;
  double r2 = 0.0;
  if ((st = red_ws_fetch(ws, &r2, 1, s))) return st;
  *norm_host = sqrt(r2);
  return PHASTB_OK;
}

int phastb_scale_set(int n, const double* x, double factor, int index, double value, double* out, void* stream) {
  if (n < 0 || (n > 0 && (!x || !out)) || index >= n) return PHASTB_ERR_ARG;
  if (n == 0) return PHASTB_OK;
  { note_launch(); scale_set_kernel<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(n, x, factor, index, value,
                                                                                         out); }
  return last_launch_status();
}

}  // extern "C"

// ------------------------------------------------------------ allocation-free elastic action
//
// Some callers cannot allocate device memory at all: a host runtime bound
// through a thin FFI with no device-memory API of its own, or an application
// whose GPU memory is owned entirely by another framework's pool and must not
// see allocations it does not control.  For them the elastic action has a
// variant whose element scratch is a file-scope device array, sized for at most
// PHASTB_NOALLOC_MAX_VOXELS voxels and resident on every GPU that loads this
// library until the process exits.  All calls share that one array.

namespace phastb {

constexpr size_t ca256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kNoAllocBytes = ca256(24 * sizeof(double) * (size_t)PHASTB_NOALLOC_MAX_VOXELS) +
                                 ca256(sizeof(double) * kRedMaxK * kMaxPartials) + 256 +
                                 ca256(sizeof(double) * kRedMaxK);
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per
// device (the array's name is only a host-side handle, not a device address).
static int noalloc_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return PHASTB_ERR_CUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return PHASTB_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PHASTB_ERR_CUDA;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return PHASTB_OK;
}

}  // namespace phastb

extern "C" int phastb_h8_mech_apply_noalloc(const phastb_voxel_grid* g, const phastb_voxel_material* m,
                                            const uint8_t* slot, int dtype, const void* x, const void* gq,
                                            const void* d, const uint8_t* mask, void* y, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !y) return PHASTB_ERR_ARG;
  if (dtype != PHASTB_F64 && dtype != PHASTB_F32) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  if (v.n_elem > PHASTB_NOALLOC_MAX_VOXELS) return PHASTB_ERR_CAPACITY;
  void* scratch = nullptr;
  int st = noalloc_scratch(&scratch);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  // The array keeps the previous call's contents: the reduction ticket must start at zero.
  const size_t elem = dtype == PHASTB_F32 ? sizeof(float) : sizeof(double);
  RedWs ws = red_ws(static_cast<char*>(scratch) + align_up(24 * elem * (size_t)v.n_elem));
  if ((st = red_ws_reset(ws, s))) return st;
  if (dtype == PHASTB_F64)
    return h8_mech_apply_t<double>(v, make_vox_mat<double>(*m), slot, (const double*)x, (const double*)gq,
                                   (const double*)d, mask, (double*)y, scratch, nullptr, s);
  return h8_mech_apply_t<float>(v, make_vox_mat<float>(*m), slot, (const float*)x, (const float*)gq,
                                (const float*)d, mask, (float*)y, scratch, nullptr, s);
}
