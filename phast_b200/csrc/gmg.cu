// Geometric multigrid V-cycle preconditioner for the periodic voxel elastic
// operator (3 levels: n^3 -> (n/2)^3 -> (n/4)^3, Chebyshev smoothing).
//
// PhAST has no voxel multigrid (its 3D mechanics PCG is Jacobi only); the
// smoother and cycle follow its 2D AMG/GMG semantics (solvers/multigrid.py:
// Chebyshev bounds [lambda_max/30, 1.1 lambda_max] from power iteration
// :860-880 and :996-1035, V-cycle :534-576 and :1038-1089).
//
// * Coarse operators are rediscretised on voxels of twice the size.  Their
//   moduli live at the Gauss points: coarse Gauss point q of coarse voxel K sits
//   in the fine voxel 2K + q, and takes that fine voxel's mean (g lambda, g mu)
//   over its eight Gauss points.  The degradation g(d) of the fine level thus
//   carries down to every level (a damaged band stays soft on the coarse grids).
// * Transfers are trilinear interpolation P and its transpose R = P^T.
// * Smoothing: Chebyshev polynomial in D^-1 A of degree `deg` on the interval
//   [lambda_max/30, 1.1 lambda_max]; the same polynomial before and after the
//   coarse correction, so the V-cycle is a symmetric positive operator (a valid
//   CG preconditioner).  The coarsest level gets a degree-`deg_coarse` polynomial.
// * The coarse periodic operators are singular (rigid translations): the coarse
//   right-hand sides and corrections have their per-component mean removed.
// * On the fine level the pinned node and the macro-strain rows are held at
//   zero by the mask; the macro-strain rows of the preconditioned vector are a
//   Jacobi step (diagonal of the E block).
#include "engine.cuh"
#include "h8_kernels.cuh"
#include "h8_tile.cuh"

#include <cstdlib>
#include <utility>

#include <cmath>
#include <vector>

namespace phastb {

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
size_t h8_scratch_bytes(const VoxGeom& v, int dtype);

__device__ __forceinline__ void elem_ijk2(const VoxGeom& g, int e, int& ie, int& je, int& ke) {
  ie = e % g.nx;
  const int r = e / g.nx;
  je = r % g.ny;
  ke = r / g.ny;
}

// ------------------------------------------------------------ coefficients

// Fine Gauss-point moduli: (g lambda, g mu) per voxel and Gauss point -> mean per
// fine voxel, stored at the coarse Gauss point that voxel hosts.
template <typename T>
__global__ void gmg_coef_from_fine(VoxGeom f, VoxGeom c, VoxMat<T> m, const uint8_t* __restrict__ slot,
                                   const T* __restrict__ d, const T* __restrict__ gq, T* __restrict__ lam_c,
                                   T* __restrict__ mu_c) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < f.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk2(f, e, ie, je, ke);
    const int s = slot[e];
    T gm = T(1);
    if (gq) {
      // the mean of the given Gauss-point degradation
      gm = T(0);
#pragma unroll
      for (int q = 0; q < 8; ++q) gm += __ldg(gq + 8 * (size_t)e + q);
      gm *= T(0.125);
    } else if (d) {
      int nd[8];
      vox_corners(f, ie, je, ke, nd);
      T dd[8], dq[8];
#pragma unroll
      for (int L = 0; L < 8; ++L) dd[L] = __ldg(d + nd[L]);
      interp_sf(dd, dq);
      gm = T(0);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const T o = T(1) - dq[q];
        gm += (T(1) - m.kappa) * o * o + m.kappa;
      }
      gm *= T(0.125);
    }
    const int ec = (ie >> 1) + c.nx * ((je >> 1) + c.ny * (ke >> 1));
    const int q = (ie & 1) + 2 * (je & 1) + 4 * (ke & 1);
    lam_c[8 * (size_t)ec + q] = gm * m.lam[s];
    mu_c[8 * (size_t)ec + q] = gm * m.mu[s];
  }
}

template <typename T>
__global__ void gmg_coef_from_coarse(VoxGeom f, VoxGeom c, const T* __restrict__ lam_f, const T* __restrict__ mu_f,
                                     T* __restrict__ lam_c, T* __restrict__ mu_c) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < f.n_elem; e += gridDim.x * blockDim.x) {
    int ie, je, ke;
    elem_ijk2(f, e, ie, je, ke);
    T la = 0, mu = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      la += lam_f[8 * (size_t)e + q];
      mu += mu_f[8 * (size_t)e + q];
    }
    const int ec = (ie >> 1) + c.nx * ((je >> 1) + c.ny * (ke >> 1));
    const int q = (ie & 1) + 2 * (je & 1) + 4 * (ke & 1);
    lam_c[8 * (size_t)ec + q] = T(0.125) * la;
    mu_c[8 * (size_t)ec + q] = T(0.125) * mu;
  }
}

// ------------------------------------------------------------ coarse operator

// Element kernel of a coarse level: per-Gauss-point isotropic moduli, no macro
// strain.  MODE 0: action (24 values per voxel into scratch); MODE 1: diagonal.
template <typename T, int MODE>
__global__ void __launch_bounds__(kThreads) gmg_coarse_elem(VoxGeom g, const T* __restrict__ lam,
                                                            const T* __restrict__ mu, const T* __restrict__ x,
                                                            T* __restrict__ scratch, const int* guard) {
  if (guard && *guard == 0) return;
  const T ihx = T(1.0 / g.hx), ihy = T(1.0 / g.hy), ihz = T(1.0 / g.hz), w = T(g.w);
  const size_t E = (size_t)g.n_elem;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.n_elem; e += gridDim.x * blockDim.x) {
    T la[8], mq[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      la[q] = __ldg(lam + 8 * (size_t)e + q) * w;
      mq[q] = __ldg(mu + 8 * (size_t)e + q) * w;
    }
    if (MODE == 1) {
#pragma unroll
      for (int L = 0; L < 8; ++L) {
        const int ax = L & 1, ay = (L >> 1) & 1, az = L >> 2;
        T o0 = 0, o1 = 0, o2 = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int qx = q & 1, qy = (q >> 1) & 1, qz = q >> 2;
          const T nx_ = (qx == ax) ? T(kC1) : T(kC2);
          const T ny_ = (qy == ay) ? T(kC1) : T(kC2);
          const T nz_ = (qz == az) ? T(kC1) : T(kC2);
          const T gx = (ax ? ihx : -ihx) * ny_ * nz_;
          const T gy = (ay ? ihy : -ihy) * nx_ * nz_;
          const T gz = (az ? ihz : -ihz) * nx_ * ny_;
          const T l2m = la[q] + 2 * mq[q];
          o0 += l2m * gx * gx + mq[q] * (gy * gy + gz * gz);
          o1 += l2m * gy * gy + mq[q] * (gx * gx + gz * gz);
          o2 += l2m * gz * gz + mq[q] * (gx * gx + gy * gy);
        }
        scratch[(size_t)(L * 3 + 0) * E + e] = o0;
        scratch[(size_t)(L * 3 + 1) * E + e] = o1;
        scratch[(size_t)(L * 3 + 2) * E + e] = o2;
      }
      continue;
    }
    int ie, je, ke;
    elem_ijk2(g, e, ie, je, ke);
    int nd[8];
    vox_corners(g, ie, je, ke, nd);
    T D[3][3][2][2];
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
          const int q = qx + 2 * qy + 4 * qz;
          const T e0 = D[0][0][qz][qy], e1 = D[1][1][qz][qx], e2 = D[2][2][qy][qx];
          const T e3 = D[1][2][qy][qx] + D[2][1][qz][qx];
          const T e4 = D[0][2][qy][qx] + D[2][0][qz][qy];
          const T e5 = D[0][1][qz][qx] + D[1][0][qz][qy];
          const T lt = la[q] * (e0 + e1 + e2), m2 = 2 * mq[q];
          const T s0 = lt + m2 * e0, s1 = lt + m2 * e1, s2 = lt + m2 * e2;
          const T s3 = mq[q] * e3, s4 = mq[q] * e4, s5 = mq[q] * e5;
          P[0][0][qz][qy] += s0;
          P[0][1][qz][qx] += s5;
          P[0][2][qy][qx] += s4;
          P[1][0][qz][qy] += s5;
          P[1][1][qz][qx] += s1;
          P[1][2][qy][qx] += s3;
          P[2][0][qz][qy] += s4;
          P[2][1][qz][qx] += s3;
          P[2][2][qy][qx] += s2;
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T out[8];
      grad_sf_t(P[c][0], P[c][1], P[c][2], ihx, ihy, ihz, out);
#pragma unroll
      for (int L = 0; L < 8; ++L) scratch[(size_t)(L * 3 + c) * E + e] = out[L];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) gmg_gather3(VoxGeom g, const T* __restrict__ scratch,
                                                        T* __restrict__ y, const int* guard) {
  if (guard && *guard == 0) return;
  const size_t E = (size_t)g.n_elem;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n_red; n += gridDim.x * blockDim.x) {
    const int ir = n % g.rx;
    const int rem = n / g.rx;
    const int jr = rem % g.ry, kr = rem / g.ry;
    T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
    for (int L = 0; L < 8; ++L) {
      int ie = ir - (L & 1), je = jr - ((L >> 1) & 1), ke = kr - ((L >> 2) & 1);
      if (g.px) { if (ie < 0) ie += g.nx; } else if (ie < 0 || ie >= g.nx) continue;
      if (g.py) { if (je < 0) je += g.ny; } else if (je < 0 || je >= g.ny) continue;
      if (g.pz) { if (ke < 0) ke += g.nz; } else if (ke < 0 || ke >= g.nz) continue;
      const size_t e = (size_t)ie + (size_t)g.nx * ((size_t)je + (size_t)g.ny * ke);
      a0 += __ldg(scratch + (size_t)(L * 3 + 0) * E + e);
      a1 += __ldg(scratch + (size_t)(L * 3 + 1) * E + e);
      a2 += __ldg(scratch + (size_t)(L * 3 + 2) * E + e);
    }
    y[3 * (size_t)n + 0] = a0;
    y[3 * (size_t)n + 1] = a1;
    y[3 * (size_t)n + 2] = a2;
  }
}

// ------------------------------------------------------------ transfers

// Coarse node index along one axis -> fine node 2I (+ offsets), with periodic wrap.
__device__ __forceinline__ int fine_of(int i, int n_f, int periodic, bool& ok) {
  ok = true;
  if (periodic) {
    if (i < 0) i += n_f;
    if (i >= n_f) i -= n_f;
  } else if (i < 0 || i >= n_f + 1) {
    ok = false;
  }
  return i;
}

// r_c = R r_f = P^T r_f (full weighting).  The fine vector may carry a mask
// (rows held at zero are skipped).  With `sum_ws`, the kernel also sums the
// three components of r_c into sum_ws.out (the coarse level's mean, in the
// order and grouping of gmg_mean3 over the same grid, so the same bits).
template <typename T>
__global__ void gmg_restrict(VoxGeom f, VoxGeom c, const T* __restrict__ rf, const uint8_t* __restrict__ mask,
                             T* __restrict__ rc, RedWs sum_ws, int want_sum, const int* guard) {
  if (guard && *guard == 0) return;
  double acc[3] = {0, 0, 0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < c.n_red; n += gridDim.x * blockDim.x) {
    const int I = n % c.rx;
    const int rem = n / c.rx;
    const int J = rem % c.ry, K = rem / c.ry;
    T a0 = 0, a1 = 0, a2 = 0;
    for (int oz = -1; oz <= 1; ++oz) {
      bool okz;
      const int k = fine_of(2 * K + oz, f.nz, f.pz, okz);
      if (!okz) continue;
      const T wz = oz == 0 ? T(1) : T(0.5);
      for (int oy = -1; oy <= 1; ++oy) {
        bool oky;
        const int j = fine_of(2 * J + oy, f.ny, f.py, oky);
        if (!oky) continue;
        const T wy = oy == 0 ? T(1) : T(0.5);
        for (int ox = -1; ox <= 1; ++ox) {
          bool okx;
          const int i = fine_of(2 * I + ox, f.nx, f.px, okx);
          if (!okx) continue;
          const T wgt = (ox == 0 ? T(1) : T(0.5)) * wy * wz;
          const size_t fn = (size_t)i + (size_t)f.rx * ((size_t)j + (size_t)f.ry * k);
          const T v0 = (mask && mask[3 * fn + 0]) ? T(0) : rf[3 * fn + 0];
          const T v1 = (mask && mask[3 * fn + 1]) ? T(0) : rf[3 * fn + 1];
          const T v2 = (mask && mask[3 * fn + 2]) ? T(0) : rf[3 * fn + 2];
          a0 += wgt * v0;
          a1 += wgt * v1;
          a2 += wgt * v2;
        }
      }
    }
    rc[3 * (size_t)n + 0] = a0;
    rc[3 * (size_t)n + 1] = a1;
    rc[3 * (size_t)n + 2] = a2;
    acc[0] += double(a0);
    acc[1] += double(a1);
    acc[2] += double(a2);
  }
  if (want_sum) reduce_multi<3>(acc, sum_ws);
}

// x_f += P x_c (trilinear), masked rows untouched.  With csums, x_c still
// carries its mean: each coarse value is read as x_c - csums[comp] / c.n_red
// (what a separate subtraction pass would have stored, so the same bits).
template <typename T>
__global__ void gmg_prolong_add(VoxGeom f, VoxGeom c, const T* __restrict__ xc, const uint8_t* __restrict__ mask,
                                T* __restrict__ xf, const double* __restrict__ csums, const int* guard) {
  if (guard && *guard == 0) return;
  T m0 = T(0), m1 = T(0), m2 = T(0);
  if (csums) {
    m0 = T(csums[0] / c.n_red);
    m1 = T(csums[1] / c.n_red);
    m2 = T(csums[2] / c.n_red);
  }
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < f.n_red; n += gridDim.x * blockDim.x) {
    const int i = n % f.rx;
    const int rem = n / f.rx;
    const int j = rem % f.ry, k = rem / f.ry;
    int I[2], J[2], K[2];
    T wx[2], wy[2], wz[2];
    int cxn = 1, cyn = 1, czn = 1;
    I[0] = i >> 1;
    wx[0] = T(1);
    if (i & 1) {
      I[1] = I[0] + 1;
      if (c.px && I[1] >= c.nx) I[1] -= c.nx;
      wx[0] = wx[1] = T(0.5);
      cxn = 2;
    }
    J[0] = j >> 1;
    wy[0] = T(1);
    if (j & 1) {
      J[1] = J[0] + 1;
      if (c.py && J[1] >= c.ny) J[1] -= c.ny;
      wy[0] = wy[1] = T(0.5);
      cyn = 2;
    }
    K[0] = k >> 1;
    wz[0] = T(1);
    if (k & 1) {
      K[1] = K[0] + 1;
      if (c.pz && K[1] >= c.nz) K[1] -= c.nz;
      wz[0] = wz[1] = T(0.5);
      czn = 2;
    }
    T a0 = 0, a1 = 0, a2 = 0;
    for (int z = 0; z < czn; ++z)
      for (int yy = 0; yy < cyn; ++yy)
        for (int xx = 0; xx < cxn; ++xx) {
          const size_t cn = (size_t)I[xx] + (size_t)c.rx * ((size_t)J[yy] + (size_t)c.ry * K[z]);
          const T wgt = wx[xx] * wy[yy] * wz[z];
          T v0 = xc[3 * cn + 0], v1 = xc[3 * cn + 1], v2 = xc[3 * cn + 2];
          if (csums) {
            v0 -= m0;
            v1 -= m1;
            v2 -= m2;
          }
          a0 += wgt * v0;
          a1 += wgt * v1;
          a2 += wgt * v2;
        }
    if (!(mask && mask[3 * (size_t)n + 0])) xf[3 * (size_t)n + 0] += a0;
    if (!(mask && mask[3 * (size_t)n + 1])) xf[3 * (size_t)n + 1] += a1;
    if (!(mask && mask[3 * (size_t)n + 2])) xf[3 * (size_t)n + 2] += a2;
  }
}

// ------------------------------------------------------------ vector pieces

// per-component mean removal of a (3 n) nodal vector (coarse periodic levels)
template <typename T>
__global__ void __launch_bounds__(kThreads) gmg_mean3(int n, const T* __restrict__ x, RedWs ws, const int* guard) {
  if (guard && *guard == 0) return;
  double acc[3] = {0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    acc[0] += double(x[3 * (size_t)i]);
    acc[1] += double(x[3 * (size_t)i + 1]);
    acc[2] += double(x[3 * (size_t)i + 2]);
  }
  reduce_multi<3>(acc, ws);
}

// First Chebyshev step from the current x: res = b - Ax; d = invd * res / theta; x += d.
// With e_nu >= 0 (the fine level's last elementwise pass), the six E rows
// i = e_nu.. of x instead receive the preconditioner's Jacobi step on the
// macro-strain block, x_E = e_mask ? 0 : b_E / e_diag.
template <typename T>
__global__ void gmg_cheb_first_res(int n, const T* __restrict__ b, const T* __restrict__ Ax,
                                   const T* __restrict__ invd, T inv_theta, T* __restrict__ res, T* __restrict__ d,
                                   T* __restrict__ x, int e_nu, const T* __restrict__ e_diag,
                                   const uint8_t* __restrict__ e_mask, const int* guard) {
  if (guard && *guard == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T r = b[i] - Ax[i];
    res[i] = r;
    const T di = invd[i] * r * inv_theta;
    d[i] = di;
    if (e_nu >= 0 && i >= e_nu && i < e_nu + 6)
      x[i] = e_mask[i] ? T(0) : b[i] / e_diag[i];
    else
      x[i] = x[i] + di;
  }
}

// First step from x = 0 reading b directly: res = b; d = invd * b / theta; x = d.
// With bsums, b (a coarse nodal vector, 3 values per node) still carries its
// mean: b -= bsums[comp] / (n / 3) is applied here and stored back.
template <typename T>
__global__ void gmg_cheb_first_b(int n, T* __restrict__ b, const T* __restrict__ invd, T inv_theta,
                                 T* __restrict__ res, T* __restrict__ d, T* __restrict__ x,
                                 const double* __restrict__ bsums, const int* guard) {
  if (guard && *guard == 0) return;
  T m[3] = {T(0), T(0), T(0)};
  if (bsums) {
    const int nn = n / 3;
    m[0] = T(bsums[0] / nn);
    m[1] = T(bsums[1] / nn);
    m[2] = T(bsums[2] / nn);
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T bi = b[i];
    if (bsums) {
      bi -= m[i % 3];
      b[i] = bi;
    }
    res[i] = bi;
    const T di = invd[i] * bi * inv_theta;
    d[i] = di;
    x[i] = di;
  }
}

// res = b - A x
template <typename T>
__global__ void gmg_invert(int n, const T* __restrict__ diag, const uint8_t* __restrict__ mask, T* __restrict__ inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    inv[i] = (mask && mask[i]) ? T(0) : T(1) / diag[i];
}

// power iteration pieces: y = invd * A v; Rayleigh quotient (v, invd A v)_D = v.Av / v.Dv
template <typename T>
__global__ void __launch_bounds__(kThreads) gmg_power_dots(int n, const T* __restrict__ v, const T* __restrict__ Av,
                                                           const T* __restrict__ diag, const uint8_t* __restrict__ mask,
                                                           RedWs ws) {
  double acc[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (mask && mask[i]) continue;
    acc[0] += double(v[i]) * double(Av[i]);
    acc[1] += double(v[i]) * double(diag[i]) * double(v[i]);
  }
  reduce_multi<2>(acc, ws);
}

// v <- invd * Av / ||invd * Av||_D (normalisation by the D-norm from the device sums)
template <typename T>
__global__ void __launch_bounds__(kThreads) gmg_power_next(int n, const T* __restrict__ Av, const T* __restrict__ invd,
                                                           const T* __restrict__ diag, T* __restrict__ v, RedWs ws) {
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T z = invd[i] * Av[i];
    v[i] = z;
    acc[0] += double(z) * double(diag[i]) * double(z);
  }
  reduce_multi<1>(acc, ws);
}

template <typename T>
__global__ void gmg_scale(int n, const double* __restrict__ sum, T* __restrict__ v) {
  const double s = sum[0] > 0 ? 1.0 / sqrt(sum[0]) : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = T(double(v[i]) * s);
}

template <typename T>
__global__ void gmg_init_vec(int n, const uint8_t* __restrict__ mask, T* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    // deterministic, non-smooth start (hash of the index)
    unsigned h = (unsigned)i * 2654435761u;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    v[i] = (mask && mask[i]) ? T(0) : T(0.5 + (h & 0xffff) / 65536.0);
  }
}

// E block of the preconditioned vector: z_E = r_E / diag_E on free rows
template <typename Ts, typename Td>
__global__ void gmg_convert(int n, const Ts* __restrict__ a, Td* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = Td(a[i]);
}

// ======================================================================= host

template <typename T>
struct GmgLevel {
  VoxGeom g;
  int n;         // vector length (3 n_red on coarse levels, n_mech on the fine level)
  int pad_;      // no implicit padding: the struct is part of a graph-cache key
  T *lam, *mu;   // coarse levels: per-Gauss-point moduli
  T *diag, *invd, *x, *b, *res, *dvec, *Ad;
  double lmax;
};

template <typename T>
struct Gmg {
  int nlev, pad_;
  GmgLevel<T> lv[3];
  VoxMat<T> mat;
  const uint8_t* slot;
  const T* dfield;       // fine-level damage (T) for g(d), may be null
  const T* gfield;       // fine-level Gauss-point degradation (E,8), used instead of g(d) when set
  const uint8_t* mask;   // fine-level mask: fixed dofs + E rows
  const uint8_t* fmask;  // the solve's own fixed mask (for the E block)
  void* scratch;         // element scratch (fine size)
  RedWs rw;
  double* rsum;          // device copy of reduction results used by kernels
  int deg, deg_coarse;
  double safety;         // Chebyshev interval [lmax/30, safety * lmax]
  const int* guard;      // set per preconditioner call: the Krylov engine's "still iterating" flag
};

template <typename T>
static int coarse_apply(const Gmg<T>& M, const GmgLevel<T>& L, const T* x, T* y, cudaStream_t s) {
  TileArgs<T> a = tile_args<T>(L.g, 1);
  a.lam_q = L.lam;
  a.mu_q = L.mu;
  a.x = x;
  a.y = y;
  a.guard = M.guard;
  return h8_tile_launch<T>(a, M.mat, kCoefQP, kModeApply, s);
}

// One fused Chebyshev step on level l: res -= A din; dout = c1 din + c2 invd res; x += dout.
template <typename T>
static int level_cheb(const Gmg<T>& M, int l, const T* din, T* dout, double c1, double c2, cudaStream_t s) {
  const GmgLevel<T>& L = M.lv[l];
  TileArgs<T> a = tile_args<T>(L.g, l == 0 ? 0 : 1);
  a.x = din;
  a.res = L.res;
  a.invd = L.invd;
  a.xs = L.x;
  a.d_out = dout;
  a.c1 = c1;
  a.c2 = c2;
  a.guard = M.guard;
  if (l == 0) {
    a.slot = M.slot;
    a.d = M.dfield;
    a.gq = M.gfield;
    a.mask = M.mask;
    return h8_tile_launch<T>(a, M.mat, M.mat.iso ? kCoefIso : kCoefAniso, kModeCheb, s);
  }
  a.lam_q = L.lam;
  a.mu_q = L.mu;
  return h8_tile_launch<T>(a, M.mat, kCoefQP, kModeCheb, s);
}

// y = A x on level l.  The fine level's smoother masks the E rows, so its action
// skips them (kModeNodal: no E-row sums, y_E = 0, as the masked full action gives).
template <typename T>
static int level_apply(const Gmg<T>& M, int l, const T* x, T* y, cudaStream_t s) {
  if (l == 0) {
    TileArgs<T> a = tile_args<T>(M.lv[0].g, 0);
    a.slot = M.slot;
    a.d = M.dfield;
    a.gq = M.gfield;
    a.x = x;
    a.y = y;
    a.mask = M.mask;
    a.guard = M.guard;
    return h8_tile_launch<T>(a, M.mat, M.mat.iso ? kCoefIso : kCoefAniso, kModeNodal, s);
  }
  return coarse_apply<T>(M, M.lv[l], x, y, s);
}

// Mean removal on a fully periodic coarse level (its null space): sums the
// three components of x into M.rw.out and sets *sums to them; the next kernel
// that reads x subtracts sums / n_red (gmg_cheb_first_b, gmg_prolong_add), so
// no separate subtraction pass is launched.  *sums = nullptr when the level
// has no null space.  No other reduction into M.rw may run in between.
template <typename T>
static int pending_mean(const Gmg<T>& M, int l, const T* x, const double** sums, cudaStream_t s) {
  const GmgLevel<T>& L = M.lv[l];
  *sums = nullptr;
  if (!(L.g.px && L.g.py && L.g.pz)) return PHASTB_OK;
  const int nn = L.g.n_red;
  { note_launch(); gmg_mean3<T><<<grid_for(nn), kThreads, 0, s>>>(nn, x, M.rw, M.guard); }
  *sums = M.rw.out;
  return last_launch_status();
}

// Chebyshev smoothing of A x = b on level l; x starts at zero (from_zero) or at
// its current value.  With need_res, L.res holds b - A x on exit.
template <typename T>
static int chebyshev(const Gmg<T>& M, int l, int deg, bool from_zero, bool need_res, const double* bsums,
                     cudaStream_t s) {
  const GmgLevel<T>& L = M.lv[l];
  const int n = L.n, G = grid_for(n);
  int st;
  const double bmax = M.safety * L.lmax, amin = L.lmax / 30.0;
  const double theta = 0.5 * (bmax + amin), delta = 0.5 * (bmax - amin), sigma = theta / delta;
  if (from_zero) {
    { note_launch(); gmg_cheb_first_b<T><<<G, kThreads, 0, s>>>(n, L.b, L.invd, T(1.0 / theta), L.res, L.dvec, L.x, bsums, M.guard); }
  } else {
    if ((st = level_apply(M, l, L.x, L.Ad, s))) return st;
    // on the fine level this is the last pass over the E rows of x: it also
    // writes their Jacobi step (the V-cycle smooths the nodal block only)
    const int e_nu = l == 0 ? 3 * L.g.n_red : -1;
    { note_launch(); gmg_cheb_first_res<T><<<G, kThreads, 0, s>>>(n, L.b, L.Ad, L.invd, T(1.0 / theta), L.res, L.dvec, L.x, e_nu, L.diag, M.fmask, M.guard); }
  }
  // later steps ping-pong the direction between dvec and Ad
  T* cur = L.dvec;
  T* oth = L.Ad;
  double rho_old = 1.0 / sigma;
  for (int k = 1; k < deg; ++k) {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    if ((st = level_cheb(M, l, cur, oth, rho * rho_old, 2.0 * rho / delta, s))) return st;
    std::swap(cur, oth);
    rho_old = rho;
  }
  // res -= A d (a step with zero coefficients leaves x unchanged)
  if (need_res && (st = level_cheb(M, l, cur, oth, 0.0, 0.0, s))) return st;
  return last_launch_status();
}

// V-cycle from level l.  bsums: the pending mean of L.b, summed by the
// parent's restriction (nullptr on the fine level and on levels without a null
// space); on coarse levels the mean of the result L.x is left pending
// (*xsums, see pending_mean) for the parent's prolongation.
template <typename T>
static int vcycle(const Gmg<T>& M, int l, const double* bsums, const double** xsums, cudaStream_t s) {
  const GmgLevel<T>& L = M.lv[l];
  int st;
  *xsums = nullptr;
  if (l == M.nlev - 1) {
    if ((st = chebyshev(M, l, M.deg_coarse, true, false, bsums, s))) return st;
    return pending_mean(M, l, L.x, xsums, s);
  }
  if ((st = chebyshev(M, l, M.deg, true, true, bsums, s))) return st;
  const GmgLevel<T>& C = M.lv[l + 1];
  const int cper = C.g.px && C.g.py && C.g.pz;  // the coarse level has a null space: sum its mean
  { note_launch(); gmg_restrict<T><<<grid_for(C.g.n_red), kThreads, 0, s>>>(L.g, C.g, L.res, l == 0 ? M.mask : nullptr, C.b, M.rw, cper, M.guard); }
  const double* csums = nullptr;
  if ((st = vcycle(M, l + 1, cper ? M.rw.out : nullptr, &csums, s))) return st;
  { note_launch(); gmg_prolong_add<T><<<grid_for(L.g.n_red), kThreads, 0, s>>>(L.g, C.g, C.x, l == 0 ? M.mask : nullptr, L.x, csums, M.guard); }
  if ((st = chebyshev(M, l, M.deg, false, false, nullptr, s))) return st;
  if (l > 0 && (st = pending_mean(M, l, L.x, xsums, s))) return st;
  return last_launch_status();
}

template <typename T>
static int estimate_lmax(Gmg<T>& M, int l, int iters, cudaStream_t s) {
  GmgLevel<T>& L = M.lv[l];
  const int n = L.n, G = grid_for(n);
  const uint8_t* mk = l == 0 ? M.mask : nullptr;
  int st;
  { note_launch(); gmg_init_vec<T><<<G, kThreads, 0, s>>>(n, mk, L.dvec); }
  double lam = 0.0;
  for (int k = 0; k < iters; ++k) {
    if ((st = level_apply(M, l, L.dvec, L.Ad, s))) return st;
    if (k == iters - 1) {
      { note_launch(); gmg_power_dots<T><<<G, kThreads, 0, s>>>(n, L.dvec, L.Ad, L.diag, mk, M.rw); }
      double o[2];
      if ((st = red_ws_fetch(M.rw, o, 2, s))) return st;
      lam = o[1] > 0 ? o[0] / o[1] : 1.0;
    } else {
      { note_launch(); gmg_power_next<T><<<G, kThreads, 0, s>>>(n, L.Ad, L.invd, L.diag, L.dvec, M.rw); }
      { note_launch(); gmg_scale<T><<<G, kThreads, 0, s>>>(n, M.rw.out, L.dvec); }
    }
  }
  L.lmax = lam;
  return last_launch_status();
}

}  // namespace phastb

namespace phastb {

template <typename T>
static VoxGeom coarse_geom(const VoxGeom& f) {
  phastb_voxel_grid cg{f.nx / 2, f.ny / 2, f.nz / 2, f.px, f.py, f.pz, 2 * f.hx, 2 * f.hy, 2 * f.hz};
  return make_vox_geom(cg);
}

__global__ void gmg_fine_mask(int n_mech, int nu, const uint8_t* __restrict__ fixed, uint8_t* __restrict__ mask) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_mech; i += gridDim.x * blockDim.x)
    mask[i] = fixed[i] || i >= nu;
}

// Bytes of one GMG hierarchy in precision T for a fine grid f (levels >= 2).
template <typename T>
size_t gmg_hier_bytes(const VoxGeom& f, int levels) {
  size_t tot = 0;
  VoxGeom g = f;
  for (int l = 0; l < levels; ++l) {
    const size_t n = (l == 0) ? 3 * (size_t)g.n_red + 6 : 3 * (size_t)g.n_red;
    tot += 7 * align_up(sizeof(T) * n);
    if (l > 0) tot += 2 * align_up(sizeof(T) * 8 * (size_t)g.n_elem);
    g = coarse_geom<T>(g);
  }
  tot += align_up(3 * (size_t)f.n_red + 6);  // fine mask
  tot += h8_scratch_bytes(f, sizeof(T) == 4 ? PHASTB_F32 : PHASTB_F64);
  tot += red_ws_bytes();
  return tot;
}

template <typename T>
static char* gmg_carve(Gmg<T>& M, const VoxGeom& f, int levels, char* p) {
  M.nlev = levels;
  VoxGeom g = f;
  for (int l = 0; l < levels; ++l) {
    GmgLevel<T>& L = M.lv[l];
    L.g = g;
    L.n = (l == 0) ? 3 * g.n_red + 6 : 3 * g.n_red;
    const size_t vb = align_up(sizeof(T) * (size_t)L.n);
    T** vecs[7] = {&L.diag, &L.invd, &L.x, &L.b, &L.res, &L.dvec, &L.Ad};
    for (auto v : vecs) {
      *v = reinterpret_cast<T*>(p);
      p += vb;
    }
    if (l > 0) {
      const size_t cb = align_up(sizeof(T) * 8 * (size_t)g.n_elem);
      L.lam = reinterpret_cast<T*>(p);
      p += cb;
      L.mu = reinterpret_cast<T*>(p);
      p += cb;
    } else {
      L.lam = L.mu = nullptr;
    }
    L.lmax = 1.0;
    g = coarse_geom<T>(g);
  }
  M.mask = reinterpret_cast<uint8_t*>(p);
  p += align_up(3 * (size_t)f.n_red + 6);
  M.scratch = p;
  p += h8_scratch_bytes(f, sizeof(T) == 4 ? PHASTB_F32 : PHASTB_F64);
  M.rw = red_ws(p);
  p += red_ws_bytes();
  return p;
}

// Build the hierarchy for the current damage field (coefficients, diagonals,
// Chebyshev bounds).  `fixed` is the solve's mask over the n_mech rows.
template <typename T>
static int gmg_setup(Gmg<T>& M, const VoxMat<T>& mat, const uint8_t* slot, const T* dfield, const uint8_t* fixed,
                     int deg, int deg_coarse, int power_iters, double safety, double* lmax_io, cudaStream_t s,
                     const T* gfield = nullptr) {
  int st;
  M.safety = safety;
  M.mat = mat;
  M.slot = slot;
  M.dfield = dfield;
  M.gfield = gfield;
  M.fmask = fixed;
  M.deg = deg;
  M.deg_coarse = deg_coarse;
  const VoxGeom& f = M.lv[0].g;
  const int nu = 3 * f.n_red, nm = nu + 6;
  if ((st = cuda_status(cudaMemsetAsync(M.rw.counter, 0, sizeof(unsigned), s)))) return st;
  { note_launch(); gmg_fine_mask<<<grid_for(nm), kThreads, 0, s>>>(nm, nu, fixed, const_cast<uint8_t*>(M.mask)); }
  // fine diagonal (its E rows serve the Jacobi step of the E block)
  RedWs sw = red_ws(static_cast<char*>(M.scratch) + (h8_scratch_bytes(f, sizeof(T) == 4 ? PHASTB_F32 : PHASTB_F64) -
                                                      red_ws_bytes()));
  if ((st = cuda_status(cudaMemsetAsync(sw.counter, 0, sizeof(unsigned), s)))) return st;
  if ((st = h8_mech_diag_t<T>(f, mat, slot, gfield, dfield, M.lv[0].diag, M.scratch, s))) return st;
  { note_launch(); gmg_invert<T><<<grid_for(nm), kThreads, 0, s>>>(nm, M.lv[0].diag, M.mask, M.lv[0].invd); }
  for (int l = 1; l < M.nlev; ++l) {
    const GmgLevel<T>& F = M.lv[l - 1];
    GmgLevel<T>& C = M.lv[l];
    if (l == 1) {
      note_launch();
      gmg_coef_from_fine<T><<<grid_for(F.g.n_elem), kThreads, 0, s>>>(F.g, C.g, mat, slot, dfield, gfield, C.lam,
                                                                         C.mu);
    } else {
      note_launch();
      gmg_coef_from_coarse<T><<<grid_for(F.g.n_elem), kThreads, 0, s>>>(F.g, C.g, F.lam, F.mu, C.lam, C.mu);
    }
    { note_launch(); gmg_coarse_elem<T, 1><<<grid_for(C.g.n_elem), kThreads, 0, s>>>(C.g, C.lam, C.mu, nullptr, static_cast<T*>(M.scratch), nullptr); }
    { note_launch(); gmg_gather3<T><<<grid_for(C.g.n_red), kThreads, 0, s>>>(C.g, static_cast<T*>(M.scratch), C.diag, nullptr); }
    { note_launch(); gmg_invert<T><<<grid_for(C.n), kThreads, 0, s>>>(C.n, C.diag, nullptr, C.invd); }
  }
  if ((st = last_launch_status())) return st;
  const bool cached = lmax_io && lmax_io[0] > 0.0;
  for (int l = 0; l < M.nlev; ++l) {
    if (cached) {
      M.lv[l].lmax = lmax_io[l];
    } else {
      if ((st = estimate_lmax(M, l, power_iters, s))) return st;
      if (lmax_io) lmax_io[l] = M.lv[l].lmax;
    }
  }
  return PHASTB_OK;
}

// z = M^-1 r: V-cycle on the fluctuation rows, Jacobi on the free E rows.
template <typename T>
static int gmg_precond_apply(const void* ctx, const T* r, T* z, const int* guard, cudaStream_t s) {
  const Gmg<T>& M = *static_cast<const Gmg<T>*>(ctx);
  int st;
  // every V-cycle kernel turns into a no-op once the Krylov solve has converged
  Gmg<T> Mg = M;
  Mg.guard = guard;
  // the fine level reads its right-hand side from r (never written there: the
  // fine level has no pending mean) and builds its iterate directly in z
  Mg.lv[0].b = const_cast<T*>(r);
  Mg.lv[0].x = z;
  const double* xsums = nullptr;
  // the fine level's post-smoothing also writes z's E rows (gmg_cheb_first_res)
  if ((st = vcycle(Mg, 0, nullptr, &xsums, s))) return st;
  return last_launch_status();
}

template size_t gmg_hier_bytes<double>(const VoxGeom&, int);
template size_t gmg_hier_bytes<float>(const VoxGeom&, int);

// Per-cell setup pieces of the packed batch's multigrid (FP32): the Gauss-point moduli of a
// coarse level from the fine level's slots and damage (lam_f == nullptr) or from the next
// finer coarse level, and a coarse level's Jacobi diagonal (24-word element scratch).
int gmg_level_coefs_f32(const VoxGeom& f, const VoxGeom& c, const VoxMat<float>& m, const uint8_t* slot,
                        const float* d, const float* lam_f, const float* mu_f, float* lam_c, float* mu_c,
                        cudaStream_t s) {
  if (!lam_f)
    { note_launch(); gmg_coef_from_fine<float><<<grid_for(f.n_elem), kThreads, 0, s>>>(f, c, m, slot, d, nullptr, lam_c, mu_c); }
  else
    { note_launch(); gmg_coef_from_coarse<float><<<grid_for(f.n_elem), kThreads, 0, s>>>(f, c, lam_f, mu_f, lam_c, mu_c); }
  return last_launch_status();
}

int gmg_coarse_diag_f32(const VoxGeom& c, const float* lam, const float* mu, float* scratch, float* diag,
                        cudaStream_t s) {
  { note_launch(); gmg_coarse_elem<float, 1><<<grid_for(c.n_elem), kThreads, 0, s>>>(c, lam, mu, nullptr, scratch, nullptr); }
  { note_launch(); gmg_gather3<float><<<grid_for(c.n_red), kThreads, 0, s>>>(c, scratch, diag, nullptr); }
  return last_launch_status();
}

}  // namespace phastb

// ======================================================================= solve

namespace phastb {

bool valid_vox(const phastb_voxel_grid* g);
bool valid_mat(const phastb_voxel_material* m);

// Multigrid-preconditioned PCG looks at its state every gmg_check() iterations
// (one captured chunk); iterations past convergence cost only no-op launches.
// PHASTB_GMG_CHECK overrides the default interval.
static int gmg_check() {
  static const int v = [] {
    const char* e = std::getenv("PHASTB_GMG_CHECK");
    const int k = e ? std::atoi(e) : 0;
    return k >= 1 && k <= 64 ? k : 1;
  }();
  return v;
}

template <typename T>
struct MechOpT {
  VoxGeom v;
  VoxMat<T> m;
  const uint8_t* slot;
  const T* d;
  const uint8_t* mask;
  void* scratch;
  const T* gq;  // Gauss-point degradation (E,8) used instead of g(d) when set
};

template <typename T>
static int mech_op_t(const void* c, const T* x, T* y, const int* guard, cudaStream_t s) {
  const MechOpT<T>* k = static_cast<const MechOpT<T>*>(c);
  return h8_mech_apply_t<T>(k->v, k->m, k->slot, x, k->gq, k->d, k->mask, y, k->scratch, guard, s);
}

template <typename T>
static int mech_op_dot_t(const void* c, const T* x, T* y, const int* guard, cudaStream_t s) {
  const MechOpT<T>* k = static_cast<const MechOpT<T>*>(c);
  return h8_mech_apply_dot_t<T>(k->v, k->m, k->slot, x, k->gq, k->d, k->mask, y, k->scratch, guard, s);
}

__global__ void ex_setup_kernel(int n, const uint8_t* __restrict__ fixed, const double* __restrict__ vals,
                                const double* __restrict__ x0, double* __restrict__ xc, double* __restrict__ x0f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool f = fixed[i];
    xc[i] = f ? vals[i] : 0.0;
    x0f[i] = f ? 0.0 : (x0 ? x0[i] : 0.0);
  }
}

// b = where(free, rhs - image, 0) with ||b||^2
__global__ void __launch_bounds__(kThreads) ex_rhs_kernel(int n, const uint8_t* __restrict__ fixed,
                                                          const double* __restrict__ base, const double* image,
                                                          double* b, RedWs ws) {
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = fixed[i] ? 0.0 : (base ? base[i] : 0.0) - image[i];
    b[i] = v;
    acc[0] += v * v;
  }
  reduce_multi<1>(acc, ws);
}

__global__ void ex_where_kernel(int n, const uint8_t* __restrict__ fixed, const double* __restrict__ xc,
                                double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (fixed[i]) x[i] = xc[i];
}

__global__ void ex_add_kernel(int n, const float* __restrict__ dx, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += double(dx[i]);
}

__global__ void ex_invert_f(int n, const float* __restrict__ diag, const uint8_t* __restrict__ fixed,
                            float* __restrict__ inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    inv[i] = 1.0f / (fixed[i] ? 1.0f : diag[i]);
}

struct ExLayout {
  PcgWs<double> w64;
  PcgWs<float> w32;
  double *xc, *bf, *r64;
  double *d64, *x64;  // workspace copies of the damage field and the FP64 iterate (stable graph pointers)
  double* gq64;       // workspace copy of a Gauss-point degradation (E,8), when one is given
  float *d32, *r32, *dx32, *inv32, *gq32;
  void* scratch64;
  RedWs rw;
  Gmg<double> g64;
  Gmg<float> g32;
  size_t bytes;
};

static ExLayout ex_layout(const VoxGeom& v, const phastb_mech_opts& o, char* base, bool with_gq = false) {
  ExLayout L{};
  char* p = base;
  const int n = 3 * v.n_red + 6;
  auto take = [&](size_t b) {
    char* q = p;
    p += align_up(b);
    return q;
  };
  L.xc = reinterpret_cast<double*>(take(sizeof(double) * n));
  L.bf = reinterpret_cast<double*>(take(sizeof(double) * n));
  L.r64 = reinterpret_cast<double*>(take(sizeof(double) * n));
  L.d64 = reinterpret_cast<double*>(take(sizeof(double) * v.n_red));
  L.x64 = reinterpret_cast<double*>(take(sizeof(double) * n));
  L.scratch64 = take(h8_scratch_bytes(v, PHASTB_F64));
  L.rw = red_ws(take(red_ws_bytes()));
  if (with_gq) {
    L.gq64 = reinterpret_cast<double*>(take(sizeof(double) * 8 * (size_t)v.n_elem));
    if (o.mixed) L.gq32 = reinterpret_cast<float*>(take(sizeof(float) * 8 * (size_t)v.n_elem));
  }
  if (!o.mixed) {
    L.w64 = pcg_ws<double>(p, n);
    p += align_up(pcg_ws_bytes<double>(n));
    if (o.precond) p = gmg_carve<double>(L.g64, v, o.levels, p);
  } else {
    L.w32 = pcg_ws<float>(p, n);
    p += align_up(pcg_ws_bytes<float>(n));
    L.d32 = reinterpret_cast<float*>(take(sizeof(float) * v.n_red));
    L.r32 = reinterpret_cast<float*>(take(sizeof(float) * n));
    L.dx32 = reinterpret_cast<float*>(take(sizeof(float) * n));
    L.inv32 = reinterpret_cast<float*>(take(sizeof(float) * n));
    if (o.precond) {
      p = gmg_carve<float>(L.g32, v, o.levels, p);
    } else {
      L.g32.scratch = p;
      p += align_up(h8_scratch_bytes(v, PHASTB_F32));
    }
  }
  L.bytes = (size_t)(p - base) + 256;
  return L;
}

static bool opts_ok(const phastb_mech_opts* o, const VoxGeom& v) {
  if (!o) return false;
  if (o->precond != 0 && o->precond != 1) return false;
  if (o->mixed != 0 && o->mixed != 1) return false;
  if (o->precond == 1) {
    if (o->levels < 2 || o->levels > 3 || o->smooth_degree < 1 || o->coarse_degree < 1 || o->power_iters < 2 ||
        !(o->lmax_safety >= 1.0))
      return false;
    const int div = 1 << (o->levels - 1);
    auto ok = [&](int nn) { return nn % div == 0 && nn / div >= 2; };
    if (!ok(v.nx) || !ok(v.ny) || !ok(v.nz)) return false;
  }
  if (o->mixed == 1 && (!(o->inner_rtol > 0) || o->max_refine < 1)) return false;
  return true;
}

}  // namespace phastb

using namespace phastb;

extern "C" {

size_t phastb_h8_mech_solve_ex_workspace_bytes(const phastb_voxel_grid* g, const phastb_mech_opts* o) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  if (!opts_ok(o, v)) return 0;
  return ex_layout(v, *o, nullptr).bytes;
}

}  // extern "C"

// The extended solve with the damage field d (g(d) of AT2 in every operator) or, when gq is
// given, a Gauss-point degradation (E,8) in its place (the PF-CZM law's g).
static int mech_solve_ex_impl(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* d, const double* gq, const uint8_t* fixed, const double* fixed_values,
                              const double* x0, double rtol, double atol, int maxiter, int check_every,
                              const phastb_mech_opts* o, double* lmax_io, double* x_out, int* info, double* rinfo,
                              void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !fixed || !fixed_values || !x_out || maxiter < 1 ||
      check_every < 1 || !(rtol >= 0) || !(atol >= 0) || (rtol == 0 && atol == 0))
    return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  if (!opts_ok(o, v)) return PHASTB_ERR_ARG;
  ExLayout L = ex_layout(v, *o, static_cast<char*>(workspace), gq != nullptr);
  if (!workspace || workspace_bytes < L.bytes) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  const int n = 3 * v.n_red + 6, G = grid_for(n);
  const VoxMat<double> m64 = make_vox_mat<double>(*m);
  int st;
  if ((st = red_ws_reset(L.rw, s))) return st;
  RedWs sw = red_ws(static_cast<char*>(L.scratch64) + h8_scratch_bytes(v, PHASTB_F64) - red_ws_bytes());
  if ((st = red_ws_reset(sw, s))) return st;
  { note_launch(); ex_setup_kernel<<<G, kThreads, 0, s>>>(n, fixed, fixed_values, x0, L.xc, x_out); }
  // captured PCG chunks read the damage field and the iterate from the workspace
  if (d && (st = cuda_status(cudaMemcpyAsync(L.d64, d, sizeof(double) * v.n_red, cudaMemcpyDeviceToDevice, s))))
    return st;
  const double* dd = d ? L.d64 : nullptr;
  if (gq && (st = cuda_status(cudaMemcpyAsync(L.gq64, gq, sizeof(double) * 8 * (size_t)v.n_elem,
                                               cudaMemcpyDeviceToDevice, s))))
    return st;
  const double* gg = gq ? L.gq64 : nullptr;
  MechOpT<double> full{v, m64, slot, dd, nullptr, L.scratch64, gg};
  MechOpT<double> freeop{v, m64, slot, dd, fixed, L.scratch64, gg};
  if ((st = mech_op_t<double>(&full, L.xc, L.r64, nullptr, s))) return st;
  { note_launch(); ex_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, nullptr, L.r64, L.bf, L.rw); }
  if ((st = last_launch_status())) return st;
  double bn2;
  if ((st = red_ws_fetch(L.rw, &bn2, 1, s))) return st;
  const double bn = std::sqrt(bn2);
  if (rinfo) rinfo[0] = bn;
  if (!std::isfinite(bn)) return PHASTB_NONFINITE;
  if (bn == 0.0) {
    { note_launch(); ex_setup_kernel<<<G, kThreads, 0, s>>>(n, fixed, fixed_values, nullptr, L.xc, x_out); }
    { note_launch(); ex_where_kernel<<<G, kThreads, 0, s>>>(n, fixed, L.xc, x_out); }
    if (info) { info[0] = 0; info[1] = 1; }
    if (rinfo) rinfo[1] = 0.0;
    return last_launch_status();
  }
  const double thr = std::max(rtol * bn, atol);
  LinOp<double> A64{mech_op_t<double>, &freeop, sizeof(freeop), mech_op_dot_t<double>,
                    h8_apply_dot_slot(v, 8, L.scratch64)};
  if (!o->mixed) {
    // FP64 PCG with the FP64 V-cycle (precond = 1) or Jacobi (0)
    PcgResult pr{};
    if (o->precond) {
      if ((st = gmg_setup<double>(L.g64, m64, slot, dd, fixed, o->smooth_degree, o->coarse_degree, o->power_iters,
                                  o->lmax_safety, lmax_io, s, gg)))
        return st;
      Precond<double> M{gmg_precond_apply<double>, &L.g64, sizeof(L.g64)};
      if ((st = cuda_status(cudaMemcpyAsync(L.x64, x_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, s))))
        return st;
      if ((st = pcg_run<double>(A64, n, L.w64, L.bf, nullptr, &M, L.x64, thr, maxiter, gmg_check(), PCG_FREEZE, 0.0,
                                &pr, s)))
        return st;
    } else {
      if ((st = h8_mech_diag_t<double>(v, m64, slot, gg, dd, L.r64, L.scratch64, s))) return st;
      { note_launch(); gmg_invert<double><<<G, kThreads, 0, s>>>(n, L.r64, fixed, L.r64); }
      if ((st = cuda_status(cudaMemcpyAsync(L.x64, x_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, s))))
        return st;
      if ((st = pcg_run<double>(A64, n, L.w64, L.bf, L.r64, nullptr, L.x64, thr, maxiter, check_every, PCG_FREEZE,
                                0.0, &pr, s)))
        return st;
    }
    if ((st = cuda_status(cudaMemcpyAsync(x_out, L.x64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s))))
      return st;
    { note_launch(); ex_where_kernel<<<G, kThreads, 0, s>>>(n, fixed, L.xc, x_out); }
    if ((st = last_launch_status())) return st;
    if (info) { info[0] = pr.iterations; info[1] = pr.converged; }
    if (rinfo) rinfo[1] = pr.rnorm;
    if (pr.nonfinite) return PHASTB_NONFINITE;
    if (pr.breakdown) return PHASTB_BREAKDOWN;
    return pr.converged ? PHASTB_OK : PHASTB_NONCONVERGED;
  }
  // FP32 inner PCG (FP64 dot products) + FP64 iterative refinement
  const VoxMat<float> m32 = make_vox_mat<float>(*m);
  if (dd) { note_launch(); gmg_convert<double, float><<<grid_for(v.n_red), kThreads, 0, s>>>(v.n_red, dd, L.d32); }
  const float* d32 = dd ? L.d32 : nullptr;
  if (gg) {
    const long long ne8 = 8LL * v.n_elem;
    { note_launch(); gmg_convert<double, float><<<grid_for(ne8), kThreads, 0, s>>>((int)ne8, gg, L.gq32); }
  }
  const float* g32 = gg ? L.gq32 : nullptr;
  void* scratch32 = L.g32.scratch;
  if (o->precond) {
    if ((st = gmg_setup<float>(L.g32, m32, slot, d32, fixed, o->smooth_degree, o->coarse_degree, o->power_iters,
                                 o->lmax_safety, lmax_io, s, g32)))
      return st;
  } else {
    RedWs s32 = red_ws(static_cast<char*>(scratch32) + h8_scratch_bytes(v, PHASTB_F32) - red_ws_bytes());
    if ((st = red_ws_reset(s32, s))) return st;
    if ((st = h8_mech_diag_t<float>(v, m32, slot, g32, d32, L.inv32, scratch32, s))) return st;
    { note_launch(); ex_invert_f<<<G, kThreads, 0, s>>>(n, L.inv32, fixed, L.inv32); }
  }
  MechOpT<float> free32{v, m32, slot, d32, fixed, scratch32, g32};
  LinOp<float> A32{mech_op_t<float>, &free32, sizeof(free32), mech_op_dot_t<float>,
                   h8_apply_dot_slot(v, 4, scratch32)};
  Precond<float> M32{gmg_precond_apply<float>, &L.g32, sizeof(L.g32)};
  int total = 0, converged = 0;
  double rn = bn;
  for (int k = 0; k < o->max_refine && total < maxiter; ++k) {
    // FP64 residual; its norm is checked on the device by the inner solve's
    // start (no host round trip): when it already meets thr the inner solve
    // does nothing and reports outer_done
    if ((st = mech_op_t<double>(&freeop, x_out, L.r64, nullptr, s))) return st;
    { note_launch(); ex_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, L.bf, L.r64, L.r64, L.rw); }
    { note_launch(); gmg_convert<double, float><<<G, kThreads, 0, s>>>(n, L.r64, L.r32); }
    if ((st = cuda_status(cudaMemsetAsync(L.dx32, 0, sizeof(float) * n, s)))) return st;
    PcgResult pr{};
    PcgThreshold tin;
    tin.abs = 0.5 * thr;       // never resolve the correction far below the outer target
    tin.rel = o->inner_rtol;   // relative to the FP32 right-hand side, i.e. the FP64 residual
    tin.outer_rr = L.rw.out;
    tin.outer_thr = thr;
    if ((st = pcg_run_thr<float>(A32, n, L.w32, L.r32, o->precond ? nullptr : L.inv32, o->precond ? &M32 : nullptr,
                                 L.dx32, tin, maxiter - total, o->precond ? gmg_check() : check_every, PCG_FREEZE, &pr,
                                 s)))
      return st;
    rn = pr.outer_rnorm;
    if (pr.outer_done) {
      converged = 1;
      break;
    }
    if (!std::isfinite(rn) || pr.nonfinite) return PHASTB_NONFINITE;
    total += pr.iterations;
    if (pr.breakdown) return PHASTB_BREAKDOWN;
    { note_launch(); ex_add_kernel<<<G, kThreads, 0, s>>>(n, L.dx32, x_out); }
  }
  if (!converged) {
    // the last correction is not yet checked
    if ((st = mech_op_t<double>(&freeop, x_out, L.r64, nullptr, s))) return st;
    { note_launch(); ex_rhs_kernel<<<G, kThreads, 0, s>>>(n, fixed, L.bf, L.r64, L.r64, L.rw); }
    double rr;
    if ((st = red_ws_fetch(L.rw, &rr, 1, s))) return st;
    rn = std::sqrt(rr);
    converged = rn <= thr;
  }
  { note_launch(); ex_where_kernel<<<G, kThreads, 0, s>>>(n, fixed, L.xc, x_out); }
  if ((st = last_launch_status())) return st;
  if (info) { info[0] = total; info[1] = converged; }
  if (rinfo) rinfo[1] = rn;
  return converged ? PHASTB_OK : PHASTB_NONCONVERGED;
}

extern "C" {

int phastb_h8_mech_solve_ex(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                            const double* d, const uint8_t* fixed, const double* fixed_values, const double* x0,
                            double rtol, double atol, int maxiter, int check_every, const phastb_mech_opts* o,
                            double* lmax_io, double* x_out, int* info, double* rinfo, void* workspace,
                            size_t workspace_bytes, void* stream) {
  return mech_solve_ex_impl(g, m, slot, d, nullptr, fixed, fixed_values, x0, rtol, atol, maxiter, check_every, o,
                            lmax_io, x_out, info, rinfo, workspace, workspace_bytes, stream);
}

size_t phastb_h8_mech_solve_ex_g_workspace_bytes(const phastb_voxel_grid* g, const phastb_mech_opts* o) {
  if (!valid_vox(g)) return 0;
  const VoxGeom v = make_vox_geom(*g);
  if (!opts_ok(o, v)) return 0;
  return ex_layout(v, *o, nullptr, true).bytes;
}

int phastb_h8_mech_solve_ex_g(const phastb_voxel_grid* g, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* gq, const uint8_t* fixed, const double* fixed_values, const double* x0,
                              double rtol, double atol, int maxiter, int check_every, const phastb_mech_opts* o,
                              double* lmax_io, double* x_out, int* info, double* rinfo, void* workspace,
                              size_t workspace_bytes, void* stream) {
  if (!gq) return PHASTB_ERR_ARG;
  return mech_solve_ex_impl(g, m, slot, nullptr, gq, fixed, fixed_values, x0, rtol, atol, maxiter, check_every, o,
                            lmax_io, x_out, info, rinfo, workspace, workspace_bytes, stream);
}

}  // extern "C"
