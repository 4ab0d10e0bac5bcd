// Structured Q4 operators: strain, internal force, stiffness diagonal,
// psi+/history, AT2 damage operator, explicit central-difference step,
// energy and reaction sums.  C ABI in include/phastb.h.
#include "q4_kernels.cuh"
#include "reduce.cuh"

namespace phastb {

// ------------------------------------------------------------------ kernels

template <typename T, bool DEG>
__global__ void __launch_bounds__(kThreads) q4_force_kernel(Q4Tab<T> t, Mat2<T> m, int split,
                                                            const T* __restrict__ u,
                                                            const T* __restrict__ d,
                                                            T* __restrict__ f,
                                                            const uint8_t* __restrict__ mask,
                                                            const int* guard) {
  if (guard && *guard == 0) return;
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  T fx = 0, fy = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int a = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      T ux[4], uy[4], dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        load2(u, n[b], ux[b], uy[b]);
        dd[b] = DEG ? ld(d + n[b]) : T(0);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        T exx = 0, eyy = 0, gxy = 0, dq = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          exx += t.gx[q][b] * ux[b];
          eyy += t.gy[q][b] * uy[b];
          gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
          dq += t.N[q][b] * dd[b];
        }
        const T g = DEG ? degr(m, dq) : T(1);
        T sxx, syy, sxy;
        stress2(m, split, exx, eyy, gxy, g, sxx, syy, sxy);
        fx += (t.gx[q][a] * sxx + t.gy[q][a] * sxy) * t.w;
        fy += (t.gy[q][a] * syy + t.gx[q][a] * sxy) * t.w;
      }
    }
  if (mask) {
    const uchar2 mk = __ldg(reinterpret_cast<const uchar2*>(mask) + node);
    if (mk.x) fx = T(0);
    if (mk.y) fy = T(0);
  }
  typename Vec2<T>::type out;
  out.x = fx;
  out.y = fy;
  reinterpret_cast<typename Vec2<T>::type*>(f)[node] = out;
}

// Consistent tangent action y = d f_int(u, d)/du [du] (node-centric gather like
// q4_force_kernel): at every Gauss point the split's stress derivative at the strain of
// u, applied to the strain of du, with g(d) fixed.  Masked rows give zero.
__global__ void __launch_bounds__(kThreads) q4_tangent_kernel(Q4Tab<double> t, Mat2<double> m, int split,
                                                              const double* __restrict__ u,
                                                              const double* __restrict__ du,
                                                              const double* __restrict__ d,
                                                              double* __restrict__ f,
                                                              const uint8_t* __restrict__ mask,
                                                              const int* guard) {
  if (guard && *guard == 0) return;
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  double fx = 0, fy = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int a = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      double ux[4], uy[4], vx[4], vy[4], dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        load2(u, n[b], ux[b], uy[b]);
        load2(du, n[b], vx[b], vy[b]);
        dd[b] = d ? ld(d + n[b]) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double exx = 0, eyy = 0, gxy = 0, vxx = 0, vyy = 0, vxy = 0, dq = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          exx += t.gx[q][b] * ux[b];
          eyy += t.gy[q][b] * uy[b];
          gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
          vxx += t.gx[q][b] * vx[b];
          vyy += t.gy[q][b] * vy[b];
          vxy += t.gy[q][b] * vx[b] + t.gx[q][b] * vy[b];
          dq += t.N[q][b] * dd[b];
        }
        const double g = d ? degr(m, dq) : 1.0;
        double sxx, syy, sxy;
        dstress2(m, split, exx, eyy, gxy, vxx, vyy, vxy, g, sxx, syy, sxy);
        fx += (t.gx[q][a] * sxx + t.gy[q][a] * sxy) * t.w;
        fy += (t.gy[q][a] * syy + t.gx[q][a] * sxy) * t.w;
      }
    }
  if (mask) {
    const uchar2 mk = __ldg(reinterpret_cast<const uchar2*>(mask) + node);
    if (mk.x) fx = 0.0;
    if (mk.y) fy = 0.0;
  }
  reinterpret_cast<double2*>(f)[node] = make_double2(fx, fy);
}

// Transposed Gauss-point energy gradient of the undegraded (isotropic) energy:
//   f_n = sum_{e in n} sum_q wq[e][q] B_q^T sigma0(u)_q,   sigma0 = d psi0 / d eps,
// i.e. (d psi0_q / d u)^T wq: the adjoint of the history update H = max(H_prev, psi0(u))
// on the Gauss points where psi0 won (compute_psi_plus, fem_operators.py:951-990).
__global__ void __launch_bounds__(kThreads) q4_psi_grad_t_kernel(Q4Tab<double> t, Mat2<double> m,
                                                                  const double* __restrict__ u,
                                                                  const double* __restrict__ wq,
                                                                  double* __restrict__ f) {
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  double fx = 0, fy = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int a = q4_local(1 - di, 1 - dj);
      const int e = ej * t.nx + ei;
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      double ux[4], uy[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) load2(u, n[b], ux[b], uy[b]);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double exx = 0, eyy = 0, gxy = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          exx += t.gx[q][b] * ux[b];
          eyy += t.gy[q][b] * uy[b];
          gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
        }
        double sxx, syy, sxy;
        stress2(m, PHASTB_SPLIT_LINEAR, exx, eyy, gxy, 1.0, sxx, syy, sxy);
        const double wv = __ldg(wq + 4 * (size_t)e + q);
        fx += (t.gx[q][a] * sxx + t.gy[q][a] * sxy) * wv;
        fy += (t.gy[q][a] * syy + t.gx[q][a] * sxy) * wv;
      }
    }
  f[2 * (size_t)node] = fx;
  f[2 * (size_t)node + 1] = fy;
}

// Derivative of z . f_int(u, d) with respect to the nodal damage, isotropic split:
//   out_n = sum_{e in n} sum_q w g'(d_q) N_q(n) eps(z)_q . sigma0(u)_q,
// g(d) = (1-d)^2 (1-eta) + eta (internal_force, fem_operators.py:598-699; degradation,
// physics/material.py:497-529).
__global__ void __launch_bounds__(kThreads) q4_force_dd_t_kernel(Q4Tab<double> t, Mat2<double> m,
                                                                  const double* __restrict__ u,
                                                                  const double* __restrict__ z,
                                                                  const double* __restrict__ d,
                                                                  double* __restrict__ out) {
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  double acc = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int a = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      double ux[4], uy[4], zx[4], zy[4], dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        load2(u, n[b], ux[b], uy[b]);
        load2(z, n[b], zx[b], zy[b]);
        dd[b] = __ldg(d + n[b]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double exx = 0, eyy = 0, gxy = 0, zxx = 0, zyy = 0, zxy = 0, dq = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          exx += t.gx[q][b] * ux[b];
          eyy += t.gy[q][b] * uy[b];
          gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
          zxx += t.gx[q][b] * zx[b];
          zyy += t.gy[q][b] * zy[b];
          zxy += t.gy[q][b] * zx[b] + t.gx[q][b] * zy[b];
          dq += t.N[q][b] * dd[b];
        }
        double sxx, syy, sxy;
        stress2(m, PHASTB_SPLIT_LINEAR, exx, eyy, gxy, 1.0, sxx, syy, sxy);
        const double dg = -2.0 * (1.0 - dq) * (1.0 - m.eta);
        acc += t.w * dg * t.N[q][a] * (zxx * sxx + zyy * syy + zxy * sxy);
      }
    }
  out[node] = acc;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) q4_kdiag_kernel(Q4Tab<T> t, Mat2<T> m, const T* __restrict__ d,
                                                            T* __restrict__ diag) {
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  const T C00 = m.lam + 2 * m.mu, C22 = m.mu;
  T kx = 0, ky = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int a = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      T dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) dd[b] = d ? ld(d + n[b]) : T(0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        T g = T(1);
        if (d) {
          T dq = 0;
#pragma unroll
          for (int b = 0; b < 4; ++b) dq += t.N[q][b] * dd[b];
          g = degr(m, dq);
        }
        const T w = g * t.w, ax = t.gx[q][a], ay = t.gy[q][a];
        kx += w * (C00 * ax * ax + C22 * ay * ay);
        ky += w * (C00 * ay * ay + C22 * ax * ax);
      }
    }
  typename Vec2<T>::type out;
  out.x = kx;
  out.y = ky;
  reinterpret_cast<typename Vec2<T>::type*>(diag)[node] = out;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) q4_elem_kernel(Q4Tab<T> t, Mat2<T> m, const T* __restrict__ u,
                                                           T* exx_o, T* eyy_o, T* gxy_o,
                                                           const T* __restrict__ Hin, T* Hout, T* psi_o) {
  const int ne = t.nx * t.ny;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int n[4];
  q4_corners(e % t.nx, e / t.nx, t.nx, n);
  T ux[4], uy[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) load2(u, n[b], ux[b], uy[b]);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    T exx = 0, eyy = 0, gxy = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      exx += t.gx[q][b] * ux[b];
      eyy += t.gy[q][b] * uy[b];
      gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
    }
    const int k = 4 * e + q;
    if (exx_o) {
      exx_o[k] = exx;
      eyy_o[k] = eyy;
      gxy_o[k] = gxy;
    }
    if (Hout || psi_o) {
      const T p = psi2(m, m.psplit, exx, eyy, gxy);
      if (psi_o) psi_o[k] = p;
      if (Hout) {
        const T h = Hin ? Hin[k] : T(0);
        Hout[k] = p > h ? p : h;
      }
    }
  }
}

// AT2 damage operator (FP64): y_i = sum_e [gcl0_e lap_e + mass_e]_i.
__global__ void __launch_bounds__(kThreads) q4_damage_apply_kernel(Q4Tab<double> t, const double* __restrict__ d,
                                                                   const double* __restrict__ Hq, double rs,
                                                                   double rsh, const double* __restrict__ rsh_e,
                                                                   double gcl0, const double* __restrict__ gcl0_e,
                                                                   double* __restrict__ y, const int* guard,
                                                                   const uint8_t* __restrict__ mask) {
  if (guard && *guard == 0) return;
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  double lap_acc = 0, mass_acc = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int e = ej * t.nx + ei;
      const int a = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      double dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) dd[b] = __ldg(d + n[b]);
      const double2 h01 = __ldg(reinterpret_cast<const double2*>(Hq) + 2 * e);
      const double2 h23 = __ldg(reinterpret_cast<const double2*>(Hq) + 2 * e + 1);
      const double H[4] = {h01.x, h01.y, h23.x, h23.y};
      const double sh = rsh_e ? __ldg(rsh_e + e) : rsh;
      double lap = 0, mass = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double gdx = 0, gdy = 0, dq = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          gdx += t.gx[q][b] * dd[b];
          gdy += t.gy[q][b] * dd[b];
          dq += t.N[q][b] * dd[b];
        }
        lap += t.w * (t.gx[q][a] * gdx + t.gy[q][a] * gdy);
        mass += t.N[q][a] * ((rs * H[q] + sh) * dq * t.w);
      }
      lap_acc += (gcl0_e ? __ldg(gcl0_e + e) : gcl0) * lap;
      mass_acc += mass;
    }
  y[node] = (mask && mask[node]) ? 0.0 : lap_acc + mass_acc;
}

// Adjoint sensitivities of the AT2 damage system A(Gc, l0, H) d = b(H) for an
// adjoint field lam (one thread per element):
//   lKd_e = lam_e^T K_e d_e,  lMd_e = lam_e^T M_e d_e   (Gauss-point sums)
//   dL/dGc_e   = -(l0 lKd_e + lMd_e / l0)
//   dL/dH_{e,q} = 2 w lam_q (1 - d_q)   (db/dH minus dA/dH d at Gauss point q)
__global__ void __launch_bounds__(kThreads) q4_damage_adjoint_kernel(Q4Tab<double> t, const double* __restrict__ lam,
                                                                     const double* __restrict__ d, double l0,
                                                                     double* __restrict__ g_gc,
                                                                     double* __restrict__ g_h,
                                                                     double* __restrict__ lkd,
                                                                     double* __restrict__ lmd) {
  const int ne = t.nx * t.ny;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int ei = e % t.nx, ej = e / t.nx;
  int n[4];
  q4_corners(ei, ej, t.nx, n);
  double la[4], dd[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    la[b] = __ldg(lam + n[b]);
    dd[b] = __ldg(d + n[b]);
  }
  double kd = 0, md = 0, gh[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double lx = 0, ly = 0, lq = 0, dx = 0, dy = 0, dq = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      lx += t.gx[q][b] * la[b];
      ly += t.gy[q][b] * la[b];
      lq += t.N[q][b] * la[b];
      dx += t.gx[q][b] * dd[b];
      dy += t.gy[q][b] * dd[b];
      dq += t.N[q][b] * dd[b];
    }
    kd += t.w * (lx * dx + ly * dy);
    md += t.w * (lq * dq);
    gh[q] = 2.0 * t.w * lq * (1.0 - dq);
  }
  if (lkd) lkd[e] = kd;
  if (lmd) lmd[e] = md;
  if (g_gc) g_gc[e] = -(l0 * kd + md / l0);
  if (g_h) {
#pragma unroll
    for (int q = 0; q < 4; ++q) g_h[4 * (size_t)e + q] = gh[q];
  }
}

__global__ void __launch_bounds__(kThreads) q4_damage_prepare_kernel(Q4Tab<double> t, const double* __restrict__ Hq,
                                                                     double gco, const double* __restrict__ gco_e,
                                                                     double gcl0, const double* __restrict__ gcl0_e,
                                                                     double* __restrict__ b, double* __restrict__ minv) {
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  double bb = 0, dg = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int e = ej * t.nx + ei;
      const int a = q4_local(1 - di, 1 - dj);
      const double2 h01 = __ldg(reinterpret_cast<const double2*>(Hq) + 2 * e);
      const double2 h23 = __ldg(reinterpret_cast<const double2*>(Hq) + 2 * e + 1);
      const double H[4] = {h01.x, h01.y, h23.x, h23.y};
      const double ratio = gco_e ? __ldg(gco_e + e) : gco;
      double lapd = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        bb += t.N[q][a] * (2.0 * H[q] * t.w);
        lapd += t.w * (t.gx[q][a] * t.gx[q][a] + t.gy[q][a] * t.gy[q][a]);
        dg += (t.N[q][a] * t.N[q][a]) * ((2.0 * H[q] + ratio) * t.w);
      }
      dg += (gcl0_e ? __ldg(gcl0_e + e) : gcl0) * lapd;
    }
  b[node] = bb;
  minv[node] = 1.0 / (dg + 1e-30);
}

// Central-difference step fused with the internal force of the predicted
// displacement (ExplicitDynamics.predictor/corrector) and the optional history
// update of the element this node anchors (lower-left corner).
template <typename T>
__global__ void __launch_bounds__(kThreads) q4_explicit_kernel(
    Q4Tab<T> t, Mat2<T> m, T dt, const T* __restrict__ minv, const T* __restrict__ u, const T* __restrict__ v,
    const T* __restrict__ a, const T* __restrict__ d, const T* __restrict__ fext, const uint8_t* __restrict__ bcm,
    const T* __restrict__ bcv, T* __restrict__ uo, T* __restrict__ vo, T* __restrict__ ao,
    const T* __restrict__ Hin, T* __restrict__ Hout) {
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  const T hdt2 = T(0.5) * dt * dt;
  auto predict = [&](int nd, T& px, T& py) {
    T ux, uy, vx, vy, ax, ay;
    load2(u, nd, ux, uy);
    load2(v, nd, vx, vy);
    load2(a, nd, ax, ay);
    const uchar2 mk = __ldg(reinterpret_cast<const uchar2*>(bcm) + nd);
    px = mk.x ? ld(bcv + 2 * nd) : (ux + dt * vx) + hdt2 * ax;
    py = mk.y ? ld(bcv + 2 * nd + 1) : (uy + dt * vy) + hdt2 * ay;
  };
  T fx = 0, fy = 0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int al = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      T ux[4], uy[4], dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        predict(n[b], ux[b], uy[b]);
        dd[b] = ld(d + n[b]);
      }
      const bool own = (di == 1 && dj == 1) && Hout != nullptr;
      const int e = ej * t.nx + ei;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        T exx = 0, eyy = 0, gxy = 0, dq = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          exx += t.gx[q][b] * ux[b];
          eyy += t.gy[q][b] * uy[b];
          gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
          dq += t.N[q][b] * dd[b];
        }
        T sxx, syy, sxy;
        stress2(m, m.ssplit, exx, eyy, gxy, degr(m, dq), sxx, syy, sxy);
        fx += (t.gx[q][al] * sxx + t.gy[q][al] * sxy) * t.w;
        fy += (t.gy[q][al] * syy + t.gx[q][al] * sxy) * t.w;
        if (own) {
          const T p = psi2(m, m.psplit, exx, eyy, gxy);
          const T h = Hin ? Hin[4 * e + q] : T(0);
          Hout[4 * e + q] = p > h ? p : h;
        }
      }
    }
  T pux, puy, vx, vy, ax, ay, fex, fey;
  predict(node, pux, puy);
  load2(v, node, vx, vy);
  load2(a, node, ax, ay);
  load2(fext, node, fex, fey);
  const T mi = ld(minv + node);
  T anx = mi * (fex - fx), any = mi * (fey - fy);
  T vnx = vx + T(0.5) * dt * (ax + anx), vny = vy + T(0.5) * dt * (ay + any);
  const uchar2 mk = __ldg(reinterpret_cast<const uchar2*>(bcm) + node);
  if (mk.x) { anx = 0; vnx = 0; }
  if (mk.y) { any = 0; vny = 0; }
  typename Vec2<T>::type o;
  o.x = pux; o.y = puy;
  reinterpret_cast<typename Vec2<T>::type*>(uo)[node] = o;
  o.x = vnx; o.y = vny;
  reinterpret_cast<typename Vec2<T>::type*>(vo)[node] = o;
  o.x = anx; o.y = any;
  reinterpret_cast<typename Vec2<T>::type*>(ao)[node] = o;
}

// ---- reverse central-difference step (FP64), for splits whose stress is linear
// in u at fixed d (isotropic, linear).  The forward step on free dofs F is
//   u' = u + dt v + dt^2/2 a,  a' = Minv (f_ext - K(d) u'),  v' = v + dt/2 (a + a'),
// and u' = bc, a' = v' = 0 on the Dirichlet dofs.  With output adjoints
// (ub', vb', ab'):  s = F Minv (ab' + dt/2 vb');  t = ub' - K(d) s;
//   ub = F t,  vb = F (vb' + dt t),  ab = F (dt/2 vb' + dt^2/2 t),  f_ext_b += s,
//   d_b += -sum_q w g'(d_q) N_q eps(s)_q . C eps(u')_q.
__global__ void __launch_bounds__(kThreads) q4_adj_s_kernel(int n2, double dt, const double* __restrict__ minv,
                                                            const uint8_t* __restrict__ bcm,
                                                            const double* __restrict__ vb,
                                                            const double* __restrict__ ab, double* __restrict__ sv,
                                                            double* __restrict__ fb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    const double v = bcm[i] ? 0.0 : minv[i >> 1] * (ab[i] + 0.5 * dt * vb[i]);
    sv[i] = v;
    if (fb) fb[i] += v;
  }
}

__global__ void __launch_bounds__(kThreads) q4_adj_combine_kernel(int n2, double dt, const uint8_t* __restrict__ bcm,
                                                                  const double* __restrict__ ub,
                                                                  const double* __restrict__ vb,
                                                                  const double* __restrict__ Ks,
                                                                  double* __restrict__ ub_out,
                                                                  double* __restrict__ vb_out,
                                                                  double* __restrict__ ab_out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    const bool f = bcm[i] != 0;
    const double t = ub[i] - Ks[i], vbi = vb[i];
    ub_out[i] = f ? 0.0 : t;
    vb_out[i] = f ? 0.0 : vbi + dt * t;
    ab_out[i] = f ? 0.0 : 0.5 * dt * vbi + 0.5 * dt * dt * t;
  }
}

// d_b[node] += -sum over its elements and Gauss points of w g'(d_q) N_q[node] eps(s):C eps(u')
__global__ void __launch_bounds__(kThreads) q4_adj_dgrad_kernel(Q4Tab<double> t, Mat2<double> m,
                                                                const double* __restrict__ un,
                                                                const double* __restrict__ sv,
                                                                const double* __restrict__ d,
                                                                double* __restrict__ db) {
  const int nn = (t.nx + 1) * (t.ny + 1);
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const int i = node % (t.nx + 1), j = node / (t.nx + 1);
  double acc = 0.0;
#pragma unroll
  for (int dj = 0; dj < 2; ++dj)
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const int ei = i - 1 + di, ej = j - 1 + dj;
      if (ei < 0 || ei >= t.nx || ej < 0 || ej >= t.ny) continue;
      const int al = q4_local(1 - di, 1 - dj);
      int n[4];
      q4_corners(ei, ej, t.nx, n);
      double ux[4], uy[4], sx[4], sy[4], dd[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        ux[b] = un[2 * n[b]];
        uy[b] = un[2 * n[b] + 1];
        sx[b] = sv[2 * n[b]];
        sy[b] = sv[2 * n[b] + 1];
        dd[b] = d[n[b]];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double exx = 0, eyy = 0, gxy = 0, fxx = 0, fyy = 0, fxy = 0, dq = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          exx += t.gx[q][b] * ux[b];
          eyy += t.gy[q][b] * uy[b];
          gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
          fxx += t.gx[q][b] * sx[b];
          fyy += t.gy[q][b] * sy[b];
          fxy += t.gy[q][b] * sx[b] + t.gx[q][b] * sy[b];
          dq += t.N[q][b] * dd[b];
        }
        double sxx, syy, sxy;
        stress2(m, PHASTB_SPLIT_LINEAR, exx, eyy, gxy, 1.0, sxx, syy, sxy);
        const double gp = -2.0 * (1.0 - dq) * (1.0 - m.eta);  // dg/dd
        acc -= t.w * gp * t.N[q][al] * (fxx * sxx + fyy * syy + fxy * sxy);
      }
    }
  db[node] += acc;
}

// Energy sums: elastic sum_q (g psi+ + psi-) w, d^T M d, d^T K d, sum |v|^2 M.
__global__ void __launch_bounds__(kThreads) q4_energy_kernel(Q4Tab<double> t, Mat2<double> m,
                                                             const double* __restrict__ u,
                                                             const double* __restrict__ d,
                                                             const double* __restrict__ v, RedWs ws) {
  const int ne = t.nx * t.ny, nn = (t.nx + 1) * (t.ny + 1);
  double acc[4] = {0, 0, 0, 0};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    int n[4];
    q4_corners(e % t.nx, e / t.nx, t.nx, n);
    double ux[4], uy[4], dd[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      load2(u, n[b], ux[b], uy[b]);
      dd[b] = __ldg(d + n[b]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double exx = 0, eyy = 0, gxy = 0, dq = 0, gdx = 0, gdy = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        exx += t.gx[q][b] * ux[b];
        eyy += t.gy[q][b] * uy[b];
        gxy += t.gy[q][b] * ux[b] + t.gx[q][b] * uy[b];
        dq += t.N[q][b] * dd[b];
        gdx += t.gx[q][b] * dd[b];
        gdy += t.gy[q][b] * dd[b];
      }
      const double pp = psi2(m, m.psplit, exx, eyy, gxy);
      const double pf = psi2(m, PHASTB_SPLIT_ISOTROPIC, exx, eyy, gxy);
      acc[0] += (degr(m, dq) * pp + (pf - pp)) * t.w;
      acc[1] += t.w * dq * dq;
      acc[2] += t.w * (gdx * gdx + gdy * gdy);
    }
  }
  if (v) {
    for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < nn; nd += gridDim.x * blockDim.x) {
      const int i = nd % (t.nx + 1), j = nd / (t.nx + 1);
      const int cnt = (1 + (i > 0 && i < t.nx)) * (1 + (j > 0 && j < t.ny));
      double vx, vy;
      load2(v, nd, vx, vy);
      acc[3] += (vx * vx + vy * vy) * (cnt * t.w);
    }
  }
  reduce_multi<4>(acc, ws);
}

__global__ void __launch_bounds__(kThreads) q4_select_sum_kernel(const double* __restrict__ f,
                                                                 const int64_t* __restrict__ nodes, int n,
                                                                 int comp, const double* __restrict__ fext,
                                                                 RedWs ws) {
  double acc[1] = {0};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int64_t nd = nodes[k];
    acc[0] += f[2 * nd + comp] - (fext ? fext[2 * nd + comp] : 0.0);
  }
  reduce_multi<1>(acc, ws);
}

// ------------------------------------------------------------------ helpers

static bool valid_grid(const phastb_q4_grid* g) {
  return g && g->nx >= 1 && g->ny >= 1 && g->hx > 0 && g->hy > 0 &&
         (long long)(g->nx + 1) * (g->ny + 1) < (1LL << 30);
}

template <typename T>
static int launch_force(const phastb_q4_grid* g, const phastb_q4_material* m, const void* u, const void* d,
                        void* f, cudaStream_t s, const uint8_t* mask = nullptr, const int* guard = nullptr) {
  const Q4Tab<T> t = make_q4_tab<T>(*g);
  const Mat2<T> mm = make_mat2<T>(*m);
  const int nn = (g->nx + 1) * (g->ny + 1);
  if (d)
    { note_launch(); q4_force_kernel<T, true><<<grid_full(nn), kThreads, 0, s>>>(t, mm, m->stress_split, (const T*)u, (const T*)d,
                                                                (T*)f, mask, guard); }
  else
    { note_launch(); q4_force_kernel<T, false><<<grid_full(nn), kThreads, 0, s>>>(t, mm, PHASTB_SPLIT_LINEAR, (const T*)u, nullptr,
                                                                 (T*)f, mask, guard); }
  return last_launch_status();
}

int q4_damage_apply_launch(const phastb_q4_grid* g, const double* d, const double* Hq, double rs, double rsh,
                           const double* rsh_e, double gcl0, const double* gcl0_e, double* y, const int* guard,
                           cudaStream_t s, const uint8_t* mask) {
  const Q4Tab<double> t = make_q4_tab<double>(*g);
  const int nn = (g->nx + 1) * (g->ny + 1);
  { note_launch(); q4_damage_apply_kernel<<<grid_full(nn), kThreads, 0, s>>>(t, d, Hq, rs, rsh, rsh_e, gcl0, gcl0_e, y, guard, mask); }
  return last_launch_status();
}

int q4_damage_adjoint_launch(const phastb_q4_grid* g, const double* lam, const double* d, double l0, double* g_gc,
                             double* g_h, double* lkd, double* lmd, cudaStream_t s) {
  const Q4Tab<double> t = make_q4_tab<double>(*g);
  const int ne = g->nx * g->ny;
  { note_launch(); q4_damage_adjoint_kernel<<<grid_full(ne), kThreads, 0, s>>>(t, lam, d, l0, g_gc, g_h, lkd, lmd); }
  return last_launch_status();
}

int q4_force_launch(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* d,
                    double* f, const uint8_t* mask, const int* guard, cudaStream_t s) {
  return launch_force<double>(g, m, u, d, f, s, mask, guard);
}

int q4_tangent_launch(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* du,
                      const double* d, double* f, const uint8_t* mask, const int* guard, cudaStream_t s) {
  const Q4Tab<double> t = make_q4_tab<double>(*g);
  const Mat2<double> mm = make_mat2<double>(*m);
  const int nn = (g->nx + 1) * (g->ny + 1);
  { note_launch(); q4_tangent_kernel<<<grid_full(nn), kThreads, 0, s>>>(t, mm, m->stress_split, u, du, d, f, mask, guard); }
  return last_launch_status();
}

}  // namespace phastb

using namespace phastb;

// ------------------------------------------------------------------ C ABI

extern "C" {

int phastb_q4_strain(const phastb_q4_grid* g, int dtype, const void* u, void* exx, void* eyy, void* gxy,
                     void* stream) {
  if (!valid_grid(g) || !u || !exx || !eyy || !gxy) return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int ne = g->nx * g->ny;
  phastb_q4_material m{};
  if (dtype == PHASTB_F64) {
    { note_launch(); q4_elem_kernel<double><<<grid_full(ne), kThreads, 0, s>>>(make_q4_tab<double>(*g), make_mat2<double>(m),
                                                             (const double*)u, (double*)exx, (double*)eyy,
                                                             (double*)gxy, nullptr, nullptr, nullptr); }
  } else if (dtype == PHASTB_F32) {
    { note_launch(); q4_elem_kernel<float><<<grid_full(ne), kThreads, 0, s>>>(make_q4_tab<float>(*g), make_mat2<float>(m),
                                                            (const float*)u, (float*)exx, (float*)eyy, (float*)gxy,
                                                            nullptr, nullptr, nullptr); }
  } else {
    return PHASTB_ERR_ARG;
  }
  return last_launch_status();
}

int phastb_q4_internal_force(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype, const void* u,
                             const void* d, void* f, void* stream) {
  if (!valid_grid(g) || !m || !u || !f) return PHASTB_ERR_ARG;
  if (dtype == PHASTB_F64) return launch_force<double>(g, m, u, d, f, (cudaStream_t)stream);
  if (dtype == PHASTB_F32) return launch_force<float>(g, m, u, d, f, (cudaStream_t)stream);
  return PHASTB_ERR_ARG;
}

int phastb_q4_tangent_apply(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u,
                            const double* du, const double* d, double* y, void* stream) {
  if (!valid_grid(g) || !m || !u || !du || !y) return PHASTB_ERR_ARG;
  return q4_tangent_launch(g, m, u, du, d, y, nullptr, nullptr, (cudaStream_t)stream);
}

int phastb_q4_psi_grad_t(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* wq,
                         double* f, void* stream) {
  if (!valid_grid(g) || !m || !u || !wq || !f) return PHASTB_ERR_ARG;
  if (m->psi_split != PHASTB_SPLIT_ISOTROPIC && m->psi_split != PHASTB_SPLIT_LINEAR) return PHASTB_UNSUPPORTED;
  const int nn = (g->nx + 1) * (g->ny + 1);
  { note_launch(); q4_psi_grad_t_kernel<<<grid_full(nn), kThreads, 0, (cudaStream_t)stream>>>(
      make_q4_tab<double>(*g), make_mat2<double>(*m), u, wq, f); }
  return last_launch_status();
}

int phastb_q4_force_dd_t(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* z,
                         const double* d, double* out, void* stream) {
  if (!valid_grid(g) || !m || !u || !z || !d || !out) return PHASTB_ERR_ARG;
  if (m->stress_split != PHASTB_SPLIT_ISOTROPIC && m->stress_split != PHASTB_SPLIT_LINEAR) return PHASTB_UNSUPPORTED;
  const int nn = (g->nx + 1) * (g->ny + 1);
  { note_launch(); q4_force_dd_t_kernel<<<grid_full(nn), kThreads, 0, (cudaStream_t)stream>>>(
      make_q4_tab<double>(*g), make_mat2<double>(*m), u, z, d, out); }
  return last_launch_status();
}

int phastb_q4_stiffness_diagonal(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype, const void* d,
                                 void* diag, void* stream) {
  if (!valid_grid(g) || !m || !diag) return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int nn = (g->nx + 1) * (g->ny + 1);
  if (dtype == PHASTB_F64)
    { note_launch(); q4_kdiag_kernel<double><<<grid_full(nn), kThreads, 0, s>>>(make_q4_tab<double>(*g), make_mat2<double>(*m),
                                                              (const double*)d, (double*)diag); }
  else if (dtype == PHASTB_F32)
    { note_launch(); q4_kdiag_kernel<float><<<grid_full(nn), kThreads, 0, s>>>(make_q4_tab<float>(*g), make_mat2<float>(*m),
                                                             (const float*)d, (float*)diag); }
  else
    return PHASTB_ERR_ARG;
  return last_launch_status();
}

int phastb_q4_psi_history(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype, const void* u,
                          const void* H_in, void* H_out, void* psi, void* stream) {
  if (!valid_grid(g) || !m || !u) return PHASTB_ERR_ARG;
  if (!H_out && !psi) return PHASTB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int ne = g->nx * g->ny;
  if (dtype == PHASTB_F64)
    { note_launch(); q4_elem_kernel<double><<<grid_full(ne), kThreads, 0, s>>>(make_q4_tab<double>(*g), make_mat2<double>(*m),
                                                             (const double*)u, nullptr, nullptr, nullptr,
                                                             (const double*)H_in, (double*)H_out, (double*)psi); }
  else if (dtype == PHASTB_F32)
    { note_launch(); q4_elem_kernel<float><<<grid_full(ne), kThreads, 0, s>>>(make_q4_tab<float>(*g), make_mat2<float>(*m),
                                                            (const float*)u, nullptr, nullptr, nullptr,
                                                            (const float*)H_in, (float*)H_out, (float*)psi); }
  else
    return PHASTB_ERR_ARG;
  return last_launch_status();
}

int phastb_q4_damage_apply(const phastb_q4_grid* g, const double* d, const double* Hq, double rd_scale,
                           double rd_shift, const double* rd_shift_e, double gcl0, const double* gcl0_e, double* y,
                           void* stream) {
  if (!valid_grid(g) || !d || !Hq || !y) return PHASTB_ERR_ARG;
  return q4_damage_apply_launch(g, d, Hq, rd_scale, rd_shift, rd_shift_e, gcl0, gcl0_e, y, nullptr,
                                (cudaStream_t)stream, nullptr);
}

int phastb_q4_damage_prepare(const phastb_q4_grid* g, const double* Hq, double gc_over_l0,
                             const double* gc_over_l0_e, double gcl0, const double* gcl0_e, double* b,
                             double* m_inv, void* stream) {
  if (!valid_grid(g) || !Hq || !b || !m_inv) return PHASTB_ERR_ARG;
  const int nn = (g->nx + 1) * (g->ny + 1);
  { note_launch(); q4_damage_prepare_kernel<<<grid_full(nn), kThreads, 0, (cudaStream_t)stream>>>(
      make_q4_tab<double>(*g), Hq, gc_over_l0, gc_over_l0_e, gcl0, gcl0_e, b, m_inv); }
  return last_launch_status();
}

int phastb_q4_explicit_step(const phastb_q4_grid* g, const phastb_q4_material* m, int dtype, double dt,
                            const void* m_inv, const void* u, const void* v, const void* a, const void* d,
                            const void* f_ext, const uint8_t* bc_mask, const void* bc_vals, void* u_out,
                            void* v_out, void* a_out, const void* H_in, void* H_out, void* stream) {
  if (!valid_grid(g) || !m || !m_inv || !u || !v || !a || !d || !f_ext || !bc_mask || !bc_vals || !u_out ||
      !v_out || !a_out)
    return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int nn = (g->nx + 1) * (g->ny + 1);
  if (dtype == PHASTB_F64)
    { note_launch(); q4_explicit_kernel<double><<<grid_full(nn), kThreads, 0, s>>>(
        make_q4_tab<double>(*g), make_mat2<double>(*m), dt, (const double*)m_inv, (const double*)u,
        (const double*)v, (const double*)a, (const double*)d, (const double*)f_ext, bc_mask,
        (const double*)bc_vals, (double*)u_out, (double*)v_out, (double*)a_out, (const double*)H_in,
        (double*)H_out); }
  else if (dtype == PHASTB_F32)
    { note_launch(); q4_explicit_kernel<float><<<grid_full(nn), kThreads, 0, s>>>(
        make_q4_tab<float>(*g), make_mat2<float>(*m), (float)dt, (const float*)m_inv, (const float*)u,
        (const float*)v, (const float*)a, (const float*)d, (const float*)f_ext, bc_mask, (const float*)bc_vals,
        (float*)u_out, (float*)v_out, (float*)a_out, (const float*)H_in, (float*)H_out); }
  else
    return PHASTB_ERR_ARG;
  return last_launch_status();
}

int phastb_q4_explicit_adjoint_step(const phastb_q4_grid* g, const phastb_q4_material* m, double dt,
                                    const double* m_inv, const double* d, const uint8_t* bc_mask,
                                    const double* u_new, const double* ub, const double* vb, const double* ab,
                                    double* ub_out, double* vb_out, double* ab_out, double* fb_acc, double* db_acc,
                                    double* scratch, void* stream) {
  if (!valid_grid(g) || !m || !m_inv || !d || !bc_mask || !ub || !vb || !ab || !ub_out || !vb_out || !ab_out ||
      !scratch)
    return PHASTB_ERR_ARG;
  if (m->stress_split != PHASTB_SPLIT_ISOTROPIC && m->stress_split != PHASTB_SPLIT_LINEAR)
    return PHASTB_UNSUPPORTED;  // the step is then nonlinear in u: its adjoint needs the split's tangent
  if (db_acc && !u_new) return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int nn = (g->nx + 1) * (g->ny + 1), n2 = 2 * nn;
  double* sv = scratch;
  double* Ks = scratch + n2;
  { note_launch(); q4_adj_s_kernel<<<grid_for(n2), kThreads, 0, s>>>(n2, dt, m_inv, bc_mask, vb, ab, sv, fb_acc); }
  int st = last_launch_status();
  if (st) return st;
  if ((st = q4_force_launch(g, m, sv, d, Ks, nullptr, nullptr, s))) return st;
  { note_launch(); q4_adj_combine_kernel<<<grid_for(n2), kThreads, 0, s>>>(n2, dt, bc_mask, ub, vb, Ks, ub_out, vb_out, ab_out); }
  if ((st = last_launch_status())) return st;
  if (db_acc && m->stress_split == PHASTB_SPLIT_ISOTROPIC) {
    note_launch();
    q4_adj_dgrad_kernel<<<grid_full(nn), kThreads, 0, s>>>(make_q4_tab<double>(*g), make_mat2<double>(*m), u_new, sv,
                                                             d, db_acc);
  }
  return last_launch_status();
}

size_t phastb_reduce_workspace_bytes(void) { return red_ws_bytes(); }

int phastb_q4_energy_sums(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* d,
                          const double* v, double* out_host, void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_grid(g) || !m || !u || !d || !out_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < red_ws_bytes()) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(workspace);
  int st = red_ws_reset(ws, s);
  if (st) return st;
  const int nn = (g->nx + 1) * (g->ny + 1);
  { note_launch(); q4_energy_kernel<<<grid_for(nn), kThreads, 0, s>>>(make_q4_tab<double>(*g), make_mat2<double>(*m), u, d, v, ws); }
  st = last_launch_status();
  if (st) return st;
  return red_ws_fetch(ws, out_host, 4, s);
}

size_t phastb_q4_reaction_workspace_bytes(int n_nodes) {
  return red_ws_bytes() + align_up(sizeof(double) * 2 * (size_t)n_nodes);
}

int phastb_q4_reaction(const phastb_q4_grid* g, const phastb_q4_material* m, const double* u, const double* d,
                       const int64_t* nodes, int n_sel, int comp, const double* f_ext, double* out_host,
                       void* workspace, size_t workspace_bytes, void* stream) {
  if (!valid_grid(g) || !m || !u || !nodes || !out_host || comp < 0 || comp > 1 || n_sel < 0) return PHASTB_ERR_ARG;
  const int nn = (g->nx + 1) * (g->ny + 1);
  if (!workspace || workspace_bytes < phastb_q4_reaction_workspace_bytes(nn)) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  RedWs ws = red_ws(workspace);
  double* f = reinterpret_cast<double*>(static_cast<char*>(workspace) + red_ws_bytes());
  int st = red_ws_reset(ws, s);
  if (st) return st;
  st = launch_force<double>(g, m, u, d, f, s);
  if (st) return st;
  { note_launch(); q4_select_sum_kernel<<<grid_for(n_sel), kThreads, 0, s>>>(f, nodes, n_sel, comp, f_ext, ws); }
  st = last_launch_status();
  if (st) return st;
  return red_ws_fetch(ws, out_host, 1, s);
}

}  // extern "C"
