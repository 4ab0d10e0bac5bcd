// Periodic voxel H8 device code.
//
// Every voxel is the same hx*hy*hz brick, so the trilinear shape functions at
// the 2x2x2 Gauss points factor into 1D tables: N1 = [[c1, c2], [c2, c1]]
// (c1,2 = (1 +- 1/sqrt 3)/2) and the derivative along an axis is a plain
// difference of the two faces divided by h.  Gradients, interpolation and the
// transposed (B^T) assembly are therefore evaluated by sum factorisation:
// about 550 flops per element for the elastic operator instead of ~5k for the
// dense B matrices.
//
// Assembly is element->node in two passes without atomics: each element
// writes its local contributions to a structure-of-arrays scratch
// ([corner][component][element], coalesced), then a node kernel gathers the
// (up to) eight contributions of its elements in a fixed order.  Local
// corners are numbered lexicographically, L = ox + 2 oy + 4 oz, and the
// Gauss points likewise, q = qx + 2 qy + 4 qz (PhAST's order, hex8.py:157-178).
#pragma once
#include "common.cuh"

namespace phastb {

constexpr double kC1 = 0.78867513459481288225;  // (1 + 1/sqrt 3) / 2
constexpr double kC2 = 0.21132486540518711775;  // (1 - 1/sqrt 3) / 2

struct VoxGeom {
  int nx, ny, nz, px, py, pz;
  int rx, ry, rz;  // reduced node counts per axis
  int n_red, n_elem;
  int pad_;        // keeps the struct free of implicit padding (it is hashed as bytes)
  double hx, hy, hz, w;
};
static_assert(sizeof(VoxGeom) == 12 * sizeof(int) + 4 * sizeof(double), "VoxGeom has implicit padding");

inline VoxGeom make_vox_geom(const phastb_voxel_grid& g) {
  VoxGeom v{};
  v.nx = g.nx; v.ny = g.ny; v.nz = g.nz;
  v.px = g.px != 0; v.py = g.py != 0; v.pz = g.pz != 0;
  v.rx = v.px ? g.nx : g.nx + 1;
  v.ry = v.py ? g.ny : g.ny + 1;
  v.rz = v.pz ? g.nz : g.nz + 1;
  v.n_red = v.rx * v.ry * v.rz;
  v.n_elem = g.nx * g.ny * g.nz;
  v.hx = g.hx; v.hy = g.hy; v.hz = g.hz;
  v.w = g.hx * g.hy * g.hz / 8.0;
  return v;
}

template <typename T>
struct VoxMat {
  T C[PHASTB_MAX_SLOTS][21];   // upper triangle of the 6x6 stiffness, row-major
  T lam[PHASTB_MAX_SLOTS], mu[PHASTB_MAX_SLOTS], Gc[PHASTB_MAX_SLOTS];
  int driver[PHASTB_MAX_SLOTS];
  int iso;
  // Form of the scalar damage operator (no implicit padding: hashed as bytes):
  // 0 AT2, Gc (M/ell + ell L) + 2 (1 - kappa) H-mass; 1 the PF-CZM Newton tangent,
  // Gc (2 ell/pi) L + the mass of the Gauss-point weights passed as the history
  // (built with kappa = 1/2, so that 2 (1 - kappa) = 1).
  int dform;
  T kappa, ell;
};
static_assert(sizeof(VoxMat<double>) == 8 * (PHASTB_MAX_SLOTS * 24 + 2) + 4 * (PHASTB_MAX_SLOTS + 2), "padding");
static_assert(sizeof(VoxMat<float>) == 4 * (PHASTB_MAX_SLOTS * 24 + 2) + 4 * (PHASTB_MAX_SLOTS + 2), "padding");

inline int tri_index(int i, int j) {  // i <= j
  return i * 6 - i * (i - 1) / 2 + (j - i);
}

template <typename T>
VoxMat<T> make_vox_mat(const phastb_voxel_material& m) {
  VoxMat<T> r{};
  for (int s = 0; s < PHASTB_MAX_SLOTS; ++s) {
    const bool on = s < m.n_slots;
    for (int i = 0; i < 6; ++i)
      for (int j = i; j < 6; ++j) r.C[s][tri_index(i, j)] = on ? T(m.C[s][i * 6 + j]) : T(0);
    r.lam[s] = on ? T(m.lam[s]) : T(0);
    r.mu[s] = on ? T(m.mu[s]) : T(0);
    r.Gc[s] = on ? T(m.Gc[s]) : T(1);
    r.driver[s] = on ? m.driver[s] : 0;
  }
  r.iso = m.isotropic;
  r.kappa = T(m.kappa);
  r.ell = T(m.ell);
  return r;
}

// The same material in another word size (field by field).
template <typename U, typename T>
VoxMat<U> vox_mat_cast(const VoxMat<T>& a) {
  VoxMat<U> r{};
  for (int s = 0; s < PHASTB_MAX_SLOTS; ++s) {
    for (int k = 0; k < 21; ++k) r.C[s][k] = U(a.C[s][k]);
    r.lam[s] = U(a.lam[s]);
    r.mu[s] = U(a.mu[s]);
    r.Gc[s] = U(a.Gc[s]);
    r.driver[s] = a.driver[s];
  }
  r.iso = a.iso;
  r.dform = a.dform;
  r.kappa = U(a.kappa);
  r.ell = U(a.ell);
  return r;
}

// Ascending eigenvalues of a symmetric 3x3 tensor by the trigonometric
// solution of the characteristic cubic (Smith 1961), as symmetric_eigvalsh_3x3
// (solid3d/splits.py:93-125).
__device__ __forceinline__ void eig3(double a11, double a22, double a33, double a12, double a13, double a23,
                                     double* ev) {
  const double q = (a11 + a22 + a33) / 3.0;
  const double b11 = a11 - q, b22 = a22 - q, b33 = a33 - q;
  const double p1 = a12 * a12 + a13 * a13 + a23 * a23;
  const double p = sqrt((b11 * b11 + b22 * b22 + b33 * b33 + 2.0 * p1) / 6.0);
  if (!(p > 2.2250738585072014e-308)) {
    ev[0] = ev[1] = ev[2] = q;
    return;
  }
  const double det = b11 * (b22 * b33 - a23 * a23) - a12 * (a12 * b33 - a23 * a13) + a13 * (a12 * a23 - b22 * a13);
  double r = det / (2.0 * p * p * p);
  r = fmin(fmax(r, -1.0), 1.0);
  const double phi = acos(r) / 3.0;
  const double big = q + 2.0 * p * cos(phi);
  const double small = q + 2.0 * p * cos(phi + 2.0943951023931954923);  // 2 pi / 3
  ev[0] = small;
  ev[1] = 3.0 * q - big - small;
  ev[2] = big;
}

__device__ __forceinline__ int wrap(int i, int n, int periodic) { return periodic ? (i >= n ? i - n : i) : i; }

// Reduced node ids of the 8 corners of element (ie, je, ke), lexicographic.
__device__ __forceinline__ void vox_corners(const VoxGeom& g, int ie, int je, int ke, int* nd) {
#pragma unroll
  for (int L = 0; L < 8; ++L) {
    const int i = wrap(ie + (L & 1), g.nx, g.px);
    const int j = wrap(je + ((L >> 1) & 1), g.ny, g.py);
    const int k = wrap(ke + ((L >> 2) & 1), g.nz, g.pz);
    nd[L] = i + g.rx * (j + g.ry * k);
  }
}

// 1D interpolation to the two Gauss points: out[q] = sum_a N1[q][a] in[a].
template <typename T>
__device__ __forceinline__ void interp2(T a0, T a1, T& q0, T& q1) {
  q0 = T(kC1) * a0 + T(kC2) * a1;
  q1 = T(kC2) * a0 + T(kC1) * a1;
}

// Gradient of a trilinear scalar field u[L] at the Gauss points:
// Dx[qz][qy], Dy[qz][qx], Dz[qy][qx] (each independent of its own axis).
template <typename T>
__device__ __forceinline__ void grad_sf(const T* u, T ihx, T ihy, T ihz, T (&Dx)[2][2], T (&Dy)[2][2],
                                        T (&Dz)[2][2]) {
  // x: difference along x, interpolate along y then z
  {
    T X[2][2];  // [az][ay]
#pragma unroll
    for (int az = 0; az < 2; ++az)
#pragma unroll
      for (int ay = 0; ay < 2; ++ay) X[az][ay] = u[1 + 2 * ay + 4 * az] - u[2 * ay + 4 * az];
    T Y[2][2];  // [az][qy]
#pragma unroll
    for (int az = 0; az < 2; ++az) interp2(X[az][0], X[az][1], Y[az][0], Y[az][1]);
#pragma unroll
    for (int qy = 0; qy < 2; ++qy) {
      T z0, z1;
      interp2(Y[0][qy], Y[1][qy], z0, z1);
      Dx[0][qy] = z0 * ihx;
      Dx[1][qy] = z1 * ihx;
    }
  }
  {
    T X[2][2];  // [az][ax]
#pragma unroll
    for (int az = 0; az < 2; ++az)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) X[az][ax] = u[ax + 2 + 4 * az] - u[ax + 4 * az];
    T Y[2][2];  // [az][qx]
#pragma unroll
    for (int az = 0; az < 2; ++az) interp2(X[az][0], X[az][1], Y[az][0], Y[az][1]);
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) {
      T z0, z1;
      interp2(Y[0][qx], Y[1][qx], z0, z1);
      Dy[0][qx] = z0 * ihy;
      Dy[1][qx] = z1 * ihy;
    }
  }
  {
    T X[2][2];  // [ay][ax]
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) X[ay][ax] = u[ax + 2 * ay + 4] - u[ax + 2 * ay];
    T Y[2][2];  // [ay][qx]
#pragma unroll
    for (int ay = 0; ay < 2; ++ay) interp2(X[ay][0], X[ay][1], Y[ay][0], Y[ay][1]);
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) {
      T z0, z1;
      interp2(Y[0][qx], Y[1][qx], z0, z1);
      Dz[0][qx] = z0 * ihz;
      Dz[1][qx] = z1 * ihz;
    }
  }
}

// Trilinear interpolation of nodal u[L] to the Gauss points uq[q].
template <typename T>
__device__ __forceinline__ void interp_sf(const T* u, T* uq) {
  T A[8];
#pragma unroll
  for (int r = 0; r < 4; ++r) interp2(u[2 * r], u[2 * r + 1], A[2 * r], A[2 * r + 1]);  // along x
  T B[8];
#pragma unroll
  for (int z = 0; z < 2; ++z)
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) interp2(A[qx + 4 * z], A[qx + 2 + 4 * z], B[qx + 4 * z], B[qx + 2 + 4 * z]);
#pragma unroll
  for (int r = 0; r < 4; ++r) interp2(B[r], B[r + 4], uq[r], uq[r + 4]);
}

// Transpose of interp_sf: out[L] = sum_q N_L(q) v[q].
template <typename T>
__device__ __forceinline__ void interp_sf_t(const T* v, T* out) {
  T B[8];
#pragma unroll
  for (int r = 0; r < 4; ++r) interp2(v[r], v[r + 4], B[r], B[r + 4]);
  T A[8];
#pragma unroll
  for (int z = 0; z < 2; ++z)
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) interp2(B[qx + 4 * z], B[qx + 2 + 4 * z], A[qx + 4 * z], A[qx + 2 + 4 * z]);
#pragma unroll
  for (int r = 0; r < 4; ++r) interp2(A[2 * r], A[2 * r + 1], out[2 * r], out[2 * r + 1]);
}

// Transposed gradient: out[L] += sum_q dN_L/dx Px-term etc., where the inputs
// are already summed over their own axis: Px[qz][qy] = sum_qx Tx(q), Py[qz][qx],
// Pz[qy][qx].  (N1 is symmetric, so the transposed 1D interpolation is interp2.)
template <typename T>
__device__ __forceinline__ void grad_sf_t(const T (&Px)[2][2], const T (&Py)[2][2], const T (&Pz)[2][2], T ihx,
                                          T ihy, T ihz, T* out) {
#pragma unroll
  for (int L = 0; L < 8; ++L) out[L] = T(0);
  {
    T Y[2][2];  // [az][qy]
#pragma unroll
    for (int qy = 0; qy < 2; ++qy) interp2(Px[0][qy], Px[1][qy], Y[0][qy], Y[1][qy]);
#pragma unroll
    for (int az = 0; az < 2; ++az) {
      T q0, q1;
      interp2(Y[az][0], Y[az][1], q0, q1);  // [ay]
      out[0 + 0 + 4 * az] -= q0 * ihx;
      out[1 + 0 + 4 * az] += q0 * ihx;
      out[0 + 2 + 4 * az] -= q1 * ihx;
      out[1 + 2 + 4 * az] += q1 * ihx;
    }
  }
  {
    T Y[2][2];  // [az][qx]
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) interp2(Py[0][qx], Py[1][qx], Y[0][qx], Y[1][qx]);
#pragma unroll
    for (int az = 0; az < 2; ++az) {
      T q0, q1;
      interp2(Y[az][0], Y[az][1], q0, q1);  // [ax]
      out[0 + 0 + 4 * az] -= q0 * ihy;
      out[0 + 2 + 4 * az] += q0 * ihy;
      out[1 + 0 + 4 * az] -= q1 * ihy;
      out[1 + 2 + 4 * az] += q1 * ihy;
    }
  }
  {
    T Y[2][2];  // [ay][qx]
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) interp2(Pz[0][qx], Pz[1][qx], Y[0][qx], Y[1][qx]);
#pragma unroll
    for (int ay = 0; ay < 2; ++ay) {
      T q0, q1;
      interp2(Y[ay][0], Y[ay][1], q0, q1);  // [ax]
      out[0 + 2 * ay + 0] -= q0 * ihz;
      out[0 + 2 * ay + 4] += q0 * ihz;
      out[1 + 2 * ay + 0] -= q1 * ihz;
      out[1 + 2 * ay + 4] += q1 * ihz;
    }
  }
}

// sigma = C eps for a material slot (engineering Voigt).
template <typename T>
__device__ __forceinline__ void voigt_stress(const VoxMat<T>& m, int s, const T* e, T* sg) {
  if (m.iso) {
    const T lam = m.lam[s], mu = m.mu[s];
    const T tr = e[0] + e[1] + e[2];
    sg[0] = lam * tr + 2 * mu * e[0];
    sg[1] = lam * tr + 2 * mu * e[1];
    sg[2] = lam * tr + 2 * mu * e[2];
    sg[3] = mu * e[3];
    sg[4] = mu * e[4];
    sg[5] = mu * e[5];
  } else {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      T acc = 0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const int a = i < j ? i : j, b = i < j ? j : i;
        acc += m.C[s][a * 6 - a * (a - 1) / 2 + (b - a)] * e[j];
      }
      sg[i] = acc;
    }
  }
}

template <typename T>
__device__ __forceinline__ T voigt_diag(const VoxMat<T>& m, int s, int k) {
  return m.C[s][k * 6 - k * (k - 1) / 2];
}

}  // namespace phastb
