// Structured Q4 (2x2 Gauss) device code: geometry tables, constitutive laws
// and the node-centric gather kernels.
//
// Every element of a structured_q4_mesh grid is the same hx x hy rectangle, so
// shape-function values and gradients at the Gauss points are four 4x4 tables
// shared by all elements; nothing geometric is read from memory.  A thread
// owns one node and recomputes the Gauss-point stresses of its (up to) four
// elements: the sum over elements happens in registers, in a fixed order,
// with no atomics (deterministic).  The grids of the 2D configurations hold
// 40k-66k nodes, so the element recomputation is cheap next to launch latency.
#pragma once
#include "common.cuh"

namespace phastb {

template <typename T>
struct Q4Tab {
  T N[4][4];   // N[q][a]
  T gx[4][4];  // dN_a/dx at q
  T gy[4][4];  // dN_a/dy at q
  T w;         // w_q det J (same at every q)
  int nx, ny;
};

// Corner signs in CCW order and Gauss points with xi fastest
// (quad_elements.py: q4_shape_functions, quad_gauss_points).
template <typename T>
Q4Tab<T> make_q4_tab(const phastb_q4_grid& g) {
  Q4Tab<T> t;
  const double s[4] = {-1, 1, 1, -1}, r[4] = {-1, -1, 1, 1};
  const double a = 0.57735026918962576451;  // 1/sqrt(3)
  const double xq[4] = {-a, a, -a, a}, yq[4] = {-a, -a, a, a};
  for (int q = 0; q < 4; ++q)
    for (int b = 0; b < 4; ++b) {
      t.N[q][b] = T(0.25 * (1 + s[b] * xq[q]) * (1 + r[b] * yq[q]));
      t.gx[q][b] = T(s[b] * (1 + r[b] * yq[q]) / (2.0 * g.hx));
      t.gy[q][b] = T(r[b] * (1 + s[b] * xq[q]) / (2.0 * g.hy));
    }
  t.w = T(0.25 * g.hx * g.hy);
  t.nx = g.nx;
  t.ny = g.ny;
  return t;
}

template <typename T>
struct Mat2 {
  T lam, mu, kap, nu, E, eta, seps;
  int ps, ssplit, psplit;
};

template <typename T>
Mat2<T> make_mat2(const phastb_q4_material& m) {
  Mat2<T> r;
  r.lam = T(m.lam); r.mu = T(m.mu); r.kap = T(m.kappa); r.nu = T(m.nu); r.E = T(m.E);
  r.eta = T(m.eta); r.seps = T(m.spectral_eps);
  r.ps = m.plane_stress; r.ssplit = m.stress_split; r.psplit = m.psi_split;
  return r;
}

template <typename T>
__device__ __forceinline__ T degr(const Mat2<T>& m, T d) {
  const T o = T(1) - d;
  return o * o * (T(1) - m.eta) + m.eta;
}

template <typename T>
__device__ __forceinline__ T ezz_of(const Mat2<T>& m, T tr2) {
  return m.ps ? -m.nu / (T(1) - m.nu) * tr2 : T(0);
}

// Degraded stress of one split (fem_operators.py:283-560).
template <typename T>
__device__ __forceinline__ void stress2(const Mat2<T>& m, int split, T exx, T eyy, T gxy, T g, T& sxx,
                                        T& syy, T& sxy) {
  const T lam = m.lam, mu = m.mu;
  switch (split) {
    case PHASTB_SPLIT_LINEAR:
      sxx = (lam + 2 * mu) * exx + lam * eyy;
      syy = lam * exx + (lam + 2 * mu) * eyy;
      sxy = mu * gxy;
      return;
    case PHASTB_SPLIT_AMOR: {
      const T tr2 = exx + eyy;
      const T tr = tr2 + ezz_of(m, tr2);
      const T trp = tr > T(0) ? tr : T(0);
      const T trm = tr - trp;
      sxx = g * (m.kap * trp + 2 * mu * (exx - tr / T(3))) + m.kap * trm;
      syy = g * (m.kap * trp + 2 * mu * (eyy - tr / T(3))) + m.kap * trm;
      sxy = g * mu * gxy;
      return;
    }
    case PHASTB_SPLIT_SPECTRAL:
    case PHASTB_SPLIT_SPECTRAL_STRESS: {
      const T exy = gxy / T(2);
      const T trace = exx + eyy;
      const T hd = (exx - eyy) / T(2);
      const T delta = sqrt(hd * hd + exy * exy + m.seps);
      const T e1 = trace / T(2) + delta, e2 = trace / T(2) - delta;
      const T inv2d = T(1) / (T(2) * delta + T(1e-30));
      const T pxx = (hd + delta) * inv2d, pyy = (-hd + delta) * inv2d, pxy = exy * inv2d;
      if (split == PHASTB_SPLIT_SPECTRAL) {
        const T e1p = e1 > T(0) ? e1 : T(0), e2p = e2 > T(0) ? e2 : T(0);
        const T trp = trace > T(0) ? trace : T(0), trm = trace - trp;
        const T xxp = e1p * pxx + e2p * (T(1) - pxx);
        const T yyp = e1p * pyy + e2p * (T(1) - pyy);
        const T xyp = (e1p - e2p) * pxy;
        sxx = g * (lam * trp + 2 * mu * xxp) + (lam * trm + 2 * mu * (exx - xxp));
        syy = g * (lam * trp + 2 * mu * yyp) + (lam * trm + 2 * mu * (eyy - yyp));
        sxy = g * (2 * mu * xyp) + 2 * mu * (exy - xyp);
      } else {
        const T s1 = lam * trace + 2 * mu * e1, s2 = lam * trace + 2 * mu * e2;
        const T s1p = s1 > T(0) ? s1 : T(0), s2p = s2 > T(0) ? s2 : T(0);
        const T s1m = s1 - s1p, s2m = s2 - s2p;
        sxx = g * (s1p * pxx + s2p * (T(1) - pxx)) + (s1m * pxx + s2m * (T(1) - pxx));
        syy = g * (s1p * pyy + s2p * (T(1) - pyy)) + (s1m * pyy + s2m * (T(1) - pyy));
        sxy = g * ((s1p - s2p) * pxy) + (s1m - s2m) * pxy;
      }
      return;
    }
    case PHASTB_SPLIT_STAR_CONVEX: {
      const T tr2 = exx + eyy;
      const T tr = tr2 + ezz_of(m, tr2);
      if (tr >= T(0)) {
        sxx = g * ((lam + 2 * mu) * exx + lam * eyy);
        syy = g * (lam * exx + (lam + 2 * mu) * eyy);
        sxy = g * (mu * gxy);
      } else {
        sxx = g * 2 * mu * (exx - tr / T(3)) + m.kap * tr;
        syy = g * 2 * mu * (eyy - tr / T(3)) + m.kap * tr;
        sxy = g * mu * gxy;
      }
      return;
    }
    default:  // PHASTB_SPLIT_ISOTROPIC
      sxx = g * ((lam + 2 * mu) * exx + lam * eyy);
      syy = g * (lam * exx + (lam + 2 * mu) * eyy);
      sxy = g * (mu * gxy);
      return;
  }
}

// Consistent tangent of stress2: the directional derivative d sigma(eps)[d eps] of the
// split stress at the strain (exx, eyy, gxy), at fixed degradation g.  This is the action
// QuasiStaticSolver takes by an autograd JVP of internal_force for the spectral, Amor and
// star-convex splits (mechanics_solver.py:1705-1733, 2000-2012); it differentiates the same
// algebra as stress2 (projectors included), with the derivative of a positive part
// max(x, 0) taken as 1 where x >= 0, as the JVP of clamp(min=0) does.  Linear and isotropic
// stresses are their own tangent; the stress-spectral split has no entry here (the reference
// linearises it by evaluating the stress at the increment, which stress2 already does).
template <typename T>
__device__ __forceinline__ void dstress2(const Mat2<T>& m, int split, T exx, T eyy, T gxy, T dexx, T deyy, T dgxy,
                                         T g, T& dsxx, T& dsyy, T& dsxy) {
  const T lam = m.lam, mu = m.mu;
  switch (split) {
    case PHASTB_SPLIT_AMOR:
    case PHASTB_SPLIT_STAR_CONVEX: {
      const T tr2 = exx + eyy;
      const T tr = tr2 + ezz_of(m, tr2);
      const T dtr2 = dexx + deyy;
      const T dtr = dtr2 + ezz_of(m, dtr2);
      const bool pos = tr >= T(0);
      if (split == PHASTB_SPLIT_AMOR) {
        const T dtrp = pos ? dtr : T(0), dtrm = dtr - dtrp;
        dsxx = g * (m.kap * dtrp + 2 * mu * (dexx - dtr / T(3))) + m.kap * dtrm;
        dsyy = g * (m.kap * dtrp + 2 * mu * (deyy - dtr / T(3))) + m.kap * dtrm;
        dsxy = g * mu * dgxy;
      } else if (pos) {
        dsxx = g * ((lam + 2 * mu) * dexx + lam * deyy);
        dsyy = g * (lam * dexx + (lam + 2 * mu) * deyy);
        dsxy = g * (mu * dgxy);
      } else {
        dsxx = g * 2 * mu * (dexx - dtr / T(3)) + m.kap * dtr;
        dsyy = g * 2 * mu * (deyy - dtr / T(3)) + m.kap * dtr;
        dsxy = g * mu * dgxy;
      }
      return;
    }
    case PHASTB_SPLIT_SPECTRAL: {
      const T exy = gxy / T(2), dexy = dgxy / T(2);
      const T trace = exx + eyy, dtrace = dexx + deyy;
      const T hd = (exx - eyy) / T(2), dhd = (dexx - deyy) / T(2);
      const T delta = sqrt(hd * hd + exy * exy + m.seps);
      const T ddelta = (hd * dhd + exy * dexy) / delta;
      const T e1 = trace / T(2) + delta, e2 = trace / T(2) - delta;
      const T de1 = dtrace / T(2) + ddelta, de2 = dtrace / T(2) - ddelta;
      const T e1p = e1 > T(0) ? e1 : T(0), e2p = e2 > T(0) ? e2 : T(0);
      const T de1p = e1 >= T(0) ? de1 : T(0), de2p = e2 >= T(0) ? de2 : T(0);
      const T dtrp = trace >= T(0) ? dtrace : T(0), dtrm = dtrace - dtrp;
      const T inv2d = T(1) / (T(2) * delta + T(1e-30));
      const T dinv2d = -T(2) * ddelta * inv2d * inv2d;
      const T pxx = (hd + delta) * inv2d, pyy = (-hd + delta) * inv2d, pxy = exy * inv2d;
      const T dpxx = (dhd + ddelta) * inv2d + (hd + delta) * dinv2d;
      const T dpyy = (-dhd + ddelta) * inv2d + (-hd + delta) * dinv2d;
      const T dpxy = dexy * inv2d + exy * dinv2d;
      const T dxxp = de1p * pxx + e1p * dpxx + de2p * (T(1) - pxx) - e2p * dpxx;
      const T dyyp = de1p * pyy + e1p * dpyy + de2p * (T(1) - pyy) - e2p * dpyy;
      const T dxyp = (de1p - de2p) * pxy + (e1p - e2p) * dpxy;
      dsxx = g * (lam * dtrp + 2 * mu * dxxp) + (lam * dtrm + 2 * mu * (dexx - dxxp));
      dsyy = g * (lam * dtrp + 2 * mu * dyyp) + (lam * dtrm + 2 * mu * (deyy - dyyp));
      dsxy = g * (2 * mu * dxyp) + 2 * mu * (dexy - dxyp);
      return;
    }
    default:  // linear in eps: the tangent is the stress of the increment
      stress2(m, split, dexx, deyy, dgxy, g, dsxx, dsyy, dsxy);
      return;
  }
}

// Tensile energy psi+ of one split (fem_operators.py:974-1161).
template <typename T>
__device__ __forceinline__ T psi2(const Mat2<T>& m, int split, T exx, T eyy, T gxy) {
  const T lam = m.lam, mu = m.mu;
  const T exy = gxy / T(2);
  switch (split) {
    case PHASTB_SPLIT_AMOR: {
      const T tr2 = exx + eyy;
      const T ezz = ezz_of(m, tr2);
      const T tr = tr2 + ezz;
      const T trp = tr > T(0) ? tr : T(0);
      const T a = exx - tr / T(3), b = eyy - tr / T(3), c = ezz - tr / T(3);
      return T(0.5) * m.kap * trp * trp + mu * (a * a + b * b + c * c + 2 * exy * exy);
    }
    case PHASTB_SPLIT_SPECTRAL:
    case PHASTB_SPLIT_SPECTRAL_STRESS: {
      const T trace = exx + eyy;
      const T hd = (exx - eyy) / T(2);
      const T delta = sqrt(hd * hd + exy * exy + m.seps);
      const T e1 = trace / T(2) + delta, e2 = trace / T(2) - delta;
      if (split == PHASTB_SPLIT_SPECTRAL) {
        const T trp = trace > T(0) ? trace : T(0);
        const T e1p = e1 > T(0) ? e1 : T(0), e2p = e2 > T(0) ? e2 : T(0);
        return T(0.5) * lam * trp * trp + mu * (e1p * e1p + e2p * e2p);
      }
      T s1 = lam * trace + 2 * mu * e1, s2 = lam * trace + 2 * mu * e2;
      s1 = s1 > T(0) ? s1 : T(0);
      s2 = s2 > T(0) ? s2 : T(0);
      return (s1 * s1 + s2 * s2 - T(2) * m.nu * s1 * s2) / (T(2) * m.E);
    }
    case PHASTB_SPLIT_STAR_CONVEX: {
      const T tr2 = exx + eyy;
      const T ezz = ezz_of(m, tr2);
      const T tr = tr2 + ezz;
      if (tr >= T(0)) return T(0.5) * lam * tr2 * tr2 + mu * (exx * exx + eyy * eyy + 2 * exy * exy);
      const T a = exx - tr / T(3), b = eyy - tr / T(3), c = ezz - tr / T(3);
      return mu * (a * a + b * b + c * c + 2 * exy * exy);
    }
    default: {  // isotropic (full energy)
      const T tr = exx + eyy;
      return T(0.5) * lam * tr * tr + mu * (exx * exx + eyy * eyy + 2 * exy * exy);
    }
  }
}

// Corner node ids of element (ei, ej), CCW.
__device__ __forceinline__ void q4_corners(int ei, int ej, int nx, int* n) {
  const int n0 = ej * (nx + 1) + ei;
  n[0] = n0;
  n[1] = n0 + 1;
  n[2] = n0 + nx + 2;
  n[3] = n0 + nx + 1;
}

// Local corner index of the node at offset (lx, ly) in its element.
__host__ __device__ constexpr int q4_local(int lx, int ly) { return ly == 0 ? lx : (lx == 1 ? 2 : 3); }

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <typename T>
__device__ __forceinline__ void load2(const T* p, int node, T& x, T& y) {
  const typename Vec2<T>::type v = __ldg(reinterpret_cast<const typename Vec2<T>::type*>(p) + node);
  x = v.x;
  y = v.y;
}

}  // namespace phastb
