// Packed FP32 variant of the tiled elastic action (included by h8_tile.cu).
//
// Same brick schedule, staging, face sums and epilogues as h8_tile_kernel, but
// every thread computes TWO x-adjacent elements of the element tile at once, one
// in each lane of a float2, with sm_100's packed FP32 instructions
// (__ffma2_rn / __fmul2_rn / __fadd2_rn: one instruction, two IEEE FP32 results).
// Each lane performs exactly the scalar kernel's operations on its element, so
// the arithmetic takes half the issue slots; the two elements share the loads of
// their common face of nodes.  In the node phase every thread owns two
// x-adjacent nodes.  Threads per block: max(element pairs, node pairs).
//
// Supported: FP32, isotropic slot coefficients (the fine operator, g(d) fused)
// and per-Gauss-point moduli (multigrid coarse levels), every epilogue; even ox.

namespace {

__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b (exact product b * -1, one rounding: the same result as a subtraction)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 neg2(float2 a) { return __fmul2_rn(a, make_float2(-1.f, -1.f)); }
__device__ __forceinline__ float hsum(float2 a, float2 mask) { return mask.x * a.x + mask.y * a.y; }

struct TileK2 {
  float2 c1, c2, x1, x2, y1, y2, z1, z2;
};

__device__ __forceinline__ TileK2 tile_k2(const TileK<float>& k) {
  return TileK2{bc2(k.c1), bc2(k.c2), bc2(k.x1), bc2(k.x2), bc2(k.y1), bc2(k.y2), bc2(k.z1), bc2(k.z2)};
}

__device__ __forceinline__ void ip2p(float2 a0, float2 a1, float2 c1, float2 c2, float2& q0, float2& q1) {
  q0 = fma2(c1, a0, mul2(c2, a1));
  q1 = fma2(c2, a0, mul2(c1, a1));
}

// grad_k on both lanes: Dx[qz][qy], Dy[qz][qx], Dz[qy][qx].
__device__ __forceinline__ void grad_p(const float2* u, const TileK2& k, float2 (&Dx)[2][2], float2 (&Dy)[2][2],
                                       float2 (&Dz)[2][2]) {
  {
    float2 Y[2][2];  // [az][qy]
#pragma unroll
    for (int az = 0; az < 2; ++az)
      ip2p(sub2(u[1 + 4 * az], u[4 * az]), sub2(u[3 + 4 * az], u[2 + 4 * az]), k.c1, k.c2, Y[az][0], Y[az][1]);
#pragma unroll
    for (int qy = 0; qy < 2; ++qy) ip2p(Y[0][qy], Y[1][qy], k.x1, k.x2, Dx[0][qy], Dx[1][qy]);
  }
  {
    float2 Y[2][2];  // [az][qx]
#pragma unroll
    for (int az = 0; az < 2; ++az)
      ip2p(sub2(u[2 + 4 * az], u[4 * az]), sub2(u[3 + 4 * az], u[1 + 4 * az]), k.c1, k.c2, Y[az][0], Y[az][1]);
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2p(Y[0][qx], Y[1][qx], k.y1, k.y2, Dy[0][qx], Dy[1][qx]);
  }
  {
    float2 Y[2][2];  // [ay][qx]
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
      ip2p(sub2(u[4 + 2 * ay], u[2 * ay]), sub2(u[5 + 2 * ay], u[1 + 2 * ay]), k.c1, k.c2, Y[ay][0], Y[ay][1]);
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2p(Y[0][qx], Y[1][qx], k.z1, k.z2, Dz[0][qx], Dz[1][qx]);
  }
}

// grad_k_t on both lanes: out[L] = +-Ax +-Ay +-Az by the corner's side on each axis.
__device__ __forceinline__ void grad_p_t(const float2 (&Px)[2][2], const float2 (&Py)[2][2], const float2 (&Pz)[2][2],
                                         const TileK2& k, float2* out) {
  float2 Ax[2][2], Ay[2][2], Az[2][2];
  {
    float2 Y[2][2];
#pragma unroll
    for (int qy = 0; qy < 2; ++qy) ip2p(Px[0][qy], Px[1][qy], k.x1, k.x2, Y[0][qy], Y[1][qy]);
#pragma unroll
    for (int az = 0; az < 2; ++az) ip2p(Y[az][0], Y[az][1], k.c1, k.c2, Ax[az][0], Ax[az][1]);  // [az][ay]
  }
  {
    float2 Y[2][2];
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2p(Py[0][qx], Py[1][qx], k.y1, k.y2, Y[0][qx], Y[1][qx]);
#pragma unroll
    for (int az = 0; az < 2; ++az) ip2p(Y[az][0], Y[az][1], k.c1, k.c2, Ay[az][0], Ay[az][1]);  // [az][ax]
  }
  {
    float2 Y[2][2];
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2p(Pz[0][qx], Pz[1][qx], k.z1, k.z2, Y[0][qx], Y[1][qx]);
#pragma unroll
    for (int ay = 0; ay < 2; ++ay) ip2p(Y[ay][0], Y[ay][1], k.c1, k.c2, Az[ay][0], Az[ay][1]);  // [ay][ax]
  }
#pragma unroll
  for (int L = 0; L < 8; ++L) {
    const int ax = L & 1, ay = (L >> 1) & 1, az = L >> 2;
    const float2 tx = Ax[az][ay], ty = Ay[az][ax], tz = Az[ay][ax];
    // +-tx +-ty +-tz with the sign of each axis' side, as two packed adds
    float2 s;
    if (ay && az) s = add2(ty, tz);
    else if (ay) s = sub2(ty, tz);
    else if (az) s = sub2(tz, ty);
    else s = neg2(add2(ty, tz));
    out[L] = ax ? add2(s, tx) : sub2(s, tx);
  }
}

// interp_sf on both lanes (nodal values to the Gauss points, q = qx + 2 qy + 4 qz).
__device__ __forceinline__ void interp_p(const float2* u, float2 c1, float2 c2, float2* uq) {
  float2 A[8];
#pragma unroll
  for (int r = 0; r < 4; ++r) ip2p(u[2 * r], u[2 * r + 1], c1, c2, A[2 * r], A[2 * r + 1]);
  float2 B[8];
#pragma unroll
  for (int z = 0; z < 2; ++z)
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2p(A[qx + 4 * z], A[qx + 2 + 4 * z], c1, c2, B[qx + 4 * z], B[qx + 2 + 4 * z]);
#pragma unroll
  for (int r = 0; r < 4; ++r) ip2p(B[r], B[r + 4], c1, c2, uq[r], uq[r + 4]);
}

__device__ __forceinline__ float2 lane_sel(bool a, bool b, float2 v) {
  return make_float2(a ? v.x : 0.f, b ? v.y : 0.f);
}

}  // namespace

constexpr int kTile2MaxThreads = 256;

// Launch geometry of the packed kernel for a tile shape: element pairs along x,
// node pairs along x (ox even), threads = max of the two rounded to a warp.
__host__ __device__ inline int tile2_epairs(int ox, int oy) { return ((ox + 2) / 2) * (oy + 1); }
__host__ __device__ inline int tile2_npairs(int ox, int oy) { return (ox / 2) * oy; }
inline int tile2_threads(const TileShape& t) {
  const int n = tile2_epairs(t.ox, t.oy) > tile2_npairs(t.ox, t.oy) ? tile2_epairs(t.ox, t.oy)
                                                                     : tile2_npairs(t.ox, t.oy);
  return (n + 31) / 32 * 32;
}
inline bool tile2_ok(const TileShape& t) {
  return t.ox >= 2 && t.ox % 2 == 0 && t.oy >= 1 && tile2_threads(t) <= kTile2MaxThreads &&
         (t.ox + 2) * (t.oy + 2) <= 2 * tile2_threads(t);
}

template <int COEF, int MODE, int OX, int OY>
__global__ void __launch_bounds__(kTile2MaxThreads, 1) h8_tile2_kernel(TileArgs<float> a, VoxMat<float> m) {
  using T = float;
  if (a.guard && *a.guard == 0) return;
  constexpr bool SLOT = COEF != kCoefQP;
  constexpr bool DOT = MODE == kModeDot, ENERGY = MODE == kModeEnergy, CHEB = MODE == kModeCheb;
  constexpr bool NODAL = MODE == kModeNodal;
  constexpr bool EROWS = SLOT && !CHEB && !NODAL;
  constexpr bool RED = EROWS || DOT || ENERGY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const VoxGeom& g = a.g;
  if (NODAL && blockIdx.x == 0 && threadIdx.x < 6 && a.y) a.y[3 * (size_t)g.n_red + threadIdx.x] = T(0);
  const T* __restrict__ x = a.x;
  const T* __restrict__ d = SLOT ? a.d : nullptr;
  const int ox = OX ? OX : a.ts.ox, oy = OY ? OY : a.ts.oy, kz = a.ts.kz;
  const int ex = ox + 1, exy = ex * (oy + 1);
  const int ntx = ox + 2, nt = ntx * (oy + 2);
  T* nb = reinterpret_cast<T*>(smem_raw);  // [3 buffers][4 fields][nt]
  T* FL = nb + 12 * nt;                    // [4 corners][3 comps][exy]
  T* FU = FL + 12 * exy;
  constexpr bool STAGE = COEF == kCoefQP || CHEB;
  constexpr int kQChunks = kStageQP * (int)sizeof(T) / 16;
  size_t off_qp = 0, off_cheb = 0;
  tile_layout<T>(ox, oy, COEF == kCoefQP, CHEB, &off_qp, &off_cheb);
  unsigned char* QS = smem_raw + off_qp;
  T* CS = reinterpret_cast<T*>(smem_raw + off_cheb);
  const int oxy = ox * oy;
  const bool q_async = COEF == kCoefQP && aligned16(a.lam_q) && aligned16(a.mu_q);
  const int tid = threadIdx.x;
  const TileK2 k2 = tile_k2(a.k);
  const T w = T(g.w);
  const T c1 = T(a.c1), c2 = T(a.c2);
  T E6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  if (EROWS) {
    const T* Ex = x + 3 * (size_t)g.n_red;
#pragma unroll
    for (int k = 0; k < 6; ++k) E6[k] = __ldg(Ex + k);
  }
  const int tiles_x = (g.rx + ox - 1) / ox, tiles_y = (g.ry + oy - 1) / oy;
  const int tiles_xy = tiles_x * tiles_y;
  const int n_tiles = tiles_xy * ((g.rz + kz - 1) / kz);
  // this thread's element pair (columns ea0, ea0 + 1 of row eb) and node pair (ni0, ni0 + 1 of row nj)
  const int px = (ox + 2) / 2, hx = ox / 2;
  const bool is_pair = tid < px * (oy + 1), is_npair = tid < hx * oy;
  const int ea0 = 2 * (tid % px), eb = tid / px;
  const int ni0 = 2 * (tid % hx), nj = tid / hx;
  const bool has_b = ea0 + 1 < ex;  // the second element lies inside the tile
  const int ida = eb * ex + ea0, idb = ida + 1;
  double accd[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  auto elem_index = [&](int i0, int j0, int ke, int ea, size_t* e) -> bool {
    const int gi = wrap_elem(i0 - 1 + ea, g.nx, g.px);
    const int gj = wrap_elem(j0 - 1 + eb, g.ny, g.py);
    const int gk = wrap_elem(ke, g.nz, g.pz);
    if (gi < 0 || gj < 0 || gk < 0) return false;
    *e = (size_t)gi + (size_t)g.nx * ((size_t)gj + (size_t)g.ny * gk);
    return true;
  };
  auto elem_slot = [&](int i0, int j0, int ke, int ea, bool live) -> int {
    size_t e;
    if (!SLOT || !is_pair || !live || !elem_index(i0, j0, ke, ea, &e)) return 0;
    return __ldg(a.slot + e);
  };
  auto node_mask = [&](int i0, int j0, int kn, int ni) -> int {
    if (!a.mask || !is_npair || kn >= g.rz) return 0;
    const int gi = i0 + ni, gj = j0 + nj;
    if (gi >= g.rx || gj >= g.ry) return 0;
    const size_t n = (size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * kn);
    return (__ldg(a.mask + 3 * n) ? 1 : 0) | (__ldg(a.mask + 3 * n + 1) ? 2 : 0) |
           (__ldg(a.mask + 3 * n + 2) ? 4 : 0);
  };
  // commit-group order as the scalar kernel: per step one Chebyshev group, one moduli group
  auto stage_qp = [&](int i0, int j0, int ke, int buf, bool live) {
    if constexpr (STAGE) {
      if (COEF == kCoefQP && live && q_async && is_pair) {
        unsigned char* dst = QS + (size_t)buf * kQChunks * exy * 16;
        size_t e;
        if (elem_index(i0, j0, ke, ea0, &e)) {
          stage_chunks(dst, exy, ida, 0, a.lam_q + 8 * e, kQChunks / 2);
          stage_chunks(dst, exy, ida, kQChunks / 2, a.mu_q + 8 * e, kQChunks / 2);
        }
        if (has_b && elem_index(i0, j0, ke, ea0 + 1, &e)) {
          stage_chunks(dst, exy, idb, 0, a.lam_q + 8 * e, kQChunks / 2);
          stage_chunks(dst, exy, idb, kQChunks / 2, a.mu_q + 8 * e, kQChunks / 2);
        }
      }
      cp_async_commit();
    }
  };
  auto stage_cheb = [&](int i0, int j0, int kn, int buf, bool live) {
    if constexpr (STAGE) {
      if (CHEB && live && is_npair) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int ni = ni0 + h, gi = i0 + ni, gj = j0 + nj;
          if (gi < g.rx && gj < g.ry) {
            const size_t n3 = 3 * ((size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * kn));
            T* dst = CS + (size_t)buf * 9 * oxy + (nj * ox + ni);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              cp_async_word(dst + c * oxy, a.res + n3 + c);
              cp_async_word(dst + (3 + c) * oxy, a.invd + n3 + c);
              cp_async_word(dst + (6 + c) * oxy, a.xs + n3 + c);
            }
          }
        }
      }
      cp_async_commit();
    }
  };

  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int tz = tile / tiles_xy, txy = tile - tz * tiles_xy;
    const int i0 = (txy % tiles_x) * ox, j0 = (txy / tiles_x) * oy;
    const int k0 = tz * kz, k1 = min(k0 + kz, g.rz);
    T tacc[8] = {T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0)};
    T pend[2][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
    Staged<T> pf;
    stage_load(g, x, d, i0, j0, k0 - 1, ntx, nt, pf);
    __syncthreads();
    stage_store(nt, pf, nb);
    stage_load(g, x, d, i0, j0, k0, ntx, nt, pf);
    int sla_next = elem_slot(i0, j0, k0 - 1, ea0, true), slb_next = elem_slot(i0, j0, k0 - 1, ea0 + 1, has_b);
    stage_qp(i0, j0, k0 - 1, 0, true);
    int mk_next[2] = {node_mask(i0, j0, k0, ni0), node_mask(i0, j0, k0, ni0 + 1)}, mk_cur[2] = {0, 0};
    const int K = k1 - k0;
    for (int kk = 0; kk <= K; ++kk) {
      const int ke = k0 - 1 + kk;
      T* b0 = nb + 4 * nt * (kk % 3);
      T* b1 = nb + 4 * nt * ((kk + 1) % 3);
      stage_store(nt, pf, b1);
      const int sla = sla_next, slb = slb_next;
      if (kk < K) {
        stage_load(g, x, d, i0, j0, ke + 2, ntx, nt, pf);
        sla_next = elem_slot(i0, j0, ke + 1, ea0, true);
        slb_next = elem_slot(i0, j0, ke + 1, ea0 + 1, has_b);
      }
      if constexpr (STAGE) {
        stage_cheb(i0, j0, ke, kk & 1, kk >= 1);
        stage_qp(i0, j0, ke + 1, (kk + 1) & 1, kk < K);
        cp_async_wait<2>();
      }
      if (kk >= 1) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          mk_cur[h] = mk_next[h];
          if (kk < K) mk_next[h] = node_mask(i0, j0, ke + 1, ni0 + h);
        }
      }
      __syncthreads();
      // ---- element phase: elements ea0 (lane x) and ea0 + 1 (lane y) of row eb
      if (is_pair) {
        size_t ea_g = 0, eb_g = 0;
        const bool va = elem_index(i0, j0, ke, ea0, &ea_g);
        const bool vb = has_b && elem_index(i0, j0, ke, ea0 + 1, &eb_g);
        float2 f[3][8];
        if (va || vb) {
          // node columns ea0, ea0 + 1, ea0 + 2 of the two rows and layers (clamped inside the halo tile)
          const int cb = min(ea0 + 2, ntx - 1);
          auto node_pair = [&](const T* buf, int field, int L) -> float2 {
            const int r = (eb + ((L >> 1) & 1)) * ntx + field * nt;
            return (L & 1) ? make_float2(buf[r + ea0 + 1], buf[r + cb]) : make_float2(buf[r + ea0], buf[r + ea0 + 1]);
          };
          const bool ownA = va && ea0 >= 1 && eb >= 1 && kk >= 1 && i0 - 1 + ea0 < g.rx && j0 - 1 + eb < g.ry;
          const bool ownB = vb && eb >= 1 && kk >= 1 && i0 + ea0 < g.rx && j0 - 1 + eb < g.ry;
          const float2 own2 = make_float2(ownA ? 1.f : 0.f, ownB ? 1.f : 0.f);
          float2 gv[8];
          if (SLOT) {
            if (a.gq) {
#pragma unroll
              for (int q = 0; q < 8; ++q)
                gv[q] = make_float2(va ? __ldg(a.gq + 8 * ea_g + q) : 0.f, vb ? __ldg(a.gq + 8 * eb_g + q) : 0.f);
            } else if (d) {
              float2 dd[8], dq[8];
#pragma unroll
              for (int L = 0; L < 8; ++L) dd[L] = node_pair((L & 4) ? b1 : b0, 3, L);
              interp_p(dd, k2.c1, k2.c2, dq);
              const float2 om = bc2(1.f - m.kappa), kap = bc2(m.kappa), one = bc2(1.f);
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const float2 o = sub2(one, dq[q]);
                gv[q] = fma2(mul2(om, o), o, kap);
              }
            } else {
#pragma unroll
              for (int q = 0; q < 8; ++q) gv[q] = bc2(1.f);
            }
          }
          float2 D[3][3][2][2];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float2 u[8];
#pragma unroll
            for (int L = 0; L < 8; ++L) u[L] = node_pair((L & 4) ? b1 : b0, c, L);
            grad_p(u, k2, D[c][0], D[c][1], D[c][2]);
          }
          if (EROWS) {
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                D[0][0][i][j] = add2(D[0][0][i][j], bc2(E6[0]));
                D[1][1][i][j] = add2(D[1][1][i][j], bc2(E6[1]));
                D[2][2][i][j] = add2(D[2][2][i][j], bc2(E6[2]));
                D[1][2][i][j] = add2(D[1][2][i][j], bc2(E6[3]));
                D[0][2][i][j] = add2(D[0][2][i][j], bc2(E6[4]));
                D[0][1][i][j] = add2(D[0][1][i][j], bc2(E6[5]));
              }
          }
          float2 P[3][3][2][2];
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
              for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) P[c][b][i][j] = bc2(0.f);
          float2 en = bc2(0.f);
          float2 lw = bc2(0.f), mw = bc2(0.f);
          float2 lm[kStageQP];
          if constexpr (COEF == kCoefIso) {
            lw = make_float2(m.lam[sla] * w, m.lam[slb] * w);
            mw = make_float2(m.mu[sla] * w, m.mu[slb] * w);
          } else {
            T la[kStageQP], lb[kStageQP];
            const unsigned char* qs = QS + (size_t)(kk & 1) * kQChunks * exy * 16;
            if (q_async) {
              load_chunks<T, kStageQP>(qs, exy, ida, la);
              if (has_b) load_chunks<T, kStageQP>(qs, exy, idb, lb);
            } else {
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                la[q] = va ? __ldg(a.lam_q + 8 * ea_g + q) : 0.f;
                la[8 + q] = va ? __ldg(a.mu_q + 8 * ea_g + q) : 0.f;
                lb[q] = vb ? __ldg(a.lam_q + 8 * eb_g + q) : 0.f;
                lb[8 + q] = vb ? __ldg(a.mu_q + 8 * eb_g + q) : 0.f;
              }
            }
#pragma unroll
            for (int q = 0; q < kStageQP; ++q) lm[q] = make_float2(la[q] * w, has_b ? lb[q] * w : 0.f);
          }
#pragma unroll
          for (int qz = 0; qz < 2; ++qz)
#pragma unroll
            for (int qy = 0; qy < 2; ++qy)
#pragma unroll
              for (int qx = 0; qx < 2; ++qx) {
                const int q = qx + 2 * qy + 4 * qz;
                float2 ep[6];
                ep[0] = D[0][0][qz][qy];
                ep[1] = D[1][1][qz][qx];
                ep[2] = D[2][2][qy][qx];
                ep[3] = add2(D[1][2][qy][qx], D[2][1][qz][qx]);
                ep[4] = add2(D[0][2][qy][qx], D[2][0][qz][qy]);
                ep[5] = add2(D[0][1][qz][qx], D[1][0][qz][qy]);
                float2 lg, mg;
                if constexpr (COEF == kCoefIso) {
                  lg = mul2(lw, gv[q]);
                  mg = mul2(mw, gv[q]);
                } else {
                  lg = lm[q];
                  mg = lm[8 + q];
                }
                const float2 mg2 = add2(mg, mg);
                const float2 lt = mul2(lg, add2(add2(ep[0], ep[1]), ep[2]));
                float2 sg[6];
                sg[0] = fma2(mg2, ep[0], lt);
                sg[1] = fma2(mg2, ep[1], lt);
                sg[2] = fma2(mg2, ep[2], lt);
                sg[3] = mul2(mg, ep[3]);
                sg[4] = mul2(mg, ep[4]);
                sg[5] = mul2(mg, ep[5]);
                if (ENERGY) {
#pragma unroll
                  for (int k = 0; k < 6; ++k) en = fma2(sg[k], ep[k], en);
                }
                P[0][0][qz][qy] = add2(P[0][0][qz][qy], sg[0]);
                P[0][1][qz][qx] = add2(P[0][1][qz][qx], sg[5]);
                P[0][2][qy][qx] = add2(P[0][2][qy][qx], sg[4]);
                P[1][0][qz][qy] = add2(P[1][0][qz][qy], sg[5]);
                P[1][1][qz][qx] = add2(P[1][1][qz][qx], sg[1]);
                P[1][2][qy][qx] = add2(P[1][2][qy][qx], sg[3]);
                P[2][0][qz][qy] = add2(P[2][0][qz][qy], sg[4]);
                P[2][1][qz][qx] = add2(P[2][1][qz][qx], sg[3]);
                P[2][2][qy][qx] = add2(P[2][2][qy][qx], sg[2]);
              }
          if (ENERGY) tacc[kOutEnergy] += 0.5f * hsum(en, own2);
          if (EROWS) {
            float2 s[6] = {bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f)};
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                s[0] = add2(s[0], P[0][0][i][j]);
                s[1] = add2(s[1], P[1][1][i][j]);
                s[2] = add2(s[2], P[2][2][i][j]);
                s[3] = add2(s[3], P[1][2][i][j]);
                s[4] = add2(s[4], P[0][2][i][j]);
                s[5] = add2(s[5], P[0][1][i][j]);
              }
#pragma unroll
            for (int k = 0; k < 6; ++k) tacc[k] += hsum(s[k], own2);
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) grad_p_t(P[c][0], P[c][1], P[c][2], k2, f[c]);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int L = 0; L < 8; ++L) f[c][L] = lane_sel(va, vb, f[c][L]);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int L = 0; L < 8; ++L) f[c][L] = bc2(0.f);
        }
#pragma unroll
        for (int L = 0; L < 4; ++L)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            FL[(L * 3 + c) * exy + ida] = f[c][L].x;
            FU[(L * 3 + c) * exy + ida] = f[c][L + 4].x;
            if (has_b) {
              FL[(L * 3 + c) * exy + idb] = f[c][L].y;
              FU[(L * 3 + c) * exy + idb] = f[c][L + 4].y;
            }
          }
      }
      __syncthreads();
      if constexpr (STAGE) cp_async_wait<1>();
      // ---- node phase: nodes ni0, ni0 + 1 of row nj
      if (is_npair) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int ni = ni0 + h;
          const int e11 = (ni + 1) + ex * (nj + 1), e01 = ni + ex * (nj + 1);
          const int e10 = (ni + 1) + ex * nj, e00 = ni + ex * nj;
          T lo[3], up[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            lo[c] = FL[(0 * 3 + c) * exy + e11] + FL[(1 * 3 + c) * exy + e01] + FL[(2 * 3 + c) * exy + e10] +
                    FL[(3 * 3 + c) * exy + e00];
            up[c] = FU[(0 * 3 + c) * exy + e11] + FU[(1 * 3 + c) * exy + e01] + FU[(2 * 3 + c) * exy + e10] +
                    FU[(3 * 3 + c) * exy + e00];
          }
          const int gi = i0 + ni, gj = j0 + nj;
          if (kk >= 1 && gi < g.rx && gj < g.ry) {
            const size_t n = (size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * ke);
            const int nid = nj * ox + ni;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              T v = pend[h][c] + lo[c];
              if (mk_cur[h] & (1 << c)) v = T(0);
              const size_t i = 3 * n + c;
              const T xin = b0[c * nt + (nj + 1) * ntx + ni + 1];
              if (CHEB) {
                const T* cs = CS + (size_t)(kk & 1) * 9 * oxy + nid;
                const T r = cs[c * oxy] - v;
                a.res[i] = r;
                const T dn = c1 * xin + c2 * cs[(3 + c) * oxy] * r;
                a.d_out[i] = dn;
                a.xs[i] = cs[(6 + c) * oxy] + dn;
              } else {
                if (a.y) a.y[i] = v;
                if (DOT) tacc[kOutDot] += xin * v;
              }
            }
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) pend[h][c] = up[c];
        }
      }
    }
    if (RED) {
#pragma unroll
      for (int k = 0; k < 8; ++k) accd[k] += double(tacc[k]);
    }
  }

  if constexpr (RED) {
    constexpr int NK = DOT ? 8 : (ENERGY ? 7 : 6);
    __shared__ double sh[32 * NK];
    double v[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) v[k] = accd[k];
    block_sum_multi<NK>(v, sh);
    if (tid == 0) {
#pragma unroll
      for (int k = 0; k < NK; ++k) a.ws.part[k * kMaxPartials + blockIdx.x] = v[k];
    }
    if (arrive_last(a.ws.counter)) {
      double fsum[NK];
      fold_sum_multi<NK>(a.ws.part, kMaxPartials, gridDim.x, fsum, sh);
      if (tid == 0) {
        double dot_e = 0.0;
#pragma unroll
        for (int k = 0; k < NK; ++k) {
          const double t = fsum[k];
          if (k < 6) {
            a.ws.out[k] = t;
            const size_t idx = 3 * (size_t)g.n_red + k;
            const T yv = (a.mask && a.mask[idx]) ? T(0) : T(t);
            if (a.y) a.y[idx] = yv;
            dot_e += double(x[idx]) * double(yv);
          } else if (k == kOutEnergy) {
            a.ws.out[k] = t;
          } else {
            a.ws.out[k] = t + dot_e;
          }
        }
        *a.ws.counter = 0u;
      }
    }
  }
}
