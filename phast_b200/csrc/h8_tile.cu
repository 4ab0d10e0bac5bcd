// Tiled z-marching voxel H8 elastic action (see h8_tile.cuh).
#include "h8_tile.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include "engine.cuh"

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

namespace phastb {

namespace {

// Index of a node coordinate along one axis after the periodic wrap; -1 when
// the coordinate lies outside a non-periodic grid.  |c| stays within one
// period because tiles are never wider than the grid.
__device__ __forceinline__ int wrap_node(int c, int n, int r, int periodic) {
  if (periodic) return c < 0 ? c + n : (c >= n ? c - n : c);
  return (c >= 0 && c < r) ? c : -1;
}

__device__ __forceinline__ int wrap_elem(int c, int n, int periodic) {
  if (periodic) return c < 0 ? c + n : (c >= n ? c - n : c);
  return (c >= 0 && c < n) ? c : -1;
}

// Asynchronous global -> shared copies (cp.async, 16 bytes, L2 only).  A thread
// stages the per-element arrays of the NEXT element layer into its own slot of
// a two-buffer shared array and waits for its own group before reading it, so
// no barrier is needed for these slots; both addresses must be 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// One word (4 or 8 bytes, naturally aligned) with cp.async.
template <typename T>
__device__ __forceinline__ void cp_async_word(T* smem, const T* gmem) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async copies 4, 8 or 16 bytes");
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- TMA staging of node layers (cp.async.bulk.tensor, completion on an mbarrier)
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Orders this thread's earlier generic-proxy accesses of shared memory (reads of
// a buffer, stores of patched halo values) before async-proxy (TMA) writes.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// 3D tiled copy global -> this CTA's shared memory (no multicast); the innermost
// coordinate c0 times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
// A TMA completion wait gives up after kTmaLimitNs of global time (a normal wait
// is well under a microsecond); the caller then marks its output non-finite.
constexpr unsigned long long kTmaLimitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;  // the usual case: the copy landed during the last layer
  const unsigned long long t0 = global_ns();
  for (unsigned i = 0; i < (1u << 26); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 63u && global_ns() - t0 > kTmaLimitNs) return false;
  }
  return false;
}
__device__ __forceinline__ int floor_mult(int v, int m) { return (v >= 0 ? v / m : -((-v + m - 1) / m)) * m; }

// Staged per-element arrays live chunk-major in shared memory: chunk c (16
// bytes) of the element owned by thread t sits at base + (c * n + t) * 16, so a
// warp reading one chunk touches consecutive 16-byte units (no bank conflicts).
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
};
template <>
struct Vec16<double> {
  using type = double2;
};

// Copies n_chunks 16-byte chunks of src into chunks c0.. of thread t's column.
__device__ __forceinline__ void stage_chunks(unsigned char* base, int n, int t, int c0, const void* src,
                                             int n_chunks) {
  for (int c = 0; c < n_chunks; ++c)
    cp_async16(base + ((size_t)(c0 + c) * n + t) * 16, static_cast<const unsigned char*>(src) + 16 * c);
}

// Reads W words of thread t's staged column (W * sizeof(T) a multiple of 16).
template <typename T, int W>
__device__ __forceinline__ void load_chunks(const unsigned char* base, int n, int t, T (&out)[W]) {
  using V = typename Vec16<T>::type;
  constexpr int per = 16 / sizeof(T);
#pragma unroll
  for (int c = 0; c < W / per; ++c) {
    const V v = *reinterpret_cast<const V*>(base + ((size_t)c * n + t) * 16);
    const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
    for (int j = 0; j < per; ++j) out[c * per + j] = pv[j];
  }
}

// Node layer kn of the brick with its one-node halo, (ox+2)(oy+2) nodes, is
// staged in two steps so the global loads of layer k+2 are in flight while
// layer k's elements are computed: stage_load reads a thread's (at most two)
// nodes into registers, stage_store writes them to buf[4][nt] (fields ux, uy,
// uz, d).  Nodes outside a non-periodic grid read as zero.
template <typename T>
struct Staged {
  T v[2][4];
};

template <typename T>
__device__ __forceinline__ void stage_load(const VoxGeom& g, const T* __restrict__ x, const T* __restrict__ d,
                                           int i0, int j0, int kn, int ntx, int nt, Staged<T>& r) {
  const int gk = wrap_node(kn, g.nz, g.rz, g.pz);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int t = threadIdx.x + h * blockDim.x;
    T u0 = T(0), u1 = T(0), u2 = T(0), dd = T(0);
    if (t < nt && gk >= 0) {
      const int a = t % ntx, b = t / ntx;
      const int gi = wrap_node(i0 - 1 + a, g.nx, g.rx, g.px);
      const int gj = wrap_node(j0 - 1 + b, g.ny, g.ry, g.py);
      if (gi >= 0 && gj >= 0) {
        const size_t n = (size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * gk);
        u0 = __ldg(x + 3 * n);
        u1 = __ldg(x + 3 * n + 1);
        u2 = __ldg(x + 3 * n + 2);
        if (d) dd = __ldg(d + n);
      }
    }
    r.v[h][0] = u0;
    r.v[h][1] = u1;
    r.v[h][2] = u2;
    r.v[h][3] = dd;
  }
}

template <typename T>
__device__ __forceinline__ void stage_store(int nt, const Staged<T>& r, T* buf) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int t = threadIdx.x + h * blockDim.x;
    if (t < nt) {
      buf[t] = r.v[h][0];
      buf[nt + t] = r.v[h][1];
      buf[2 * nt + t] = r.v[h][2];
      buf[3 * nt + t] = r.v[h][3];
    }
  }
}


template <typename T>
__device__ __forceinline__ void ip2(T a0, T a1, T c1, T c2, T& q0, T& q1) {
  q0 = c1 * a0 + c2 * a1;
  q1 = c2 * a0 + c1 * a1;
}

// Gradient of a trilinear field u[L] at the Gauss points: Dx[qz][qy],
// Dy[qz][qx], Dz[qy][qx] (each independent of its own axis).
template <typename T>
__device__ __forceinline__ void grad_k(const T* u, const TileK<T>& k, T (&Dx)[2][2], T (&Dy)[2][2],
                                       T (&Dz)[2][2]) {
  {
    T Y[2][2];  // [az][qy]
#pragma unroll
    for (int az = 0; az < 2; ++az)
      ip2(u[1 + 4 * az] - u[4 * az], u[3 + 4 * az] - u[2 + 4 * az], k.c1, k.c2, Y[az][0], Y[az][1]);
#pragma unroll
    for (int qy = 0; qy < 2; ++qy) ip2(Y[0][qy], Y[1][qy], k.x1, k.x2, Dx[0][qy], Dx[1][qy]);
  }
  {
    T Y[2][2];  // [az][qx]
#pragma unroll
    for (int az = 0; az < 2; ++az)
      ip2(u[2 + 4 * az] - u[4 * az], u[3 + 4 * az] - u[1 + 4 * az], k.c1, k.c2, Y[az][0], Y[az][1]);
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2(Y[0][qx], Y[1][qx], k.y1, k.y2, Dy[0][qx], Dy[1][qx]);
  }
  {
    T Y[2][2];  // [ay][qx]
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
      ip2(u[4 + 2 * ay] - u[2 * ay], u[5 + 2 * ay] - u[1 + 2 * ay], k.c1, k.c2, Y[ay][0], Y[ay][1]);
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2(Y[0][qx], Y[1][qx], k.z1, k.z2, Dz[0][qx], Dz[1][qx]);
  }
}

// Transposed gradient: out[L] = sum over the Gauss points of dN_L/dx_a times
// the summed terms Px[qz][qy], Py[qz][qx], Pz[qy][qx].
template <typename T>
__device__ __forceinline__ void grad_k_t(const T (&Px)[2][2], const T (&Py)[2][2], const T (&Pz)[2][2],
                                         const TileK<T>& k, T* out) {
  T Ax[2][2], Ay[2][2], Az[2][2];
  {
    T Y[2][2];  // [az][qy]
#pragma unroll
    for (int qy = 0; qy < 2; ++qy) ip2(Px[0][qy], Px[1][qy], k.x1, k.x2, Y[0][qy], Y[1][qy]);
#pragma unroll
    for (int az = 0; az < 2; ++az) ip2(Y[az][0], Y[az][1], k.c1, k.c2, Ax[az][0], Ax[az][1]);  // [az][ay]
  }
  {
    T Y[2][2];  // [az][qx]
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2(Py[0][qx], Py[1][qx], k.y1, k.y2, Y[0][qx], Y[1][qx]);
#pragma unroll
    for (int az = 0; az < 2; ++az) ip2(Y[az][0], Y[az][1], k.c1, k.c2, Ay[az][0], Ay[az][1]);  // [az][ax]
  }
  {
    T Y[2][2];  // [ay][qx]
#pragma unroll
    for (int qx = 0; qx < 2; ++qx) ip2(Pz[0][qx], Pz[1][qx], k.z1, k.z2, Y[0][qx], Y[1][qx]);
#pragma unroll
    for (int ay = 0; ay < 2; ++ay) ip2(Y[ay][0], Y[ay][1], k.c1, k.c2, Az[ay][0], Az[ay][1]);  // [ay][ax]
  }
#pragma unroll
  for (int L = 0; L < 8; ++L) {
    const int ax = L & 1, ay = (L >> 1) & 1, az = L >> 2;
    const T tx = ax ? Ax[az][ay] : -Ax[az][ay];
    const T ty = ay ? Ay[az][ax] : -Ay[az][ax];
    const T tz = az ? Az[ay][ax] : -Az[ay][ax];
    out[L] = tx + ty + tz;
  }
}

template <typename T>
__device__ __forceinline__ T g_deg(T kappa, T d) {
  const T o = T(1) - d;
  return (T(1) - kappa) * o * o + kappa;
}

}  // namespace

// One launch = every brick of the grid (persistent blocks).  COEF selects the
// element coefficients (material slot + g(d), isotropic or general Voigt, or
// per-Gauss-point moduli of a multigrid coarse level); MODE selects the node
// epilogue: y = A x, y plus x . y, y plus the energy, or one Chebyshev
// smoothing step on (res, d, x) driven by A d.
// TMA: the node layers are staged by tensor-map copies (tmx: u~ as a (3 rx,
// ry, rz) array, tmd: d as (rx, ry, rz)) issued by one thread and completed on an
// mbarrier per layer buffer; halo nodes that wrap around a periodic edge read
// the zero fill and are patched by per-thread loads.  Otherwise every thread
// stages its (at most two) halo-tile nodes through registers.
// The action over the bricks vb, vb + vgrid, ... of one grid: a plain launch runs it with
// its block index and grid size, a batched launch with the block's virtual index inside its cell.
template <typename T, int COEF, int MODE, int OX, int OY, bool TMA>
__device__ __forceinline__ void tile_body(const TileArgs<T>& a, const VoxMat<T>& m, const CUtensorMap* tmx,
                                          const CUtensorMap* tmd, const int vb, const int vgrid) {
  if (a.guard && *a.guard == 0) return;
  constexpr bool SLOT = COEF != kCoefQP;
  constexpr bool DOT = MODE == kModeDot, ENERGY = MODE == kModeEnergy, CHEB = MODE == kModeCheb;
  // E rows (macro strain) exist on the fine operator; a Chebyshev step and a
  // nodal-block action leave them alone (masked)
  constexpr bool NODAL = MODE == kModeNodal;
  constexpr bool EROWS = SLOT && !CHEB && !NODAL;
  constexpr bool RED = EROWS || DOT || ENERGY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const VoxGeom& g = a.g;
  if (NODAL && vb == 0 && threadIdx.x < 6 && a.y) a.y[3 * (size_t)g.n_red + threadIdx.x] = T(0);
  const T* __restrict__ x = a.x;
  const T* __restrict__ d = SLOT ? a.d : nullptr;
  // OX, OY > 0: a compiled tile shape (constant shared-memory offsets)
  const int ox = OX ? OX : a.ts.ox, oy = OY ? OY : a.ts.oy, kz = a.ts.kz;
  const int ex = ox + 1, exy = ex * (oy + 1);
  const int ntx = ox + 2, nt = ntx * (oy + 2);
  // TMA: shared memory from a 128-byte boundary; u~ layer buffers of W words per
  // halo row, d layer buffers of Wd words, each started from a 16-byte aligned column
  unsigned char* sbase =
      TMA ? reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127))
          : smem_raw;
  const int W = tma_wx<T>(ox), Wd = tma_wd<T>(ox);
  const size_t xbb = tma_xbytes<T>(ox, oy), dbb = tma_dbytes<T>(ox, oy);
  T* nb = reinterpret_cast<T*>(sbase);  // [3 buffers][4 fields][nt] (without TMA)
  size_t off_face = 0, off_qp = 0, off_cheb = 0;
  if (TMA) {
    tile_layout_tma<T>(ox, oy, COEF == kCoefQP, CHEB, &off_face, &off_qp, &off_cheb);
  } else {
    tile_layout<T>(ox, oy, COEF == kCoefQP, CHEB, &off_qp, &off_cheb);
    off_face = sizeof(T) * 12 * (size_t)nt;
  }
  T* FL = reinterpret_cast<T*>(sbase + off_face);  // [4 corners][3 comps][exy], lower face (oz = 0)
  T* FU = FL + 12 * exy;                           // upper face (oz = 1)
  // staged by cp.async, two buffers each: kCoefQP (lam_q, mu_q) of this thread's
  // element one element layer ahead, chunk-major [2][chunks][exy]; kModeCheb
  // (res, invd, xs) of this thread's owned node, [2][9][ox*oy], copied while the
  // layer's elements are computed
  constexpr bool STAGE = COEF == kCoefQP || CHEB;
  constexpr int kQChunks = kStageQP * (int)sizeof(T) / 16;
  unsigned char* QS = sbase + off_qp;
  T* CS = reinterpret_cast<T*>(sbase + off_cheb);
  __shared__ __align__(8) unsigned long long s_mbar[3];
  unsigned mphase = 0;  // bit b: parity of the next completion of buffer b's barrier
  bool tma_fault = false;
  const bool use_d = SLOT && d != nullptr && a.gq == nullptr;
  const unsigned tma_tx = (unsigned)(sizeof(T) * (size_t)W * (oy + 2) + (use_d ? sizeof(T) * (size_t)Wd * (oy + 2) : 0));
  if (TMA) {
    if (threadIdx.x == 0) {
      for (int b = 0; b < 3; ++b) mbar_init(&s_mbar[b], 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  const int oxy = ox * oy;
  const bool q_async = COEF == kCoefQP && aligned16(a.lam_q) && aligned16(a.mu_q);
  const int tid = threadIdx.x;
  const T w = T(g.w);
  const T c1 = T(a.c1), c2 = T(a.c2);
  T E6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  if (EROWS) {  // a Chebyshev step smooths the nodal block only (E rows masked)
    const T* Ex = x + 3 * (size_t)g.n_red;
#pragma unroll
    for (int k = 0; k < 6; ++k) E6[k] = __ldg(Ex + k);
  }
  const int tiles_x = (g.rx + ox - 1) / ox, tiles_y = (g.ry + oy - 1) / oy;
  const int tiles_xy = tiles_x * tiles_y;
  const int n_tiles = tiles_xy * ((g.rz + kz - 1) / kz);
  // element / owned-node coordinates of this thread inside the tile
  const int ea = tid % ex, eb = tid / ex;
  const int ni = tid % ox, nj = tid / ox;
  const bool is_elem = tid < exy, is_node = tid < ox * oy;
  constexpr int kA = 16 / (int)sizeof(T);  // words per 16 bytes
  int xr = 0, dr = 0, xs0 = 0, ds0 = 0;    // TMA: row start columns and remainders of the current tile
  // node value of component c (3: d) at halo-tile position (row, col) of layer buffer `buf`
  auto nval = [&](int buf, int c, int row, int col) -> T {
    if constexpr (TMA) {
      if (c < 3) return reinterpret_cast<const T*>(sbase + (size_t)buf * xbb)[row * W + xr + 3 * col + c];
      return reinterpret_cast<const T*>(sbase + 3 * xbb + (size_t)buf * dbb)[row * Wd + dr + col];
    } else {
      return nb[4 * nt * buf + c * nt + row * ntx + col];
    }
  };
  // TMA: thread 0 issues the copies of node layer kn into buffer b
  auto tma_issue = [&](int i0, int j0, int kn, int b) {
    if constexpr (TMA) {
      if (threadIdx.x == 0) {
        const int gz = g.pz ? wrap_node(kn, g.nz, g.rz, 1) : kn;  // out of range: the zero fill
        fence_proxy_async();
        mbar_expect_tx(&s_mbar[b], tma_tx);
        tma_load_3d(sbase + (size_t)b * xbb, tmx, xs0, j0 - 1, gz, &s_mbar[b]);
        if (use_d) tma_load_3d(sbase + 3 * xbb + (size_t)b * dbb, tmd, ds0, j0 - 1, gz, &s_mbar[b]);
      }
    }
  };
  // TMA: halo nodes of layer kn that wrap around a periodic edge (the copy read the zero fill there)
  auto wrap_load = [&](int i0, int j0, int kn, Staged<T>& r, unsigned& on) {
    on = 0;
    if constexpr (TMA) {
      const int gk = wrap_node(kn, g.nz, g.rz, g.pz);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = threadIdx.x + h * blockDim.x;
        if (t < nt && gk >= 0) {
          const int ri = i0 - 1 + t % ntx, rj = j0 - 1 + t / ntx;
          const bool wx = g.px && (ri < 0 || ri >= g.rx), wy = g.py && (rj < 0 || rj >= g.ry);
          if (wx || wy) {
            const int gi = wrap_node(ri, g.nx, g.rx, g.px), gj = wrap_node(rj, g.ny, g.ry, g.py);
            if (gi >= 0 && gj >= 0) {
              const size_t n = (size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * gk);
              r.v[h][0] = __ldg(x + 3 * n);
              r.v[h][1] = __ldg(x + 3 * n + 1);
              r.v[h][2] = __ldg(x + 3 * n + 2);
              r.v[h][3] = use_d ? __ldg(d + n) : T(0);
              on |= 1u << h;
            }
          }
        }
      }
    }
  };
  auto wrap_store = [&](const Staged<T>& r, unsigned on, int b) {
    if constexpr (TMA) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (on & (1u << h)) {
          const int t = threadIdx.x + h * blockDim.x, col = t % ntx, row = t / ntx;
          T* xbuf = reinterpret_cast<T*>(sbase + (size_t)b * xbb);
#pragma unroll
          for (int c = 0; c < 3; ++c) xbuf[row * W + xr + 3 * col + c] = r.v[h][c];
          if (use_d) reinterpret_cast<T*>(sbase + 3 * xbb + (size_t)b * dbb)[row * Wd + dr + col] = r.v[h][3];
        }
      }
      // these generic-proxy writes must be ordered before the tensor copy that later refills the buffer
      if (on) fence_proxy_async();
    }
  };
  // TMA: waits (bounded) for buffer b's copies of its current fill
  auto tma_wait = [&](int b) {
    if constexpr (TMA) {
      if (!mbar_wait(&s_mbar[b], (mphase >> b) & 1u)) tma_fault = true;
      mphase ^= 1u << b;
    }
  };
  double accd[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // material slot of this thread's element in layer ke (0 outside the grid)
  auto elem_slot = [&](int i0, int j0, int ke) -> int {
    if (!SLOT || !is_elem) return 0;
    const int gi = wrap_elem(i0 - 1 + ea, g.nx, g.px);
    const int gj = wrap_elem(j0 - 1 + eb, g.ny, g.py);
    const int gk = wrap_elem(ke, g.nz, g.pz);
    if (gi < 0 || gj < 0 || gk < 0) return 0;
    return __ldg(a.slot + (size_t)gi + (size_t)g.nx * ((size_t)gj + (size_t)g.ny * gk));
  };
  // fixed-dof bits (one per component) of this thread's owned node in layer kn
  auto node_mask = [&](int i0, int j0, int kn) -> int {
    if (!a.mask || !is_node || kn >= g.rz) return 0;
    const int gi = i0 + ni, gj = j0 + nj;
    if (gi >= g.rx || gj >= g.ry) return 0;
    const size_t n = (size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * kn);
    return (__ldg(a.mask + 3 * n) ? 1 : 0) | (__ldg(a.mask + 3 * n + 1) ? 2 : 0) |
           (__ldg(a.mask + 3 * n + 2) ? 4 : 0);
  };
  // Staging commit groups, in order: per step kk one Chebyshev group (node layer
  // ke) then one moduli group (element layer ke + 1), each possibly empty, so the
  // number of groups committed after any one of them is fixed.
  // kCoefQP: copies element layer ke's (lam_q, mu_q) into buffer `buf`.
  auto stage_qp = [&](int i0, int j0, int ke, int buf, bool live) {
    if constexpr (STAGE) {
      if (COEF == kCoefQP && live && q_async && is_elem) {
        const int gi = wrap_elem(i0 - 1 + ea, g.nx, g.px);
        const int gj = wrap_elem(j0 - 1 + eb, g.ny, g.py);
        const int gk = wrap_elem(ke, g.nz, g.pz);
        if (gi >= 0 && gj >= 0 && gk >= 0) {
          const size_t e = (size_t)gi + (size_t)g.nx * ((size_t)gj + (size_t)g.ny * gk);
          unsigned char* dst = QS + (size_t)buf * kQChunks * exy * 16;
          stage_chunks(dst, exy, tid, 0, a.lam_q + 8 * e, kQChunks / 2);
          stage_chunks(dst, exy, tid, kQChunks / 2, a.mu_q + 8 * e, kQChunks / 2);
        }
      }
      cp_async_commit();
    }
  };
  // kModeCheb: copies (res, invd, xs) of the owned node in node layer kn into buffer `buf`.
  auto stage_cheb = [&](int i0, int j0, int kn, int buf, bool live) {
    if constexpr (STAGE) {
      const int gi = i0 + ni, gj = j0 + nj;
      if (CHEB && live && is_node && gi < g.rx && gj < g.ry) {
        const size_t n3 = 3 * ((size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * kn));
        T* dst = CS + (size_t)buf * 9 * oxy + tid;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cp_async_word(dst + c * oxy, a.res + n3 + c);
          cp_async_word(dst + (3 + c) * oxy, a.invd + n3 + c);
          cp_async_word(dst + (6 + c) * oxy, a.xs + n3 + c);
        }
      }
      cp_async_commit();
    }
  };

  for (int tile = vb; tile < n_tiles; tile += vgrid) {
    const int tz = tile / tiles_xy, txy = tile - tz * tiles_xy;
    const int i0 = (txy % tiles_x) * ox, j0 = (txy / tiles_x) * oy;
    const int k0 = tz * kz, k1 = min(k0 + kz, g.rz);
    T tacc[8] = {T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0)};
    T pend[3] = {T(0), T(0), T(0)};
    Staged<T> pf;
    unsigned pf_on = 0;
    if constexpr (TMA) {
      xs0 = floor_mult(3 * (i0 - 1), kA);
      xr = 3 * (i0 - 1) - xs0;
      ds0 = floor_mult(i0 - 1, kA);
      dr = (i0 - 1) - ds0;
      __syncthreads();  // the previous tile's last node phase is done with the buffers
      tma_issue(i0, j0, k0 - 1, 0);
      tma_issue(i0, j0, k0, 1);
      wrap_load(i0, j0, k0 - 1, pf, pf_on);
      tma_wait(0);
      wrap_store(pf, pf_on, 0);
      wrap_load(i0, j0, k0, pf, pf_on);
    } else {
      stage_load(g, x, d, i0, j0, k0 - 1, ntx, nt, pf);
      __syncthreads();  // the previous tile's last node phase is done with the buffers
      stage_store(nt, pf, nb);
      stage_load(g, x, d, i0, j0, k0, ntx, nt, pf);
    }
    int sl_next = elem_slot(i0, j0, k0 - 1);
    stage_qp(i0, j0, k0 - 1, 0, true);
    int mk_next = node_mask(i0, j0, k0), mk_cur = 0;
    const int K = k1 - k0;
    for (int kk = 0; kk <= K; ++kk) {
      const int ke = k0 - 1 + kk;  // element layer of this step
      const int ib0 = kk % 3, ib1 = (kk + 1) % 3;
      if constexpr (TMA) {
        tma_wait(ib1);  // node layer ke + 1
        wrap_store(pf, pf_on, ib1);
      } else {
        stage_store(nt, pf, nb + 4 * nt * ib1);  // node layer ke + 1
      }
      const int sl = sl_next;
      if (kk < K) {
        if constexpr (TMA)
          wrap_load(i0, j0, ke + 2, pf, pf_on);
        else
          stage_load(g, x, d, i0, j0, ke + 2, ntx, nt, pf);
        sl_next = elem_slot(i0, j0, ke + 1);
      }
      if constexpr (STAGE) {
        stage_cheb(i0, j0, ke, kk & 1, kk >= 1);
        stage_qp(i0, j0, ke + 1, (kk + 1) & 1, kk < K);
        cp_async_wait<2>();  // this thread's moduli of element layer ke have landed
      }
      if (kk >= 1) {
        mk_cur = mk_next;
        if (kk < K) mk_next = node_mask(i0, j0, ke + 1);
      }
      __syncthreads();
      // every thread is done with buffer (kk + 2) % 3 (node layer ke - 1): refill it with layer ke + 2
      if (kk < K) tma_issue(i0, j0, ke + 2, (kk + 2) % 3);
      // ---- element phase: one element of the (ox+1) x (oy+1) tile per thread
      if (is_elem) {
        const int gi = wrap_elem(i0 - 1 + ea, g.nx, g.px);
        const int gj = wrap_elem(j0 - 1 + eb, g.ny, g.py);
        const int gk = wrap_elem(ke, g.nz, g.pz);
        T f[3][8];
        if (gi >= 0 && gj >= 0 && gk >= 0) {
          const size_t e = (size_t)gi + (size_t)g.nx * ((size_t)gj + (size_t)g.ny * gk);
          const bool own = ea >= 1 && eb >= 1 && kk >= 1 && i0 - 1 + ea < g.rx && j0 - 1 + eb < g.ry;
          T gv[8];
          if (SLOT) {
            if (a.gq) {
#pragma unroll
              for (int q = 0; q < 8; ++q) gv[q] = __ldg(a.gq + 8 * e + q);
            } else if (d) {
              T dd[8], dq[8];
#pragma unroll
              for (int L = 0; L < 8; ++L) dd[L] = nval((L & 4) ? ib1 : ib0, 3, eb + ((L >> 1) & 1), ea + (L & 1));
              interp_sf(dd, dq);
#pragma unroll
              for (int q = 0; q < 8; ++q) gv[q] = g_deg(m.kappa, dq[q]);
            } else {
#pragma unroll
              for (int q = 0; q < 8; ++q) gv[q] = T(1);
            }
          }
          T D[3][3][2][2];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            T u[8];
#pragma unroll
            for (int L = 0; L < 8; ++L) u[L] = nval((L & 4) ? ib1 : ib0, c, eb + ((L >> 1) & 1), ea + (L & 1));
            grad_k(u, a.k, D[c][0], D[c][1], D[c][2]);
          }
          if (EROWS) {
            // the macro strain enters each strain component once: fold it into
            // the gradient term that component starts from
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                D[0][0][i][j] += E6[0];
                D[1][1][i][j] += E6[1];
                D[2][2][i][j] += E6[2];
                D[1][2][i][j] += E6[3];
                D[0][2][i][j] += E6[4];
                D[0][1][i][j] += E6[5];
              }
          }
          T P[3][3][2][2];
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
              for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) P[c][b][i][j] = T(0);
          // w * g_q * sigma_q at the eight Gauss points, summed into the P terms
          auto qp_loop = [&](auto stress) {
#pragma unroll
            for (int qz = 0; qz < 2; ++qz)
#pragma unroll
              for (int qy = 0; qy < 2; ++qy)
#pragma unroll
                for (int qx = 0; qx < 2; ++qx) {
                  T ep[6];
                  ep[0] = D[0][0][qz][qy];
                  ep[1] = D[1][1][qz][qx];
                  ep[2] = D[2][2][qy][qx];
                  ep[3] = D[1][2][qy][qx] + D[2][1][qz][qx];
                  ep[4] = D[0][2][qy][qx] + D[2][0][qz][qy];
                  ep[5] = D[0][1][qz][qx] + D[1][0][qz][qy];
                  T sg[6];
                  stress(ep, qx + 2 * qy + 4 * qz, sg);
                  if (ENERGY && own) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) tacc[kOutEnergy] += T(0.5) * sg[k] * ep[k];
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
          };
          auto iso_stress = [&](const T* ep, T lg, T mg, T* sg) {
            const T mg2 = mg + mg;
            const T lt = lg * (ep[0] + ep[1] + ep[2]);
            sg[0] = mg2 * ep[0] + lt;
            sg[1] = mg2 * ep[1] + lt;
            sg[2] = mg2 * ep[2] + lt;
            sg[3] = mg * ep[3];
            sg[4] = mg * ep[4];
            sg[5] = mg * ep[5];
          };
          if constexpr (COEF == kCoefIso) {
            const T lw = m.lam[sl] * w, mw = m.mu[sl] * w;
            qp_loop([&](const T* ep, int q, T* sg) { iso_stress(ep, lw * gv[q], mw * gv[q], sg); });
          } else if constexpr (COEF == kCoefAniso) {
            qp_loop([&](const T* ep, int q, T* sg) {
              voigt_stress(m, sl, ep, sg);
              const T gw = gv[q] * w;
#pragma unroll
              for (int k = 0; k < 6; ++k) sg[k] *= gw;
            });
          } else {
            T lm[kStageQP];  // lam_q[0..7], mu_q[0..7]
            if (q_async) {
              load_chunks<T, kStageQP>(QS + (size_t)(kk & 1) * kQChunks * exy * 16, exy, tid, lm);
            } else {
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                lm[q] = __ldg(a.lam_q + 8 * e + q);
                lm[8 + q] = __ldg(a.mu_q + 8 * e + q);
              }
            }
            qp_loop([&](const T* ep, int q, T* sg) { iso_stress(ep, lm[q] * w, lm[8 + q] * w, sg); });
          }
          if (EROWS && own) {
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                tacc[0] += P[0][0][i][j];
                tacc[1] += P[1][1][i][j];
                tacc[2] += P[2][2][i][j];
                tacc[3] += P[1][2][i][j];
                tacc[4] += P[0][2][i][j];
                tacc[5] += P[0][1][i][j];
              }
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) grad_k_t(P[c][0], P[c][1], P[c][2], a.k, f[c]);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int L = 0; L < 8; ++L) f[c][L] = T(0);
        }
#pragma unroll
        for (int L = 0; L < 4; ++L)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            FL[(L * 3 + c) * exy + tid] = f[c][L];
            FU[(L * 3 + c) * exy + tid] = f[c][L + 4];
          }
      }
      __syncthreads();
      if constexpr (STAGE) cp_async_wait<1>();  // this thread's (res, invd, xs) of node layer ke
      // ---- node phase: node layer ke = lower faces of this layer + upper faces of the previous
      if (is_node) {
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
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            T v = pend[c] + lo[c];
            if (mk_cur & (1 << c)) v = T(0);
            const size_t i = 3 * n + c;
            const T xin = nval(ib0, c, nj + 1, ni + 1);
            if (CHEB) {
              const T* cs = CS + (size_t)(kk & 1) * 9 * oxy + tid;
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
        for (int c = 0; c < 3; ++c) pend[c] = up[c];
      }
    }
    if (RED) {
#pragma unroll
      for (int k = 0; k < 8; ++k) accd[k] += double(tacc[k]);
    }
  }
  if (TMA && tma_fault) {
    // a layer copy did not complete in time: the result is unusable, so make it non-finite
    // (every solver reports PHASTB_NONFINITE for it) instead of returning wrong numbers
    const T bad = T(NAN);
    if (a.y) a.y[0] = bad;
    if (CHEB && a.res) a.res[0] = bad;
#pragma unroll
    for (int k = 0; k < 8; ++k) accd[k] = NAN;
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
      for (int k = 0; k < NK; ++k) a.ws.part[k * kMaxPartials + vb] = v[k];
    }
    if (arrive_last_n(a.ws.counter, vgrid)) {
      double f[NK];
      fold_sum_multi<NK>(a.ws.part, kMaxPartials, vgrid, f, sh);
      if (tid == 0) {
        double dot_e = 0.0;
#pragma unroll
        for (int k = 0; k < NK; ++k) {
          const double t = f[k];
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

template <typename T, int COEF, int MODE, int OX, int OY, bool TMA>
__global__ void __launch_bounds__(kTileMaxThreads, sizeof(T) == 4 ? 2 : 1)
    h8_tile_kernel(TileArgs<T> a, VoxMat<T> m, const __grid_constant__ CUtensorMap tmx,
                   const __grid_constant__ CUtensorMap tmd) {
  tile_body<T, COEF, MODE, OX, OY, TMA>(a, m, &tmx, &tmd, blockIdx.x, gridDim.x);
}

#include "h8_tile2.cuh"

// ------------------------------------------------------------------ damage action

// Scalar AT2 damage action on the same brick schedule:
//   y = scale * [Gc_e (M / ell + ell L) d + 2 (1 - kappa) sum_q w H_q N_q N_q^T d]
// (the element arithmetic of h8_damage_elem_kernel), masked rows zero.  One
// pass covers every brick of this (persistent) block: node values come from
// node_val(n), each owned node's result goes to on_owned(n, x_n, y_n), and the
// return value is this thread's share of sum_n x_n y_n (with DOT).
template <typename T, int OX, int OY, bool DOT, class NodeVal, class OnOwned>
__device__ __forceinline__ double dtile_pass(const DTileArgs<T>& a, unsigned char* smem_raw, NodeVal node_val,
                                             OnOwned on_owned, const int vb, const int vgrid) {
  const VoxGeom& g = a.g;
  const int ox = OX ? OX : a.ts.ox, oy = OY ? OY : a.ts.oy, kz = a.ts.kz;
  const int ex = ox + 1, exy = ex * (oy + 1);
  const int ntx = ox + 2, nt = ntx * (oy + 2);
  T* nb = reinterpret_cast<T*>(smem_raw);  // [3 buffers][nt]
  T* FL = nb + 3 * nt;                     // [4 corners][exy]
  T* FU = FL + 4 * exy;
  // H of this thread's element, staged one element layer ahead, chunk-major [2][chunks][exy]
  constexpr int kHChunks = kStageH * (int)sizeof(T) / 16;
  unsigned char* HS = smem_raw + tile_stage_offset<T>(nt, exy, 3, 8);
  const int tid = threadIdx.x;
  const T w = T(g.w), ch = T(2.0 * (1.0 - a.kappa)), sc = T(a.scale);
  const int tiles_x = (g.rx + ox - 1) / ox, tiles_y = (g.ry + oy - 1) / oy;
  const int tiles_xy = tiles_x * tiles_y;
  const int n_tiles = tiles_xy * ((g.rz + kz - 1) / kz);
  const int ea = tid % ex, eb = tid / ex;
  const int ni = tid % ox, nj = tid / ox;
  const bool is_elem = tid < exy, is_node = tid < ox * oy;
  const bool h_async = a.H != nullptr && aligned16(a.H);
  double accd = 0.0;
  // issues the copy of element layer ke's H into buffer `buf` (one commit group
  // per call, empty when there is nothing to copy) and returns its material slot
  auto stage_elem = [&](int i0, int j0, int ke, int buf) -> int {
    int sl = 0;
    if (is_elem) {
      const int gi = wrap_elem(i0 - 1 + ea, g.nx, g.px);
      const int gj = wrap_elem(j0 - 1 + eb, g.ny, g.py);
      const int gk = wrap_elem(ke, g.nz, g.pz);
      if (gi >= 0 && gj >= 0 && gk >= 0) {
        const size_t e = (size_t)gi + (size_t)g.nx * ((size_t)gj + (size_t)g.ny * gk);
        sl = __ldg(a.slot + e);
        if (h_async) stage_chunks(HS + (size_t)buf * kHChunks * exy * 16, exy, tid, 0, a.H + kStageH * e, kHChunks);
      }
    }
    cp_async_commit();
    return sl;
  };
  auto stage1 = [&](int i0, int j0, int kn, T (&r)[2]) {
    const int gk = wrap_node(kn, g.nz, g.rz, g.pz);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = tid + h * blockDim.x;
      T v = T(0);
      if (t < nt && gk >= 0) {
        const int gi = wrap_node(i0 - 1 + t % ntx, g.nx, g.rx, g.px);
        const int gj = wrap_node(j0 - 1 + t / ntx, g.ny, g.ry, g.py);
        if (gi >= 0 && gj >= 0) v = node_val((size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * gk));
      }
      r[h] = v;
    }
  };
  auto store1 = [&](const T (&r)[2], T* buf) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = tid + h * blockDim.x;
      if (t < nt) buf[t] = r[h];
    }
  };
  for (int tile = vb; tile < n_tiles; tile += vgrid) {
    const int tz = tile / tiles_xy, txy = tile - tz * tiles_xy;
    const int i0 = (txy % tiles_x) * ox, j0 = (txy / tiles_x) * oy;
    const int k0 = tz * kz, k1 = min(k0 + kz, g.rz);
    T tdot = T(0), pend = T(0);
    T pf[2];
    stage1(i0, j0, k0 - 1, pf);
    __syncthreads();
    store1(pf, nb);
    stage1(i0, j0, k0, pf);
    int sl_next = stage_elem(i0, j0, k0 - 1, 0);
    const int K = k1 - k0;
    for (int kk = 0; kk <= K; ++kk) {
      const int ke = k0 - 1 + kk;
      T* b0 = nb + nt * (kk % 3);
      T* b1 = nb + nt * ((kk + 1) % 3);
      store1(pf, b1);
      const int sl = sl_next;
      if (kk < K) {
        stage1(i0, j0, ke + 2, pf);
        sl_next = stage_elem(i0, j0, ke + 1, (kk + 1) & 1);
        cp_async_wait<1>();  // this thread's copy of layer ke has landed
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      if (is_elem) {
        const int gi = wrap_elem(i0 - 1 + ea, g.nx, g.px);
        const int gj = wrap_elem(j0 - 1 + eb, g.ny, g.py);
        const int gk = wrap_elem(ke, g.nz, g.pz);
        T out[8];
        if (gi >= 0 && gj >= 0 && gk >= 0) {
          const size_t e = (size_t)gi + (size_t)g.nx * ((size_t)gj + (size_t)g.ny * gk);
          const T gc_ell = a.gc_ell[sl], k2 = a.gc_k2[sl];
          T dd[8], dq[8];
#pragma unroll
          for (int L = 0; L < 8; ++L) {
            const T* bb = (L & 4) ? b1 : b0;
            dd[L] = bb[(eb + ((L >> 1) & 1)) * ntx + ea + (L & 1)];
          }
          interp_sf(dd, dq);
          T hq[kStageH];
          if (h_async) {
            load_chunks<T, kStageH>(HS + (size_t)(kk & 1) * kHChunks * exy * 16, exy, tid, hq);
          } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) hq[q] = a.H ? __ldg(a.H + 8 * e + q) : T(0);
          }
          T mq[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) mq[q] = w * (gc_ell + ch * hq[q]) * dq[q];
          interp_sf_t(mq, out);
          T Dx[2][2], Dy[2][2], Dz[2][2];
          grad_k(dd, a.k, Dx, Dy, Dz);
#pragma unroll
          for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              Dx[i][j] *= k2;
              Dy[i][j] *= k2;
              Dz[i][j] *= k2;
            }
          T og[8];
          grad_k_t(Dx, Dy, Dz, a.k, og);
#pragma unroll
          for (int L = 0; L < 8; ++L) out[L] = sc * (out[L] + og[L]);
        } else {
#pragma unroll
          for (int L = 0; L < 8; ++L) out[L] = T(0);
        }
#pragma unroll
        for (int L = 0; L < 4; ++L) {
          FL[L * exy + tid] = out[L];
          FU[L * exy + tid] = out[L + 4];
        }
      }
      __syncthreads();
      if (is_node) {
        const int e11 = (ni + 1) + ex * (nj + 1), e01 = ni + ex * (nj + 1);
        const int e10 = (ni + 1) + ex * nj, e00 = ni + ex * nj;
        const T lo = FL[0 * exy + e11] + FL[1 * exy + e01] + FL[2 * exy + e10] + FL[3 * exy + e00];
        const T up = FU[0 * exy + e11] + FU[1 * exy + e01] + FU[2 * exy + e10] + FU[3 * exy + e00];
        const int gi = i0 + ni, gj = j0 + nj;
        if (kk >= 1 && gi < g.rx && gj < g.ry) {
          const size_t n = (size_t)gi + (size_t)g.rx * ((size_t)gj + (size_t)g.ry * ke);
          T v = pend + lo;
          if (a.mask && __ldg(a.mask + n)) v = T(0);
          const T xn = b0[(nj + 1) * ntx + ni + 1];
          on_owned(n, xn, v);
          if (DOT) tdot += xn * v;
        }
        pend = up;
      }
    }
    if (DOT) accd += double(tdot);
  }
  return accd;
}

// Per-slot factors of the damage element, Gc / ell and 2 w Gc ell, formed once on
// the host in the order the element arithmetic would form them (same bits).
template <typename T>
void damage_slot_coefs(DTileArgs<T>& a, const VoxMat<T>& m) {
  const T w = T(a.g.w), ell = T(a.ell);
  // PF-CZM tangent: no mass term of its own, Gc (2 ell / pi) L
  const T lt = T(2.0 * a.ell / 3.14159265358979323846);
  for (int i = 0; i < PHASTB_MAX_SLOTS; ++i) {
    const T gc = m.Gc[i];
    a.gc_ell[i] = m.dform == 1 ? T(0) : gc / ell;
    a.gc_k2[i] = m.dform == 1 ? T(2) * w * gc * lt : T(2) * w * gc * ell;
  }
}

// The damage action as its own launch (MODE == kModeDot also x . y into ws.out[kOutDot]).
template <typename T, int MODE, int OX, int OY>
__device__ __forceinline__ void dtile_body(const DTileArgs<T>& a, const int vb, const int vgrid) {
  if (a.guard && *a.guard == 0) return;
  constexpr bool DOT = MODE == kModeDot;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const T* __restrict__ x = a.x;
  T* __restrict__ y = a.y;
  const double accd = dtile_pass<T, OX, OY, DOT>(
      a, smem_raw, [&](size_t n) { return __ldg(x + n); }, [&](size_t n, T, T v) { y[n] = v; }, vb, vgrid);
  if constexpr (DOT) {
    __shared__ double sh[32];
    const double sm = block_sum(accd, sh);
    if (threadIdx.x == 0) a.ws.part[kOutDot * kMaxPartials + vb] = sm;
    if (arrive_last_n(a.ws.counter, vgrid)) {
      const double t = fold_sum(a.ws.part + kOutDot * kMaxPartials, vgrid, sh);
      if (threadIdx.x == 0) {
        a.ws.out[kOutDot] = t;
        *a.ws.counter = 0u;
      }
    }
  }
}

template <typename T, int MODE, int OX, int OY>
__global__ void __launch_bounds__(kTileMaxThreads, 2) h8_dtile_kernel(DTileArgs<T> a) {
  dtile_body<T, MODE, OX, OY>(a, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------- persistent damage PCG

// A grid-barrier wait gives up after kBarLimitNs of the GPU's global timer (a
// normal wait is a few microseconds); kBarSpins polls of ~64 ns sleep bound it
// a second time, should the timer not advance.
constexpr unsigned long long kBarLimitNs = 2000000000ull;
constexpr unsigned kBarSpins = 1u << 26;

// Grid-wide barrier of a cooperative launch (every block resident).  The last
// block to arrive resets the count and advances the generation; the others
// poll the generation.  A wait that runs out (limit_ns of global time) sets
// st->grid_error, and every block that sees the error leaves the barrier with
// false, so the kernel ends instead of hanging.  gen: this block's copy of the
// generation (thread 0).
__device__ __forceinline__ bool grid_barrier(PcgState* st, unsigned& gen,
                                             unsigned long long limit_ns = kBarLimitNs) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g0 = gen;
    __threadfence();
    if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned spins = 0;
      while (*reinterpret_cast<volatile unsigned*>(&st->bar_gen) == g0) {
        if (++spins > kBarSpins || global_ns() - t0 > limit_ns ||
            *reinterpret_cast<volatile int*>(&st->grid_error)) {
          atomicExch(&st->grid_error, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    gen = g0 + 1;
    s_ok = ok && !*reinterpret_cast<volatile int*>(&st->grid_error);
  }
  __syncthreads();
  return s_ok != 0;
}

// Self-test of the barrier's bounded wait: every block but `skip` arrives twice;
// with skip >= 0 the first wait of the others runs out after limit_ns and the
// kernel ends with st->grid_error set.
__global__ void grid_barrier_test_kernel(PcgState* st, int skip, unsigned long long limit_ns, int* passed) {
  if ((int)blockIdx.x == skip) return;
  unsigned gen = 0;
  if (!grid_barrier(st, gen, limit_ns)) return;
  if (!grid_barrier(st, gen, limit_ns)) return;
  if (threadIdx.x == 0) atomicAdd(passed, 1);
}

template <typename T>
struct DamagePcgArgs {
  int n, maxiter, mode, pad_;
  T *r, *z, *p, *p_alt, *Ap, *x;
  const T* inv_diag;
  double* part;  // 3 * kMaxPartials
  PcgState* st;
};

// Every iteration of a Jacobi-preconditioned CG on the damage operator in one
// cooperative launch, continuing from the state left by pcg_start_kernel:
//   A: p = z + beta p (formed while the bricks are staged; two direction
//      buffers, so a neighbour's halo never sees a new value), Ap, p . Ap
//   -- grid barrier --  alpha = rz / p.Ap  (every block folds the partials)
//   B: x += alpha p, r -= alpha Ap, z = r / diag, r . z, r . r
//   -- grid barrier --  beta, convergence: the state rules of
//      pcg_update_dot_kernel, evaluated identically in every block.
// Data written inside the launch is read through L2 (__ldcg).
template <typename T, int OX, int OY>
__global__ void __launch_bounds__(kTileMaxThreads, 2) h8_damage_pcg_kernel(DTileArgs<T> a, DamagePcgArgs<T> c) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sh[64];
  const int tid = threadIdx.x;
  PcgState S = *c.st;
  unsigned gen = S.bar_gen;
  const T* p_src = c.p;
  T* p_dst = c.p_alt;
  const int n = c.n;
  for (int it = 0; it < c.maxiter && S.active; ++it) {
    const T beta = T(S.beta);
    double pap = dtile_pass<T, OX, OY, true>(
        a, smem_raw, [&](size_t i) { return __ldcg(c.z + i) + beta * __ldcg(p_src + i); },
        [&](size_t i, T pn, T v) {
          c.Ap[i] = v;
          p_dst[i] = pn;
        },
        blockIdx.x, gridDim.x);
    pap = block_sum(pap, sh);
    if (tid == 0) c.part[blockIdx.x] = pap;
    if (!grid_barrier(c.st, gen)) return;
    const double PAP = fold_sum(c.part, gridDim.x, sh);
    const bool ok = isfinite(PAP) && PAP > 0.0;
    const double alpha = S.rz / PAP;
    const T al = T(alpha);
    double v2[2] = {0.0, 0.0};  // r . z, r . r
    if (ok) {
      for (int i = blockIdx.x * blockDim.x + tid; i < n; i += gridDim.x * blockDim.x) {
        c.x[i] = c.x[i] + al * __ldcg(p_dst + i);
        const T r = c.r[i] - al * __ldcg(c.Ap + i);
        c.r[i] = r;
        v2[1] += double(r) * double(r);
        const T z = c.inv_diag ? r * __ldg(c.inv_diag + i) : r;
        c.z[i] = z;
        v2[0] += double(r) * double(z);
      }
    }
    block_sum_multi<2>(v2, sh);
    if (tid == 0) {
      c.part[kMaxPartials + blockIdx.x] = v2[0];
      c.part[2 * kMaxPartials + blockIdx.x] = v2[1];
    }
    if (!grid_barrier(c.st, gen)) return;
    double f2[2];
    fold_sum_multi<2>(c.part + kMaxPartials, kMaxPartials, gridDim.x, f2, sh);
    const double RZ = f2[0], RR = f2[1];
    // the state rules of pcg_update_dot_kernel (Jacobi / identity, not PCG_PERIODIC)
    S.iter += 1;
    if (!ok) {
      if (!isfinite(PAP)) S.nonfinite = 1;
      if (!(PAP > 0.0)) S.breakdown = 1;
      S.active = 0;
    } else {
      S.alpha = alpha;
      S.steps += 1;
      if (!isfinite(RR) || !isfinite(RZ)) S.nonfinite = 1;
      S.rr = RR;
      if (!(RR > S.thr_sq)) {
        S.converged = 1;
        S.active = 0;
      } else {
        if (c.mode == PCG_STRICT && !(RZ > 0.0)) S.breakdown = 1;
        S.beta = (c.mode == PCG_STRICT) ? RZ / S.rz : ((S.rz > 0.0) ? RZ / S.rz : 0.0);
        S.rz = RZ;
      }
      if (S.breakdown || S.nonfinite) S.active = 0;
    }
    if (blockIdx.x == 0 && tid == 0) {
      PcgState& o = *c.st;
      o.rz = S.rz;
      o.rr = S.rr;
      o.alpha = S.alpha;
      o.beta = S.beta;
      o.active = S.active;
      o.breakdown = S.breakdown;
      o.nonfinite = S.nonfinite;
      o.steps = S.steps;
      o.iter = S.iter;
      o.converged = S.converged;
    }
    const T* t = p_src;
    p_src = p_dst;
    p_dst = const_cast<T*>(t);
  }
}

// ------------------------------------------------------------------ host side

namespace {

std::mutex g_shape_mu;
std::map<std::tuple<int, int, int, int, int, int, int, int>, TileShape> g_shapes;

auto shape_key(const VoxGeom& g, int word, int cls) {
  return std::make_tuple(g.rx, g.ry, g.rz, g.px, g.py, g.pz, word, cls);
}

// Heuristic: among owned-node tiles of <= kTileMaxThreads element threads,
// prefer shapes whose sides divide the grid (no ragged tiles) and the least
// recomputed halo; the z depth is left to the launch (kz = 0, launch_kz).
TileShape heuristic_shape(const VoxGeom& g, int word) {
  static const int cand[][2] = {{16, 12}, {12, 16}, {14, 14}, {24, 8}, {16, 8}, {8, 16}, {20, 8}, {32, 4},
                                {12, 12}, {10, 10}, {8, 8},   {6, 6},   {4, 4},  {2, 2},  {1, 1}};
  TileShape best{1, 1, 1};
  double best_cost = 1e300;
  for (const auto& c : cand) {
    TileShape t{std::min(c[0], g.rx), std::min(c[1], g.ry), 1};
    if (!tile_ok(t)) continue;
    const int tx = (g.rx + t.ox - 1) / t.ox, ty = (g.ry + t.oy - 1) / t.oy;
    // element-thread slots launched per node layer / useful nodes per layer
    const double cost = double(tx) * ty * tile_threads(t) / (double(g.rx) * g.ry);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = t;
    }
  }
  best.kz = 0;
  (void)word;
  return best;
}

// Z depth of a tile whose shape leaves it to the launch (kz = 0), from the
// number of blocks that can be resident at once (`capacity`): the fewest
// rounds of resident blocks, each round costing one tile's kz + 1 element
// layers plus its two-layer prologue.  A power-of-two depth leaves a second,
// mostly idle round on e.g. 64^3 (512 tiles of kz = 4 for 444 resident blocks);
// kz = 5 runs 416 tiles in one round.
int launch_kz(long long tiles_xy, int rz, long long capacity) {
  int best = 1;
  double best_cost = 1e300;
  for (int kz = 1; kz <= rz; ++kz) {
    const long long tiles = tiles_xy * ((rz + kz - 1) / kz);
    const double cost = double((tiles + capacity - 1) / capacity) * (kz + 2);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = kz;
    }
  }
  return best;
}

// TMA staging of the elastic action's node layers (PHASTB_TMA=1 turns it on).
bool tma_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PHASTB_TMA");
    return e && e[0] == '1';
  }();
  return on;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor maps of u~ (a (3 rx, ry, rz) array) and d ((rx, ry, rz)) for the TMA
// staging of a launch; false (stage through registers instead) when TMA is off,
// the row strides are not multiples of 16 bytes (rx a multiple of 16 / sizeof(T)),
// a buffer is not 16-byte aligned, or the driver refuses a map.
template <typename T>
bool tile_tensor_maps(const TileArgs<T>& a, CUtensorMap* mx, CUtensorMap* md) {
  std::memset(mx, 0, sizeof(*mx));
  std::memset(md, 0, sizeof(*md));
  if (!tma_enabled()) return false;
  const VoxGeom& v = a.g;
  const int A = 16 / (int)sizeof(T);
  if (v.rx % A != 0) return false;
  if ((reinterpret_cast<uintptr_t>(a.x) & 15u) || (a.d && (reinterpret_cast<uintptr_t>(a.d) & 15u))) return false;
  const int W = tma_wx<T>(a.ts.ox), Wd = tma_wd<T>(a.ts.ox), rows = a.ts.oy + 2;
  if (W > 256 || Wd > 256 || rows > 256) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const cuuint32_t es[3] = {1, 1, 1};
  {
    const cuuint64_t dims[3] = {3ull * (cuuint64_t)v.rx, (cuuint64_t)v.ry, (cuuint64_t)v.rz};
    const cuuint64_t strides[2] = {3ull * v.rx * sizeof(T), 3ull * v.rx * v.ry * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)W, (cuuint32_t)rows, 1};
    if (enc(mx, dt, 3, const_cast<T*>(a.x), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  if (a.d) {
    const cuuint64_t dims[3] = {(cuuint64_t)v.rx, (cuuint64_t)v.ry, (cuuint64_t)v.rz};
    const cuuint64_t strides[2] = {(cuuint64_t)v.rx * sizeof(T), (cuuint64_t)v.rx * v.ry * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)Wd, (cuuint32_t)rows, 1};
    if (enc(md, dt, 3, const_cast<T*>(a.d), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

template <typename T, int COEF, int MODE, int OX, int OY, bool TMA>
int launch_variant_t(const TileArgs<T>& a, const VoxMat<T>& m, cudaStream_t s, const CUtensorMap& mx,
                     const CUtensorMap& md) {
  auto kern = h8_tile_kernel<T, COEF, MODE, OX, OY, TMA>;
  size_t off_face = 0, off_qp = 0, off_cheb = 0;
  const size_t smem = TMA ? tile_layout_tma<T>(a.ts.ox, a.ts.oy, COEF == kCoefQP, MODE == kModeCheb, &off_face,
                                               &off_qp, &off_cheb)
                          : tile_layout<T>(a.ts.ox, a.ts.oy, COEF == kCoefQP, MODE == kModeCheb, &off_qp, &off_cheb);
  const int threads = tile_threads(a.ts);
  static std::mutex mu;
  static size_t smem_set = 0;
  static std::map<std::pair<int, size_t>, int> occ;  // (threads, smem) -> resident blocks per SM
  int per_sm = 1;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (smem > smem_set) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return PHASTB_ERR_CUDA;
      }
      smem_set = smem;
    }
    auto it = occ.find({threads, smem});
    if (it == occ.end()) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        b = 1;
      }
      it = occ.emplace(std::make_pair(threads, smem), b < 1 ? 1 : b).first;
    }
    per_sm = it->second;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const VoxGeom& v = a.g;
  const long long tiles_xy = (long long)((v.rx + a.ts.ox - 1) / a.ts.ox) * ((v.ry + a.ts.oy - 1) / a.ts.oy);
  const long long cap = std::min<long long>((long long)per_sm * sms, kMaxPartials);
  TileArgs<T> b = a;
  if (b.ts.kz <= 0) b.ts.kz = launch_kz(tiles_xy, v.rz, cap);
  const long long n_tiles = tiles_xy * ((v.rz + b.ts.kz - 1) / b.ts.kz);
  const long long grid = std::min<long long>(n_tiles, cap);
  { note_launch(); kern<<<(int)grid, threads, smem, s>>>(b, m, mx, md); }
  return last_launch_status();
}

template <typename T, int COEF, int MODE, int OX, int OY>
int launch_variant(const TileArgs<T>& a, const VoxMat<T>& m, cudaStream_t s) {
  CUtensorMap mx, md;
  const bool tma = tile_tensor_maps<T>(a, &mx, &md);
  return tma ? launch_variant_t<T, COEF, MODE, OX, OY, true>(a, m, s, mx, md)
             : launch_variant_t<T, COEF, MODE, OX, OY, false>(a, m, s, mx, md);
}

}  // namespace

bool tile_shape_lookup(const VoxGeom& g, int word, int cls, TileShape* t) {
  std::lock_guard<std::mutex> lk(g_shape_mu);
  auto it = g_shapes.find(shape_key(g, word, cls));
  if (it == g_shapes.end()) return false;
  *t = it->second;
  return true;
}

TileShape tile_shape_for(const VoxGeom& g, int word, int cls) {
  TileShape t;
  if (tile_shape_lookup(g, word, cls, &t)) return t;
  return heuristic_shape(g, word);
}

void tile_shape_record(const VoxGeom& g, int word, int cls, const TileShape& t) {
  std::lock_guard<std::mutex> lk(g_shape_mu);
  g_shapes[shape_key(g, word, cls)] = t;
}

namespace {

// Lazy tuning is opt-in (PHASTB_AUTOTUNE=1): shapes picked by timing can differ
// between processes, and the tile shape sets the grouping of the fused dot
// products, so only the deterministic heuristic keeps runs bit-reproducible.
// On the 64^3 cell the heuristic's shapes are also faster inside the solver
// than the ones timed in isolation.
bool autotune_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PHASTB_AUTOTUNE");
    return e && e[0] == '1';
  }();
  return on;
}

TileShape clamp_shape(TileShape t, const VoxGeom& v) {
  t.ox = std::min(t.ox, v.rx);
  t.oy = std::min(t.oy, v.ry);
  t.kz = std::min(t.kz, v.rz);
  return t;
}

// The packed FP32 kernel (two elements per thread in float2 lanes) is opt-in
// (PHASTB_TILE2=1): with twice the live registers per thread it keeps 9 warps
// per SM resident instead of 15, and measured 38.8 us against the scalar
// kernel's 31.8 us per 64^3 action (0.442 against 0.451 ms at 192^3), so the
// scalar kernel stays the default.
bool tile2_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PHASTB_TILE2");
    return e && e[0] == '1';
  }();
  return on;
}

template <int COEF, int MODE, int OX, int OY>
int launch_variant2(const TileArgs<float>& a, const VoxMat<float>& m, cudaStream_t s) {
  auto kern = h8_tile2_kernel<COEF, MODE, OX, OY>;
  size_t off_qp = 0, off_cheb = 0;
  const size_t smem = tile_layout<float>(a.ts.ox, a.ts.oy, COEF == kCoefQP, MODE == kModeCheb, &off_qp, &off_cheb);
  const int threads = tile2_threads(a.ts);
  static std::mutex mu;
  static size_t smem_set = 0;
  static std::map<std::pair<int, size_t>, int> occ;
  int per_sm = 1;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (smem > smem_set) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return PHASTB_ERR_CUDA;
      }
      smem_set = smem;
    }
    auto it = occ.find({threads, smem});
    if (it == occ.end()) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        b = 1;
      }
      it = occ.emplace(std::make_pair(threads, smem), b < 1 ? 1 : b).first;
    }
    per_sm = it->second;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const VoxGeom& v = a.g;
  const long long tiles_xy = (long long)((v.rx + a.ts.ox - 1) / a.ts.ox) * ((v.ry + a.ts.oy - 1) / a.ts.oy);
  const long long cap = std::min<long long>((long long)per_sm * sms, kMaxPartials);
  TileArgs<float> b = a;
  if (b.ts.kz <= 0) b.ts.kz = launch_kz(tiles_xy, v.rz, cap);
  const long long n_tiles = tiles_xy * ((v.rz + b.ts.kz - 1) / b.ts.kz);
  const long long grid = std::min<long long>(n_tiles, cap);
  { note_launch(); kern<<<(int)grid, threads, smem, s>>>(b, m); }
  return last_launch_status();
}

template <int COEF, int MODE>
int by_shape2(const TileArgs<float>& a, const VoxMat<float>& m, cudaStream_t s) {
  const int ox = a.ts.ox, oy = a.ts.oy;
  if (ox == 16 && oy == 8) return launch_variant2<COEF, MODE, 16, 8>(a, m, s);
  if (ox == 16 && oy == 12) return launch_variant2<COEF, MODE, 16, 12>(a, m, s);
  if (ox == 8 && oy == 8) return launch_variant2<COEF, MODE, 8, 8>(a, m, s);
  return launch_variant2<COEF, MODE, 0, 0>(a, m, s);
}

// Packed-kernel dispatch for FP32; PHASTB_UNSUPPORTED when it does not apply.
template <typename T>
int dispatch2(const TileArgs<T>& a, const VoxMat<T>& m, int coef, int mode, cudaStream_t s) {
  if constexpr (!std::is_same<T, float>::value) {
    return PHASTB_UNSUPPORTED;
  } else {
    if (!tile2_enabled() || !tile2_ok(a.ts)) return PHASTB_UNSUPPORTED;
    switch (coef * 8 + mode) {
      case kCoefIso * 8 + kModeApply: return by_shape2<kCoefIso, kModeApply>(a, m, s);
      case kCoefIso * 8 + kModeDot: return by_shape2<kCoefIso, kModeDot>(a, m, s);
      case kCoefIso * 8 + kModeEnergy: return launch_variant2<kCoefIso, kModeEnergy, 0, 0>(a, m, s);
      case kCoefIso * 8 + kModeCheb: return by_shape2<kCoefIso, kModeCheb>(a, m, s);
      case kCoefIso * 8 + kModeNodal: return by_shape2<kCoefIso, kModeNodal>(a, m, s);
      case kCoefQP * 8 + kModeApply: return by_shape2<kCoefQP, kModeApply>(a, m, s);
      case kCoefQP * 8 + kModeCheb: return by_shape2<kCoefQP, kModeCheb>(a, m, s);
      default: return PHASTB_UNSUPPORTED;
    }
  }
}

// The hot variants are also compiled for a few fixed tile shapes (every
// shared-memory offset then becomes a constant); other shapes run the generic
// kernel.
template <typename T, int COEF, int MODE>
int by_shape(const TileArgs<T>& a, const VoxMat<T>& m, cudaStream_t s) {
  const int ox = a.ts.ox, oy = a.ts.oy;
  if (ox == 16 && oy == 8) return launch_variant<T, COEF, MODE, 16, 8>(a, m, s);
  if (ox == 32 && oy == 4) return launch_variant<T, COEF, MODE, 32, 4>(a, m, s);
  if (ox == 8 && oy == 8) return launch_variant<T, COEF, MODE, 8, 8>(a, m, s);
  if (ox == 8 && oy == 4) return launch_variant<T, COEF, MODE, 8, 4>(a, m, s);
  if (ox == 4 && oy == 4) return launch_variant<T, COEF, MODE, 4, 4>(a, m, s);
  return launch_variant<T, COEF, MODE, 0, 0>(a, m, s);
}

template <typename T>
int dispatch(const TileArgs<T>& a, const VoxMat<T>& m, int coef, int mode, cudaStream_t s) {
  const int st2 = dispatch2<T>(a, m, coef, mode, s);
  if (st2 != PHASTB_UNSUPPORTED) return st2;
  switch (coef * 8 + mode) {
    case kCoefIso * 8 + kModeApply: return by_shape<T, kCoefIso, kModeApply>(a, m, s);
    case kCoefIso * 8 + kModeDot: return by_shape<T, kCoefIso, kModeDot>(a, m, s);
    case kCoefIso * 8 + kModeEnergy: return launch_variant<T, kCoefIso, kModeEnergy, 0, 0>(a, m, s);
    case kCoefIso * 8 + kModeCheb: return by_shape<T, kCoefIso, kModeCheb>(a, m, s);
    case kCoefIso * 8 + kModeNodal: return by_shape<T, kCoefIso, kModeNodal>(a, m, s);
    case kCoefAniso * 8 + kModeApply: return launch_variant<T, kCoefAniso, kModeApply, 0, 0>(a, m, s);
    case kCoefAniso * 8 + kModeDot: return launch_variant<T, kCoefAniso, kModeDot, 0, 0>(a, m, s);
    case kCoefAniso * 8 + kModeEnergy: return launch_variant<T, kCoefAniso, kModeEnergy, 0, 0>(a, m, s);
    case kCoefAniso * 8 + kModeCheb: return launch_variant<T, kCoefAniso, kModeCheb, 0, 0>(a, m, s);
    case kCoefAniso * 8 + kModeNodal: return launch_variant<T, kCoefAniso, kModeNodal, 0, 0>(a, m, s);
    case kCoefQP * 8 + kModeApply: return by_shape<T, kCoefQP, kModeApply>(a, m, s);
    case kCoefQP * 8 + kModeCheb: return by_shape<T, kCoefQP, kModeCheb>(a, m, s);
    default: return PHASTB_ERR_ARG;
  }
}

// Times the (coef, mode) launch of `a` over the candidate shapes (a's outputs
// are overwritten; modes that update their inputs in place are not timed).
template <typename T>
int tune_shape(TileArgs<T> a, const VoxMat<T>& m, int coef, int mode, cudaStream_t s, TileShape* best_out,
               float* best_ms) {
  static const int cand[][2] = {{16, 8}, {32, 4},  {8, 8},   {8, 4},   {4, 4},   {16, 12}, {12, 16},
                                {14, 14}, {24, 8}, {20, 8}, {12, 12}, {10, 10}, {6, 6},   {2, 4}};
  static const int kzs[] = {0, 1, 2, 4, 8, 16};  // 0: chosen at launch
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return PHASTB_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return PHASTB_ERR_CUDA;
  }
  int st = PHASTB_OK;
  float best = 1e30f;
  TileShape bs = clamp_shape(heuristic_shape(a.g, (int)sizeof(T)), a.g);
  std::vector<TileShape> seen;
  for (const auto& c : cand) {
    for (int kz : kzs) {
      const TileShape t = clamp_shape(TileShape{c[0], c[1], kz}, a.g);
      if (!tile_ok(t)) continue;
      bool dup = false;
      for (const auto& q : seen) dup |= (q.ox == t.ox && q.oy == t.oy && q.kz == t.kz);
      if (dup) continue;
      seen.push_back(t);
      a.ts = t;
      if ((st = dispatch<T>(a, m, coef, mode, s))) break;
      const int reps = 3;
      cudaEventRecord(e0, s);
      for (int r = 0; r < reps && !st; ++r) st = dispatch<T>(a, m, coef, mode, s);
      cudaEventRecord(e1, s);
      if (st || (st = cuda_status(cudaEventSynchronize(e1)))) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= reps;
      if (ms < best) {
        best = ms;
        bs = t;
      }
    }
    if (st) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  *best_out = bs;
  if (best_ms) *best_ms = best;
  return PHASTB_OK;
}

}  // namespace

template <typename T>
TileArgs<T> tile_args(const VoxGeom& v, int cls) {
  TileArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  a.g = v;
  a.ts = clamp_shape(tile_shape_for(v, (int)sizeof(T), cls), v);
  a.k.c1 = T(kC1);
  a.k.c2 = T(kC2);
  a.k.x1 = T(kC1 / v.hx);
  a.k.x2 = T(kC2 / v.hx);
  a.k.y1 = T(kC1 / v.hy);
  a.k.y2 = T(kC2 / v.hy);
  a.k.z1 = T(kC1 / v.hz);
  a.k.z2 = T(kC2 / v.hz);
  return a;
}

template <typename T>
int h8_tile_launch(const TileArgs<T>& a, const VoxMat<T>& m, int coef, int mode, cudaStream_t s, bool tune) {
  if (!tile_ok(a.ts) || a.ts.ox > a.g.rx || a.ts.oy > a.g.ry || a.ts.kz > a.g.rz) return PHASTB_ERR_ARG;
  const int cls = coef == kCoefQP ? 1 : 0;
  TileShape known;
  if (tune && autotune_enabled() && (mode == kModeApply || mode == kModeDot) && a.guard == nullptr &&
      !tile_shape_lookup(a.g, (int)sizeof(T), cls, &known)) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
      TileShape best;
      int st = tune_shape<T>(a, m, coef, mode, s, &best, nullptr);
      if (st) return st;
      tile_shape_record(a.g, (int)sizeof(T), cls, best);
      TileArgs<T> b = a;
      b.ts = best;
      return dispatch<T>(b, m, coef, mode, s);
    }
    cudaGetLastError();
  }
  return dispatch<T>(a, m, coef, mode, s);
}

template <typename T>
int h8_mech_tile_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* x, const T* gq,
                        const T* d, const uint8_t* mask, T* y, RedWs ws, const int* guard, bool dot, bool energy,
                        cudaStream_t s, const TileShape* force_shape) {
  TileArgs<T> a = tile_args<T>(v, 0);
  if (force_shape) a.ts = clamp_shape(*force_shape, v);
  a.slot = slot;
  a.gq = gq;
  a.d = d;
  a.x = x;
  a.y = y;
  a.mask = mask;
  a.ws = ws;
  a.guard = guard;
  const int coef = m.iso ? kCoefIso : kCoefAniso;
  return h8_tile_launch<T>(a, m, coef, dot ? kModeDot : (energy ? kModeEnergy : kModeApply), s, !force_shape);
}

template <typename T, int MODE, int OX, int OY>
int dlaunch_variant(const DTileArgs<T>& a, cudaStream_t s) {
  auto kern = h8_dtile_kernel<T, MODE, OX, OY>;
  const int nt = (a.ts.ox + 2) * (a.ts.oy + 2), exy = (a.ts.ox + 1) * (a.ts.oy + 1);
  const size_t smem = tile_stage_offset<T>(nt, exy, 3, 8) + sizeof(T) * 2 * kStageH * (size_t)exy;
  const int threads = tile_threads(a.ts);
  static std::mutex mu;
  static size_t smem_set = 0;
  static std::map<std::pair<int, size_t>, int> occ;
  int per_sm = 1;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (smem > smem_set) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return PHASTB_ERR_CUDA;
      }
      smem_set = smem;
    }
    auto it = occ.find({threads, smem});
    if (it == occ.end()) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        b = 1;
      }
      it = occ.emplace(std::make_pair(threads, smem), b < 1 ? 1 : b).first;
    }
    per_sm = it->second;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const VoxGeom& v = a.g;
  const long long tiles_xy = (long long)((v.rx + a.ts.ox - 1) / a.ts.ox) * ((v.ry + a.ts.oy - 1) / a.ts.oy);
  const long long cap = std::min<long long>((long long)per_sm * sms, kMaxPartials);
  DTileArgs<T> b = a;
  if (b.ts.kz <= 0) b.ts.kz = launch_kz(tiles_xy, v.rz, cap);
  const long long n_tiles = tiles_xy * ((v.rz + b.ts.kz - 1) / b.ts.kz);
  const long long grid = std::min<long long>(n_tiles, cap);
  { note_launch(); kern<<<(int)grid, threads, smem, s>>>(b); }
  return last_launch_status();
}

template <typename T, int MODE>
int dby_shape(const DTileArgs<T>& a, cudaStream_t s) {
  const int ox = a.ts.ox, oy = a.ts.oy;
  if (ox == 16 && oy == 8) return dlaunch_variant<T, MODE, 16, 8>(a, s);
  if (ox == 32 && oy == 4) return dlaunch_variant<T, MODE, 32, 4>(a, s);
  if (ox == 8 && oy == 8) return dlaunch_variant<T, MODE, 8, 8>(a, s);
  return dlaunch_variant<T, MODE, 0, 0>(a, s);
}

template <typename T, int OX, int OY>
int dpcg_variant(const DTileArgs<T>& a0, const DamagePcgArgs<T>& c0, cudaStream_t s) {
  auto kern = h8_damage_pcg_kernel<T, OX, OY>;
  const int nt = (a0.ts.ox + 2) * (a0.ts.oy + 2), exy = (a0.ts.ox + 1) * (a0.ts.oy + 1);
  const size_t smem = tile_stage_offset<T>(nt, exy, 3, 8) + sizeof(T) * 2 * kStageH * (size_t)exy;
  const int threads = tile_threads(a0.ts);
  static std::mutex mu;
  static size_t smem_set = 0;
  static std::map<std::pair<int, size_t>, int> occ;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (smem > smem_set) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return PHASTB_UNSUPPORTED;
      }
      smem_set = smem;
    }
    auto it = occ.find({threads, smem});
    if (it == occ.end()) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        b = 0;
      }
      it = occ.emplace(std::make_pair(threads, smem), b).first;
    }
    per_sm = it->second;
  }
  int dev = 0, sms = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess) {
    cudaGetLastError();
    return PHASTB_UNSUPPORTED;
  }
  if (!coop || per_sm < 1 || sms < 1) return PHASTB_UNSUPPORTED;
  const VoxGeom& v = a0.g;
  const long long tiles_xy = (long long)((v.rx + a0.ts.ox - 1) / a0.ts.ox) * ((v.ry + a0.ts.oy - 1) / a0.ts.oy);
  // every block must be resident at once (the grid barriers wait for all of them)
  const long long cap = std::min<long long>((long long)per_sm * sms, kMaxPartials);
  DTileArgs<T> a = a0;
  if (a.ts.kz <= 0) a.ts.kz = launch_kz(tiles_xy, v.rz, cap);
  const long long n_tiles = tiles_xy * ((v.rz + a.ts.kz - 1) / a.ts.kz);
  const int grid = (int)std::min<long long>(n_tiles, cap);
  DamagePcgArgs<T> c = c0;
  void* args[] = {&a, &c};
  if (cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(threads), args, smem, s) != cudaSuccess) {
    cudaGetLastError();
    return PHASTB_UNSUPPORTED;
  }
  note_launch();
  return PHASTB_OK;
}

// PHASTB_PERSISTENT_PCG=0 runs the damage CG as separate launches per iteration.
bool persistent_pcg_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PHASTB_PERSISTENT_PCG");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename T>
int h8_damage_tile_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* x, const T* H,
                          double scale, const uint8_t* mask, T* y, RedWs ws, const int* guard, bool dot,
                          cudaStream_t s) {
  DTileArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  const TileArgs<T> base = tile_args<T>(v, 2);
  a.g = v;
  a.ts = base.ts;
  a.k = base.k;
  a.slot = slot;
  a.kappa = double(m.kappa);
  a.ell = double(m.ell);
  damage_slot_coefs(a, m);
  a.scale = scale;
  a.H = H;
  a.x = x;
  a.y = y;
  a.mask = mask;
  a.ws = ws;
  a.guard = guard;
  if (!tile_ok(a.ts)) return PHASTB_ERR_ARG;
  auto run = [&](const DTileArgs<T>& b) { return dot ? dby_shape<T, kModeDot>(b, s) : dby_shape<T, kModeApply>(b, s); };
  TileShape known;
  if (autotune_enabled() && guard == nullptr && !tile_shape_lookup(v, (int)sizeof(T), 2, &known)) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
      // time the candidate shapes on this call's buffers (y is recomputed below)
      static const int cand[][2] = {{16, 8}, {32, 4}, {8, 8}, {16, 12}, {14, 14}, {10, 10}, {8, 4}, {4, 4}};
      static const int kzs[] = {0, 2, 4, 8, 16};  // 0: chosen at launch
      cudaEvent_t e0, e1;
      if (cudaEventCreate(&e0) != cudaSuccess) return PHASTB_ERR_CUDA;
      if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return PHASTB_ERR_CUDA;
      }
      int st = PHASTB_OK;
      float best = 1e30f;
      TileShape bs = a.ts;
      DTileArgs<T> b = a;
      for (const auto& c : cand) {
        for (int kz : kzs) {
          b.ts = clamp_shape(TileShape{c[0], c[1], kz}, v);
          if (!tile_ok(b.ts)) continue;
          if ((st = run(b))) break;
          cudaEventRecord(e0, s);
          for (int r = 0; r < 3 && !st; ++r) st = run(b);
          cudaEventRecord(e1, s);
          if (st || (st = cuda_status(cudaEventSynchronize(e1)))) break;
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          if (ms < best) {
            best = ms;
            bs = b.ts;
          }
        }
        if (st) break;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (st) return st;
      tile_shape_record(v, (int)sizeof(T), 2, bs);
      a.ts = bs;
    } else {
      cudaGetLastError();
    }
  }
  return run(a);
}

template int h8_damage_tile_launch<double>(const VoxGeom&, const VoxMat<double>&, const uint8_t*, const double*,
                                           const double*, double, const uint8_t*, double*, RedWs, const int*, bool,
                                           cudaStream_t);
template int h8_damage_tile_launch<float>(const VoxGeom&, const VoxMat<float>&, const uint8_t*, const float*,
                                          const float*, double, const uint8_t*, float*, RedWs, const int*, bool,
                                          cudaStream_t);

template <typename T>
int h8_damage_pcg_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* H, double scale,
                         const uint8_t* mask, const PcgWs<T>& w, T* p_alt, T* x, const T* inv_diag, int maxiter,
                         int mode, cudaStream_t s) {
  if (mode == PCG_PERIODIC || !persistent_pcg_enabled()) return PHASTB_UNSUPPORTED;
  DTileArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  const TileArgs<T> base = tile_args<T>(v, 2);
  a.g = v;
  a.ts = base.ts;
  a.k = base.k;
  a.slot = slot;
  a.kappa = double(m.kappa);
  a.ell = double(m.ell);
  damage_slot_coefs(a, m);
  a.scale = scale;
  a.H = H;
  a.mask = mask;
  if (!tile_ok(a.ts)) return PHASTB_ERR_ARG;
  DamagePcgArgs<T> c;
  std::memset(&c, 0, sizeof(c));
  c.n = v.n_red;
  c.maxiter = maxiter;
  c.mode = mode;
  c.r = w.r;
  c.z = w.z;
  c.p = w.p;
  c.p_alt = p_alt;
  c.Ap = w.Ap;
  c.x = x;
  c.inv_diag = inv_diag;
  c.part = w.part;
  c.st = w.st;
  const int ox = a.ts.ox, oy = a.ts.oy;
  if (ox == 16 && oy == 8) return dpcg_variant<T, 16, 8>(a, c, s);
  if (ox == 32 && oy == 4) return dpcg_variant<T, 32, 4>(a, c, s);
  if (ox == 8 && oy == 8) return dpcg_variant<T, 8, 8>(a, c, s);
  return dpcg_variant<T, 0, 0>(a, c, s);
}

template int h8_damage_pcg_launch<double>(const VoxGeom&, const VoxMat<double>&, const uint8_t*, const double*,
                                          double, const uint8_t*, const PcgWs<double>&, double*, double*,
                                          const double*, int, int, cudaStream_t);
template int h8_damage_pcg_launch<float>(const VoxGeom&, const VoxMat<float>&, const uint8_t*, const float*,
                                         double, const uint8_t*, const PcgWs<float>&, float*, float*, const float*,
                                         int, int, cudaStream_t);
// ------------------------------------------------------------ packed cell batches

template <typename T>
__device__ __forceinline__ TileK<T> batch_k(const BatchCell& c) {
  if constexpr (sizeof(T) == 4)
    return c.kf;
  else
    return c.kd;
}

// One brick of one cell per block: the block builds its cell's arguments in shared
// memory and runs the single-grid tile body with its brick index inside the cell.
template <typename T, int MODE, int OX, int OY, int COEF = kCoefIso>
__global__ void __launch_bounds__(kTileMaxThreads, sizeof(T) == 4 ? 2 : 1)
    h8_tile_batch_kernel(TileBatchArgs<T> b, VoxMat<T> m) {
  __shared__ TileArgs<T> sa;
  const int2 wk = b.work[blockIdx.x];
  const BatchCell& c = b.cells[wk.x];
  if (threadIdx.x == 0) {
    TileArgs<T> a;
    a.g = c.g;
    a.ts = c.ts;
    a.pad_ = 0;
    a.slot = b.slot ? b.slot + c.elem_off : nullptr;
    a.gq = nullptr;
    a.d = b.d ? b.d + c.node_off : nullptr;
    a.lam_q = b.lam_q ? b.lam_q + 8 * c.elem_off : nullptr;
    a.mu_q = b.mu_q ? b.mu_q + 8 * c.elem_off : nullptr;
    a.x = b.x + c.mech_off;
    a.y = b.y ? b.y + c.mech_off : nullptr;
    a.mask = b.mask ? b.mask + c.mech_off : nullptr;
    a.res = b.res ? b.res + c.mech_off : nullptr;
    a.invd = b.invd ? b.invd + c.mech_off : nullptr;
    a.xs = b.xs ? b.xs + c.mech_off : nullptr;
    a.d_out = b.d_out ? b.d_out + c.mech_off : nullptr;
    a.c1 = b.c1;
    a.c2 = b.c2 * (b.c2_scale ? b.c2_scale[wk.x] : 1.0);
    a.ws = red_ws(b.ws + (size_t)wk.x * red_ws_bytes());
    a.guard = b.guard ? b.guard + (size_t)wk.x * b.guard_stride : nullptr;
    a.k = batch_k<T>(c);
    sa = a;
  }
  __syncthreads();
  tile_body<T, COEF, MODE, OX, OY, false>(sa, m, nullptr, nullptr, wk.y, c.nvb);
}

template <typename T, int MODE, int OX, int OY>
__global__ void __launch_bounds__(kTileMaxThreads, 2) h8_dtile_batch_kernel(TileBatchArgs<T> b, VoxMat<T> m) {
  __shared__ DTileArgs<T> sa;
  const int2 wk = b.work[blockIdx.x];
  const BatchCell& c = b.cells[wk.x];
  if (threadIdx.x == 0) {
    DTileArgs<T> a;
    a.g = c.g;
    a.ts = c.ts;
    a.pad_ = 0;
    a.slot = b.slot + c.elem_off;
    // per-slot factors in the order of damage_slot_coefs (same bits as a single-cell launch)
    const T w = T(c.g.w), ell = T(c.ell);
    for (int i = 0; i < PHASTB_MAX_SLOTS; ++i) {
      const T gc = m.Gc[i];
      a.gc_ell[i] = gc / ell;
      a.gc_k2[i] = T(2) * w * gc * ell;
    }
    a.kappa = b.kappa;
    a.ell = c.ell;
    a.scale = b.dscale ? c.dscale : 1.0;
    a.H = b.H ? b.H + 8 * c.elem_off : nullptr;
    a.x = b.x + c.node_off;
    a.y = b.y + c.node_off;
    a.mask = b.mask ? b.mask + c.node_off : nullptr;
    a.ws = red_ws(b.ws + (size_t)wk.x * red_ws_bytes());
    a.guard = b.guard ? b.guard + (size_t)wk.x * b.guard_stride : nullptr;
    a.k = batch_k<T>(c);
    sa = a;
  }
  __syncthreads();
  dtile_body<T, MODE, OX, OY>(sa, wk.y, c.nvb);
}

namespace {

template <class K>
int batch_smem_attr(K kern, size_t smem) {
  static std::mutex mu;
  static std::map<const void*, size_t> set;
  std::lock_guard<std::mutex> lk(mu);
  auto it = set.find((const void*)kern);
  if (it != set.end() && it->second >= smem) return PHASTB_OK;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return PHASTB_ERR_CUDA;
  }
  set[(const void*)kern] = smem;
  return PHASTB_OK;
}

template <typename T, int MODE, int OX, int OY>
int tile_batch_variant(const TileBatchArgs<T>& b, const VoxMat<T>& m, cudaStream_t s) {
  auto kern = h8_tile_batch_kernel<T, MODE, OX, OY>;
  size_t oq = 0, oc = 0;
  const size_t smem = tile_layout<T>(OX, OY, false, false, &oq, &oc);
  int st = batch_smem_attr(kern, smem);
  if (st) return st;
  const int threads = ((OX + 1) * (OY + 1) + 31) / 32 * 32;
  { note_launch(); kern<<<b.n_blocks, threads, smem, s>>>(b, m); }
  return last_launch_status();
}

template <int COEF, int MODE, int OX, int OY>
int tile_batch_level_variant(const TileBatchArgs<float>& b, const VoxMat<float>& m, cudaStream_t s) {
  auto kern = h8_tile_batch_kernel<float, MODE, OX, OY, COEF>;
  size_t oq = 0, oc = 0;
  const size_t smem = tile_layout<float>(OX, OY, COEF == kCoefQP, MODE == kModeCheb, &oq, &oc);
  int st = batch_smem_attr(kern, smem);
  if (st) return st;
  const int threads = ((OX + 1) * (OY + 1) + 31) / 32 * 32;
  { note_launch(); kern<<<b.n_blocks, threads, smem, s>>>(b, m); }
  return last_launch_status();
}

template <typename T, int MODE, int OX, int OY>
int dtile_batch_variant(const TileBatchArgs<T>& b, const VoxMat<T>& m, cudaStream_t s) {
  auto kern = h8_dtile_batch_kernel<T, MODE, OX, OY>;
  const int nt = (OX + 2) * (OY + 2), exy = (OX + 1) * (OY + 1);
  const size_t smem = tile_stage_offset<T>(nt, exy, 3, 8) + sizeof(T) * 2 * kStageH * (size_t)exy;
  int st = batch_smem_attr(kern, smem);
  if (st) return st;
  const int threads = ((OX + 1) * (OY + 1) + 31) / 32 * 32;
  { note_launch(); kern<<<b.n_blocks, threads, smem, s>>>(b, m); }
  return last_launch_status();
}

}  // namespace

template <typename T>
int h8_tile_batch_launch(const TileBatchArgs<T>& b, const VoxMat<T>& m, int mode, int ox, int oy, cudaStream_t s) {
  if (!m.iso) return PHASTB_UNSUPPORTED;
  if (b.n_blocks < 1) return PHASTB_OK;
  const bool dot = mode == kModeDot;
  if (mode != kModeApply && !dot) return PHASTB_ERR_ARG;
  if (ox == 16 && oy == 8)
    return dot ? tile_batch_variant<T, kModeDot, 16, 8>(b, m, s) : tile_batch_variant<T, kModeApply, 16, 8>(b, m, s);
  if (ox == 8 && oy == 8)
    return dot ? tile_batch_variant<T, kModeDot, 8, 8>(b, m, s) : tile_batch_variant<T, kModeApply, 8, 8>(b, m, s);
  return PHASTB_ERR_ARG;
}

int h8_tile_batch_level_launch(const TileBatchArgs<float>& b, const VoxMat<float>& m, int coef, int mode, int ox,
                               int oy, cudaStream_t s) {
  if (b.n_blocks < 1) return PHASTB_OK;
  if (coef == kCoefIso && !m.iso) return PHASTB_UNSUPPORTED;
  if (coef == kCoefIso && ox == 16 && oy == 8) {
    if (mode == kModeCheb) return tile_batch_level_variant<kCoefIso, kModeCheb, 16, 8>(b, m, s);
    if (mode == kModeNodal) return tile_batch_level_variant<kCoefIso, kModeNodal, 16, 8>(b, m, s);
  }
  if (coef == kCoefIso && ox == 8 && oy == 8) {
    if (mode == kModeCheb) return tile_batch_level_variant<kCoefIso, kModeCheb, 8, 8>(b, m, s);
    if (mode == kModeNodal) return tile_batch_level_variant<kCoefIso, kModeNodal, 8, 8>(b, m, s);
  }
  if (coef == kCoefQP && ox == 8 && oy == 8) {
    if (mode == kModeCheb) return tile_batch_level_variant<kCoefQP, kModeCheb, 8, 8>(b, m, s);
    if (mode == kModeApply) return tile_batch_level_variant<kCoefQP, kModeApply, 8, 8>(b, m, s);
  }
  return PHASTB_ERR_ARG;
}

template <typename T>
int h8_dtile_batch_launch(const TileBatchArgs<T>& b, const VoxMat<T>& m, bool dot, int ox, int oy, cudaStream_t s) {
  if (b.n_blocks < 1) return PHASTB_OK;
  if (ox == 16 && oy == 8)
    return dot ? dtile_batch_variant<T, kModeDot, 16, 8>(b, m, s) : dtile_batch_variant<T, kModeApply, 16, 8>(b, m, s);
  if (ox == 8 && oy == 8)
    return dot ? dtile_batch_variant<T, kModeDot, 8, 8>(b, m, s) : dtile_batch_variant<T, kModeApply, 8, 8>(b, m, s);
  return PHASTB_ERR_ARG;
}

template int h8_tile_batch_launch<double>(const TileBatchArgs<double>&, const VoxMat<double>&, int, int, int,
                                          cudaStream_t);
template int h8_tile_batch_launch<float>(const TileBatchArgs<float>&, const VoxMat<float>&, int, int, int,
                                         cudaStream_t);
template int h8_dtile_batch_launch<double>(const TileBatchArgs<double>&, const VoxMat<double>&, bool, int, int,
                                           cudaStream_t);

template TileArgs<double> tile_args<double>(const VoxGeom&, int);
template TileArgs<float> tile_args<float>(const VoxGeom&, int);
template int h8_tile_launch<double>(const TileArgs<double>&, const VoxMat<double>&, int, int, cudaStream_t, bool);
template int h8_tile_launch<float>(const TileArgs<float>&, const VoxMat<float>&, int, int, cudaStream_t, bool);
template int h8_mech_tile_launch<double>(const VoxGeom&, const VoxMat<double>&, const uint8_t*, const double*,
                                         const double*, const double*, const uint8_t*, double*, RedWs, const int*,
                                         bool, bool, cudaStream_t, const TileShape*);
template int h8_mech_tile_launch<float>(const VoxGeom&, const VoxMat<float>&, const uint8_t*, const float*,
                                        const float*, const float*, const uint8_t*, float*, RedWs, const int*, bool,
                                        bool, cudaStream_t, const TileShape*);

}  // namespace phastb

// ------------------------------------------------------------------ autotuner

namespace phastb {
bool valid_vox(const phastb_voxel_grid* g);
bool valid_mat(const phastb_voxel_material* m);

namespace {

template <typename T>
int tune_t(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* x, const T* d, T* y, RedWs ws,
           cudaStream_t s, TileShape* best_out, float* best_ms) {
  TileArgs<T> a = tile_args<T>(v, 0);
  a.slot = slot;
  a.d = d;
  a.x = x;
  a.y = y;
  a.ws = ws;
  int st = tune_shape<T>(a, m, m.iso ? kCoefIso : kCoefAniso, kModeApply, s, best_out, best_ms);
  if (st) return st;
  tile_shape_record(v, (int)sizeof(T), 0, *best_out);
  return PHASTB_OK;
}

}  // namespace
}  // namespace phastb

using namespace phastb;

extern "C" {

int phastb_h8_tile_shape(const phastb_voxel_grid* g, int dtype, int set, int* shape) {
  if (!valid_vox(g) || !shape || (dtype != PHASTB_F32 && dtype != PHASTB_F64)) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  const int word = dtype == PHASTB_F32 ? 4 : 8;
  if (set) {
    TileShape t{shape[0], shape[1], shape[2]};
    if (!tile_ok(t)) return PHASTB_ERR_ARG;
    tile_shape_record(v, word, 0, t);
    return PHASTB_OK;
  }
  const TileShape t = tile_shape_for(v, word, 0);
  shape[0] = std::min(t.ox, v.rx);
  shape[1] = std::min(t.oy, v.ry);
  shape[2] = std::min(t.kz, v.rz);
  return PHASTB_OK;
}

int phastb_h8_autotune(const phastb_voxel_grid* g, const phastb_voxel_material* m, int dtype, const uint8_t* slot,
                       const void* x, const void* d, void* y, void* scratch, size_t scratch_bytes, int* shape,
                       float* ms, void* stream) {
  if (!valid_vox(g) || !valid_mat(m) || !slot || !x || !y || !shape || !ms) return PHASTB_ERR_ARG;
  if (dtype != PHASTB_F32 && dtype != PHASTB_F64) return PHASTB_ERR_ARG;
  if (!scratch || scratch_bytes < red_ws_bytes()) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return PHASTB_ERR_ARG;
  const VoxGeom v = make_vox_geom(*g);
  RedWs ws = red_ws(scratch);
  int st;
  if ((st = red_ws_reset(ws, s))) return st;
  TileShape t{};
  if (dtype == PHASTB_F64)
    st = tune_t<double>(v, make_vox_mat<double>(*m), slot, (const double*)x, (const double*)d, (double*)y, ws, s,
                        &t, ms);
  else
    st = tune_t<float>(v, make_vox_mat<float>(*m), slot, (const float*)x, (const float*)d, (float*)y, ws, s, &t, ms);
  if (st) return st;
  shape[0] = t.ox;
  shape[1] = t.oy;
  shape[2] = t.kz;
  return PHASTB_OK;
}

}  // extern "C"

extern "C" int phastb_test_grid_barrier(int blocks, int skip_block, double limit_s, int* grid_error_host,
                                        int* passed_host) {
  using namespace phastb;
  if (blocks < 1 || blocks > 64 || skip_block >= blocks || !(limit_s > 0) || limit_s > 10.0 || !grid_error_host ||
      !passed_host)
    return PHASTB_ERR_ARG;
  int dev = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
    return PHASTB_UNSUPPORTED;
  PcgState* st = nullptr;
  int* passed = nullptr;
  if (cudaMalloc(&st, sizeof(PcgState)) != cudaSuccess) return PHASTB_ERR_CUDA;
  if (cudaMalloc(&passed, sizeof(int)) != cudaSuccess) {
    cudaFree(st);
    return PHASTB_ERR_CUDA;
  }
  int status = cuda_status(cudaMemset(st, 0, sizeof(PcgState)));
  if (!status) status = cuda_status(cudaMemset(passed, 0, sizeof(int)));
  unsigned long long limit_ns = (unsigned long long)(limit_s * 1e9);
  void* args[] = {&st, &skip_block, &limit_ns, &passed};
  if (!status) {
    note_launch();
    status = cuda_status(cudaLaunchCooperativeKernel((const void*)grid_barrier_test_kernel, dim3(blocks), dim3(32),
                                                     args, 0, nullptr));
  }
  if (!status) status = cuda_status(cudaDeviceSynchronize());
  PcgState hs{};
  if (!status) status = cuda_status(cudaMemcpy(&hs, st, sizeof(PcgState), cudaMemcpyDeviceToHost));
  if (!status) status = cuda_status(cudaMemcpy(passed_host, passed, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(st);
  cudaFree(passed);
  if (status) return status;
  *grid_error_host = hs.grid_error;
  return hs.grid_error ? PHASTB_ERR_CUDA : PHASTB_OK;
}

extern "C" int phastb_h8_tma_staging(const phastb_voxel_grid* g, int dtype) {
  using namespace phastb;
  if (!valid_vox(g) || (dtype != PHASTB_F64 && dtype != PHASTB_F32)) return -1;
  const VoxGeom v = make_vox_geom(*g);
  const int A = dtype == PHASTB_F32 ? 4 : 2;
  return (tma_enabled() && v.rx % A == 0 && tensor_map_encoder() != nullptr) ? 1 : 0;
}
