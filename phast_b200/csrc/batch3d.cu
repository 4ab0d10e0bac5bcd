// Packed batches of periodic voxel cells: many cells of different sizes advanced
// together, every Krylov iteration one launch per operator apply and per vector
// step over all cells, with each cell's solver state (alpha, beta, residual
// norms, flags) in device memory.
//
// Packed layout: cell c's reduced nodes start at node_off[c], its mechanics
// unknowns [u~ (3 n_red), E (6)] at mech_off[c] and its elements at elem_off[c]
// (material slots one per element, histories eight per element).  A vector
// family (nodes or mechanics unknowns) is cut into chunks that never cross a
// cell boundary; a reducing kernel writes one partial per chunk into the cell's
// own reduction workspace and the cell's last chunk folds them in a fixed order
// (the same deterministic last-block fold as a single-grid launch).
//
// The solvers follow the single-cell ones in solvers3d.cu and gmg.cu, per cell:
//   constrained Jacobi PCG mechanics (solid3d/linalg.py:99-287), optionally as
//   FP32 inner solves under FP64 iterative refinement (mixed_precision_cg.py);
//   primal active-set box-KKT damage with a Dirichlet PCG per set
//   (solvers/box_kkt_h8.py:256-778).
#include "engine.cuh"
#include "h8_kernels.cuh"
#include "h8_tile.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

namespace phastb {

bool valid_vox(const phastb_voxel_grid* g);
bool valid_mat(const phastb_voxel_material* m);
size_t h8_scratch_bytes(const VoxGeom& v, int dtype);
template <typename T>
int h8_mech_diag_t(const VoxGeom& v, const VoxMat<T>& mm, const uint8_t* slot, const T* gq, const T* d, T* diag,
                   void* scratch, cudaStream_t s);
int h8_damage_launch(const VoxGeom& v, const VoxMat<double>& mm, const uint8_t* slot, int mode, const double* d,
                     const double* H, double scale, double* y, const uint8_t* mask, void* scratch,
                     const int* guard, cudaStream_t s);

// A packed vector family cut into per-cell chunks: block b covers [begin, end)
// of cell `cell` (global packed indices) and is partial j of that cell.
struct BChunk {
  int cell, begin, end, j;
};

struct BVec {
  const BChunk* chunks;
  const int* nchunk;  // chunks per cell
  int n_chunks;
  int pad_;
};

}  // namespace phastb

// Host plan of a batch (opaque to C callers).
struct phastb_batch {
  int n_cells = 0, ox = 16, oy = 8, kz = 8;
  std::vector<phastb::VoxGeom> geom;
  std::vector<phastb::BatchCell> cells;
  std::vector<int2> work;
  std::vector<phastb::BChunk> node_chunks, mech_chunks;
  std::vector<int> node_nchunk, mech_nchunk;
  long long n_nodes = 0, n_mech = 0, n_elem = 0;
  long long max_elem = 0;
  // device copies of the tables (inside the caller's plan buffer)
  phastb::BatchCell* d_cells = nullptr;
  int2* d_work = nullptr;
  phastb::BChunk* d_node_chunks = nullptr;
  phastb::BChunk* d_mech_chunks = nullptr;
  int* d_node_nchunk = nullptr;
  int* d_mech_nchunk = nullptr;
  bool bound = false;
  size_t table_bytes = 0;     // this level's tables
  // coarse multigrid levels (cells of edge n/2 and n/4 with 8 x 8 x 4 bricks), when every cell
  // is periodic with edges divisible by 4 and at least 32
  phastb_batch* lev[2] = {nullptr, nullptr};
  int nlev = 1;
  ~phastb_batch() {
    delete lev[0];
    delete lev[1];
  }
  size_t all_table_bytes() const {
    size_t t = table_bytes;
    for (int l = 0; l < nlev - 1; ++l) t += lev[l]->table_bytes;
    return t;
  }
};

namespace phastb {

namespace {

constexpr int kBatchMaxChunks = 1024;  // partials per cell and vector family (<= kMaxPartials)

void make_chunks(const std::vector<long long>& off, const std::vector<long long>& len, std::vector<BChunk>* out,
                 std::vector<int>* counts) {
  out->clear();
  counts->clear();
  for (size_t c = 0; c < off.size(); ++c) {
    const long long n = len[c];
    const long long per = (n + (long long)kThreads * kBatchMaxChunks - 1) / ((long long)kThreads * kBatchMaxChunks);
    const long long ch = (long long)kThreads * std::max<long long>(8, per);
    int j = 0;
    for (long long b = 0; b < n; b += ch, ++j)
      out->push_back(BChunk{(int)c, (int)(off[c] + b), (int)(off[c] + std::min(n, b + ch)), j});
    counts->push_back(j);
  }
}

inline BVec node_vec(const phastb_batch* B) {
  return BVec{B->d_node_chunks, B->d_node_nchunk, (int)B->node_chunks.size(), 0};
}
inline BVec mech_vec(const phastb_batch* B) {
  return BVec{B->d_mech_chunks, B->d_mech_nchunk, (int)B->mech_chunks.size(), 0};
}

__host__ __device__ inline char* cell_ws(char* base, int c) { return base + (size_t)c * red_ws_bytes(); }
__host__ __device__ inline const double* cell_out(const char* base, int c) {
  return red_ws(const_cast<char*>(base) + (size_t)c * red_ws_bytes()).out;
}

// Per-cell fold of K sums: block partials into cell c's workspace, the cell's
// last chunk folds them and runs epi(sums) in thread 0.
template <int K, class Epi>
__device__ __forceinline__ void seg_fold(double (&v)[K], char* ws_base, const BChunk& ck, int nchunk, Epi epi) {
  __shared__ double sh[32 * K];
  RedWs w = red_ws(cell_ws(ws_base, ck.cell));
  block_sum_multi<K>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) w.part[k * kMaxPartials + ck.j] = v[k];
  }
  if (arrive_last_n(w.counter, nchunk)) {
    double f[K];
    fold_sum_multi<K>(w.part, kMaxPartials, nchunk, f, sh);
    if (threadIdx.x == 0) {
      epi(f, w);
      *w.counter = 0u;
    }
  }
}

// ------------------------------------------------------------------ batched PCG

template <typename T>
struct BPcg {
  T *r, *z, *p, *Ap;
  PcgState* st;  // one per cell
  char* red;     // per-cell reduction workspaces of the vector steps
};

// r = b - Ap (A x formed before), z = invd r, p = z; per-cell rz, rr and the
// start-of-solve decisions of pcg_start_kernel.  Threshold of cell c:
// thr^2 = max(abs_sq[c] (or abs_sq0), (rel max(||r0||, rel_floor))^2).  With
// outer_rr, cell c first checks outer_rr[c] <= outer_thr_sq[c] (the enclosing
// refinement's FP64 residual) and does nothing when it holds.  live[c] == 0:
// the cell takes no part (inactive, not converged).
template <typename T>
__global__ void __launch_bounds__(kThreads) bpcg_start_kernel(BVec V, BPcg<T> w, const T* __restrict__ b,
                                                              const T* __restrict__ invd, const double* abs_sq,
                                                              double abs_sq0, double rel, double rel_floor,
                                                              const char* outer_red, const double* outer_thr_sq,
                                                              const int* live, int mode) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (live && !live[ck.cell]) {
    if (ck.j == 0 && threadIdx.x == 0) w.st[ck.cell] = PcgState{};
    return;
  }
  double v[2] = {0.0, 0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const T r = b[i] - w.Ap[i];
    w.r[i] = r;
    const T z = invd ? r * invd[i] : r;
    w.z[i] = z;
    w.p[i] = z;
    v[0] += double(r) * double(z);
    v[1] += double(r) * double(r);
  }
  const int c = ck.cell;
  seg_fold<2>(v, w.red, ck, V.nchunk[c], [&](const double* f, RedWs&) {
    PcgState& st = w.st[c];
    const double RZ = f[0], RR = f[1];
    st.rz = RZ;
    st.rr = RR;
    st.rr0 = RR;
    const double t = rel > 0.0 ? rel * fmax(sqrt(RR), rel_floor) : 0.0;
    const double a = abs_sq ? abs_sq[c] : abs_sq0;
    st.thr_sq = fmax(a, t * t);
    st.alpha = st.beta = 0.0;
    st.breakdown = 0;
    st.nonfinite = !isfinite(RR) || !isfinite(RZ);
    st.steps = 0;
    st.iter = 0;
    st.converged = 0;
    st.active = 1;
    st.outer_done = 0;
    st.outer_rr = 0.0;
    if (outer_red) st.outer_rr = cell_out(outer_red, c)[0];
    if (outer_red && isfinite(st.outer_rr) && !(st.outer_rr > outer_thr_sq[c])) {
      st.outer_done = 1;
      st.active = 0;
    } else if (st.nonfinite || (outer_red && !isfinite(st.outer_rr))) {
      st.nonfinite = 1;
      st.active = 0;
    } else if (!(RR > st.thr_sq)) {
      st.converged = 1;
      st.active = 0;
    } else if (mode == PCG_STRICT && !(RZ > 0.0)) {
      st.breakdown = 1;
      st.active = 0;
    }
  });
}

// alpha from the action's per-cell p . Ap, x += alpha p, r -= alpha Ap, z = invd r,
// per-cell rz and rr, then the state bookkeeping of pcg_update_dot_kernel.
template <typename T>
__global__ void __launch_bounds__(kThreads) bpcg_update_kernel(BVec V, BPcg<T> w, T* __restrict__ x,
                                                               const T* __restrict__ invd, int mode,
                                                               const char* dot_red) {
  const BChunk ck = V.chunks[blockIdx.x];
  const int c = ck.cell;
  PcgState* S = w.st + c;
  if (!S->active) return;
  const double PAP = cell_out(dot_red, c)[kOutDot];
  const bool ok = isfinite(PAP) && PAP > 0.0;
  const double alpha = S->rz / PAP;
  const T a = T(alpha);
  double v[2] = {0.0, 0.0};
  if (ok) {
    for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
      x[i] = x[i] + a * w.p[i];
      const T r = w.r[i] - a * w.Ap[i];
      w.r[i] = r;
      const T z = invd ? r * invd[i] : r;
      w.z[i] = z;
      v[0] += double(r) * double(z);
      v[1] += double(r) * double(r);
    }
  }
  seg_fold<2>(v, w.red, ck, V.nchunk[c], [&](const double* f, RedWs&) {
    PcgState& st = *S;
    const double RZ = f[0], RR = f[1];
    st.iter += 1;
    if (!ok) {
      if (!isfinite(PAP)) st.nonfinite = 1;
      if (!(PAP > 0.0)) st.breakdown = 1;
      st.active = 0;
      return;
    }
    st.alpha = alpha;
    st.steps += 1;
    if (!isfinite(RR) || !isfinite(RZ)) st.nonfinite = 1;
    st.rr = RR;
    if (!(RR > st.thr_sq)) {
      st.converged = 1;
      st.active = 0;
    } else {
      if (mode == PCG_STRICT && !(RZ > 0.0)) st.breakdown = 1;
      st.beta = (mode == PCG_STRICT) ? RZ / st.rz : ((st.rz > 0.0) ? RZ / st.rz : 0.0);
      st.rz = RZ;
    }
    if (st.breakdown || st.nonfinite) st.active = 0;
  });
}

template <typename T>
__global__ void bpcg_dir_kernel(BVec V, BPcg<T> w) {
  const BChunk ck = V.chunks[blockIdx.x];
  const PcgState* S = w.st + ck.cell;
  if (!S->active) return;
  const T beta = T(S->beta);
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) w.p[i] = w.z[i] + beta * w.p[i];
}

// number of cells still iterating -> *out
__global__ void bpcg_count_kernel(int n_cells, const PcgState* st, int* out) {
  __shared__ int sh[32];
  int k = 0;
  for (int c = threadIdx.x; c < n_cells; c += blockDim.x) k += st[c].active ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    *out = t;
  }
}

// One batched operator y = A x over every cell, guarded per cell by guard[c * stride].
template <typename T>
using BatchOp = std::function<int(const T* x, T* y, const int* guard, int guard_stride, bool dot, cudaStream_t s)>;

struct BpcgThr {
  const double* abs_sq = nullptr;  // per cell
  double abs_sq0 = 0.0;
  double rel = 0.0, rel_floor = 0.0;
  const char* outer_red = nullptr;
  const double* outer_thr_sq = nullptr;
  const int* live = nullptr;  // per cell, 0: no part in this solve
};

constexpr int kStateInts = (int)(sizeof(PcgState) / sizeof(int));
static_assert(sizeof(PcgState) % sizeof(int) == 0, "PcgState is not a whole number of ints");

// Runs the batched PCG from x (initial iterate) for every cell; the caller has
// not formed r.  Chunks of check_every iterations are captured as one CUDA graph
// (keyed by every pointer and value the launches read) and the host reads the
// number of still-active cells after each chunk.
template <typename T>
int bpcg_run(const phastb_batch* B, const BatchOp<T>& A, const GraphKey& op_key, const BVec& V, const BPcg<T>& w,
             const T* b, const T* invd, T* x, const BpcgThr& thr, int maxiter, int check_every, int mode,
             const char* dot_red, int* d_count, int* h_count, cudaStream_t s) {
  int st;
  if ((st = A(x, w.Ap, thr.live, 1, false, s))) return st;
  {
    note_launch();
    bpcg_start_kernel<T><<<V.n_chunks, kThreads, 0, s>>>(V, w, b, invd, thr.abs_sq, thr.abs_sq0, thr.rel,
                                                         thr.rel_floor, thr.outer_red, thr.outer_thr_sq, thr.live,
                                                         mode);
  }
  if ((st = last_launch_status())) return st;
  const int* guard = &w.st[0].active;
  auto iterate = [&](int k_iters) -> int {
    int e;
    for (int k = 0; k < k_iters; ++k) {
      if ((e = A(w.p, w.Ap, guard, kStateInts, true, s))) return e;
      { note_launch(); bpcg_update_kernel<T><<<V.n_chunks, kThreads, 0, s>>>(V, w, x, invd, mode, dot_red); }
      { note_launch(); bpcg_dir_kernel<T><<<V.n_chunks, kThreads, 0, s>>>(V, w); }
    }
    { note_launch(); bpcg_count_kernel<<<1, 256, 0, s>>>(B->n_cells, w.st, d_count); }
    return last_launch_status();
  };
  GraphKey key = op_key;
  key_val(key, w);
  key_val(key, x);
  key_val(key, invd);
  key_val(key, V);
  key_val(key, mode);
  key_val(key, check_every);
  key_val(key, dot_red);
  key_val(key, d_count);
  const int word = sizeof(T);
  key_val(key, word);
  long long glaunch = 0;
  cudaGraphExec_t gexec =
      maxiter >= check_every ? graph_for(key, s, [&] { return iterate(check_every); }, &glaunch) : nullptr;
  int it = 0;
  while (it < maxiter) {
    const int chunk = std::min(check_every, maxiter - it);
    if (gexec && chunk == check_every) {
      note_launch(glaunch);
      if ((st = cuda_status(cudaGraphLaunch(gexec, s)))) return st;
    } else if ((st = iterate(chunk))) {
      return st;
    }
    it += chunk;
    if ((st = cuda_status(cudaMemcpyAsync(h_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    if (*h_count == 0) break;
  }
  return PHASTB_OK;
}

// ------------------------------------------------------------ pointwise helpers

// xc = where(fixed, vals, 0); x0f = where(fixed, 0, x0); invd = 1/where(fixed, 1, diag) (in place)
template <typename T>
__global__ void b_mech_setup_kernel(long long n, const uint8_t* __restrict__ fixed, const double* __restrict__ vals,
                                    const double* __restrict__ x0, double* __restrict__ xc, double* __restrict__ x0f,
                                    T* __restrict__ invd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const bool f = fixed[i];
    xc[i] = f ? vals[i] : 0.0;
    x0f[i] = f ? 0.0 : (x0 ? x0[i] : 0.0);
    invd[i] = T(1) / (f ? T(1) : invd[i]);
  }
}

// bf = where(free, rhs - image, 0) and per cell ||bf||^2 -> bb[c]; with rtol/atol
// also thr_sq[c] = max(rtol ||bf||, atol)^2 (the solve's stopping threshold).
__global__ void __launch_bounds__(kThreads) b_rhs_kernel(BVec V, const uint8_t* __restrict__ fixed,
                                                         const double* __restrict__ rhs,
                                                         const double* __restrict__ image, double* __restrict__ bf,
                                                         float* __restrict__ bf32, char* red, double* bb,
                                                         double* thr_sq, double rtol, double atol) {
  const BChunk ck = V.chunks[blockIdx.x];
  double v[1] = {0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const double r = fixed[i] ? 0.0 : (rhs ? rhs[i] : 0.0) - image[i];
    bf[i] = r;
    if (bf32) bf32[i] = float(r);
    v[0] += r * r;
  }
  const int c = ck.cell;
  seg_fold<1>(v, red, ck, V.nchunk[c], [&](const double* f, RedWs& w) {
    w.out[0] = f[0];
    if (bb) bb[c] = f[0];
    if (thr_sq) {
      const double t = fmax(rtol * sqrt(f[0]), atol);
      thr_sq[c] = t * t;
    }
  });
}

__global__ void b_where_kernel(long long n, const uint8_t* __restrict__ fixed, const double* __restrict__ a,
                               const double* __restrict__ b, double* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = fixed[i] ? b[i] : a[i];
}

template <typename Ts, typename Td>
__global__ void b_convert_kernel(long long n, const Ts* __restrict__ a, Td* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = Td(a[i]);
}

__global__ void b_add_kernel(long long n, const float* __restrict__ dx, double* __restrict__ x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] += double(dx[i]);
}

inline int grid_ll(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}

// per-cell (iterations, converged, nonfinite, breakdown, rr, outer_done, outer_rr) read back to the host
int fetch_states(const phastb_batch* B, const PcgState* d_st, std::vector<PcgState>* h, cudaStream_t s) {
  h->resize(B->n_cells);
  int st = cuda_status(cudaMemcpyAsync(h->data(), d_st, sizeof(PcgState) * B->n_cells, cudaMemcpyDeviceToHost, s));
  if (st) return st;
  return cuda_status(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------ box-KKT helpers

// cells whose active-set loop has finished (live[c] == 0) are left untouched
__global__ void b_kkt_setup_kernel(BVec V, const int* __restrict__ live, const uint8_t* __restrict__ la,
                                   const uint8_t* __restrict__ ua, const double* __restrict__ lower, double upper,
                                   const double* __restrict__ initial, const double* __restrict__ diag,
                                   uint8_t* __restrict__ fixed, double* __restrict__ known, double* __restrict__ x0f,
                                   double* __restrict__ invd) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (!live[ck.cell]) return;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const bool peq = lower[i] == upper;
    const bool f = la[i] || ua[i] || peq;
    fixed[i] = f;
    known[i] = f ? (ua[i] ? upper : lower[i]) : 0.0;
    x0f[i] = f ? 0.0 : (initial ? initial[i] : 0.0);
    invd[i] = 1.0 / (f ? 1.0 : diag[i]);
  }
}

__global__ void b_kkt_rhs_kernel(BVec V, const int* __restrict__ live, const uint8_t* __restrict__ fixed,
                                 const double* __restrict__ rhs, const double* __restrict__ image,
                                 double* __restrict__ bf) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (!live[ck.cell]) return;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) bf[i] = fixed[i] ? 0.0 : rhs[i] - image[i];
}

__global__ void b_kkt_where_kernel(BVec V, const int* __restrict__ live, const uint8_t* __restrict__ fixed,
                                   const double* __restrict__ a, const double* __restrict__ b,
                                   double* __restrict__ out) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (!live[ck.cell]) return;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) out[i] = fixed[i] ? b[i] : a[i];
}

// out = a on cells with keep[c] != 0, out = b elsewhere
__global__ void b_select_kernel(BVec V, const int* __restrict__ keep, const double* __restrict__ a,
                                const double* __restrict__ b, double* __restrict__ out) {
  const BChunk ck = V.chunks[blockIdx.x];
  const double* src = keep[ck.cell] ? a : b;
  if (src == out) return;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) out[i] = src[i];
}

__global__ void b_copy_live_kernel(BVec V, const int* __restrict__ live, const double* __restrict__ a,
                                   double* __restrict__ out) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (!live[ck.cell]) return;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) out[i] = a[i];
}

// ||rhs - A d||^2 per cell -> red_c.out[0] (the staggered solver's damage residual)
__global__ void __launch_bounds__(kThreads) b_resid_norm_kernel(BVec V, const double* __restrict__ rhs,
                                                                const double* __restrict__ Ad, char* red) {
  const BChunk ck = V.chunks[blockIdx.x];
  double v[1] = {0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const double r = rhs[i] - Ad[i];
    v[0] += r * r;
  }
  seg_fold<1>(v, red, ck, V.nchunk[ck.cell], [&](const double* f, RedWs& w) { w.out[0] = f[0]; });
}

// Active-set update and KKT audit of the updated sets (kkt_update_kernel then
// kkt_audit_kernel, elementwise the same); per cell out[0] set changes,
// out[1] violations, out[2..4] max |free grad|, |projected grad|, |complementarity|.
__global__ void __launch_bounds__(kThreads) b_kkt_update_kernel(BVec V, const int* __restrict__ live,
                                                                const uint8_t* __restrict__ fixed,
                                                                const double* __restrict__ cand,
                                                                const double* __restrict__ Acand,
                                                                const double* __restrict__ rhs,
                                                                const double* __restrict__ lower, double upper,
                                                                double kkt_tol, uint8_t* __restrict__ la,
                                                                uint8_t* __restrict__ ua, double* __restrict__ grad,
                                                                char* red) {
  const BChunk ck = V.chunks[blockIdx.x];
  const int c = ck.cell;
  if (!live[c]) return;
  double chg = 0, cnt = 0, fs = 0, pg = 0, cm = 0;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const double gr = Acand[i] - rhs[i];
    grad[i] = gr;
    const double s = cand[i], lo = lower[i];
    const bool fr = !fixed[i];
    const bool add_l = fr && (s < lo);
    const bool add_u = fr && (s > upper);
    const bool rel_l = la[i] && (gr < -kkt_tol);
    const bool rel_u = ua[i] && (gr > kkt_tol);
    if (add_l || add_u || rel_l || rel_u) chg += 1.0;
    const bool l = (la[i] || add_l) && !rel_l;
    const bool u = (ua[i] || add_u) && !rel_u;
    la[i] = l;
    ua[i] = u;
    const bool peq = lo == upper;
    const bool fx = l || u || peq;
    if (s < lo || s > upper) cnt += 1.0;
    if (l && gr < -kkt_tol) cnt += 1.0;
    if (u && -gr < -kkt_tol) cnt += 1.0;
    if (!fx) {
      fs = fmax(fs, fabs(gr));
      pg = fmax(pg, fabs(gr));
    }
    if (l) {
      pg = fmax(pg, fabs(fmin(gr, 0.0)));
      cm = fmax(cm, fabs(fmax(gr, 0.0) * (s - lo)));
    }
    if (u) {
      pg = fmax(pg, fabs(fmax(gr, 0.0)));
      cm = fmax(cm, fabs(fmax(-gr, 0.0) * (upper - s)));
    }
  }
  __shared__ double sh[32];
  RedWs w = red_ws(cell_ws(red, c));
  const int nch = V.nchunk[c];
  double v = block_sum(chg, sh);
  if (threadIdx.x == 0) w.part[ck.j] = v;
  v = block_sum(cnt, sh);
  if (threadIdx.x == 0) w.part[kMaxPartials + ck.j] = v;
  const double mx[3] = {fs, pg, cm};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v = block_max(mx[k], sh);
    if (threadIdx.x == 0) w.part[(k + 2) * kMaxPartials + ck.j] = v;
  }
  if (arrive_last_n(w.counter, nch)) {
    double t = fold_sum(w.part, nch, sh);
    if (threadIdx.x == 0) w.out[0] = t;
    t = fold_sum(w.part + kMaxPartials, nch, sh);
    if (threadIdx.x == 0) w.out[1] = t;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      t = fold_max(w.part + (k + 2) * kMaxPartials, nch, sh);
      if (threadIdx.x == 0) w.out[k + 2] = t;
    }
    if (threadIdx.x == 0) *w.counter = 0u;
  }
}

// Per cell after one active-set step: PCG iterations, then failed (not converged,
// breakdown, non-finite), finished (no set change: KKT audit verdict) or go on.
// status[c]: 0 running, 1 converged, 2 not converged, 3 breakdown, 4 non-finite.
__global__ void b_kkt_decide_kernel(int n_cells, int maxiter, const PcgState* st, const char* red, int* live,
                                    int* status, int* iters, int* sets, int* kkt_ok, double kkt_tol, int* running) {
  __shared__ int sh[32];
  int k = 0;
  for (int c = threadIdx.x; c < n_cells; c += blockDim.x) {
    if (!live[c]) continue;
    const PcgState& S = st[c];
    iters[c] += S.converged ? S.steps : min(S.iter, maxiter);
    sets[c] += 1;
    const double* o = cell_out(red, c);
    if (S.nonfinite) {
      status[c] = 4;
      live[c] = 0;
    } else if (S.breakdown) {
      status[c] = 3;
      live[c] = 0;
    } else if (!S.converged) {
      status[c] = 2;
      live[c] = 0;
    } else if (o[0] == 0.0) {
      kkt_ok[c] = o[1] == 0.0 && o[2] <= kkt_tol && o[3] <= kkt_tol && o[4] <= kkt_tol;
      status[c] = kkt_ok[c] ? 1 : 2;
      live[c] = 0;
    } else {
      ++k;
    }
  }
  for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    *running = t;
  }
}

// per-cell damage linear tolerance from the residual of the start iterate:
// tol = max(min(lin_tol, 0.1 kkt_tol / max(r0, 1)), min_tol) (staggered.py:766-770)
__global__ void b_lin_tol_kernel(int n_cells, const char* red, double lin_tol, double kkt_tol, double min_tol,
                                 double* tol, double* r0) {
  for (int c = threadIdx.x; c < n_cells; c += blockDim.x) {
    const double r = sqrt(cell_out(red, c)[0]);
    r0[c] = r;
    tol[c] = fmax(fmin(lin_tol, 0.1 * kkt_tol / fmax(r, 1.0)), min_tol);
  }
}

// rel threshold per cell for the Dirichlet PCG: the start kernel takes a scalar
// rel, so a per-cell tolerance is applied as thr_sq = (tol_c max(||r0||, 1))^2
// by a dedicated start variant below.
template <typename T>
__global__ void __launch_bounds__(kThreads) bpcg_start_rel_kernel(BVec V, BPcg<T> w, const T* __restrict__ b,
                                                                  const T* __restrict__ invd,
                                                                  const double* __restrict__ rel_c,
                                                                  const int* __restrict__ live, int mode) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (live && !live[ck.cell]) {
    if (ck.j == 0 && threadIdx.x == 0) w.st[ck.cell] = PcgState{};
    return;
  }
  double v[2] = {0.0, 0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const T r = b[i] - w.Ap[i];
    w.r[i] = r;
    const T z = invd ? r * invd[i] : r;
    w.z[i] = z;
    w.p[i] = z;
    v[0] += double(r) * double(z);
    v[1] += double(r) * double(r);
  }
  const int c = ck.cell;
  seg_fold<2>(v, w.red, ck, V.nchunk[c], [&](const double* f, RedWs&) {
    PcgState& st = w.st[c];
    const double RZ = f[0], RR = f[1];
    st = PcgState{};
    st.rz = RZ;
    st.rr = RR;
    st.rr0 = RR;
    const double t = rel_c[c] * fmax(sqrt(RR), 1.0);
    st.thr_sq = t * t;
    st.nonfinite = !isfinite(RR) || !isfinite(RZ);
    st.active = 1;
    if (st.nonfinite) {
      st.active = 0;
    } else if (!(RR > st.thr_sq)) {
      st.converged = 1;
      st.active = 0;
    } else if (mode == PCG_STRICT && !(RZ > 0.0)) {
      st.breakdown = 1;
      st.active = 0;
    }
  });
}

// x_out = factor x with each cell's E[comp] = value; values_out = 0 except there
__global__ void b_predictor_kernel(BVec V, const BatchCell* cells, const double* __restrict__ x, double factor,
                                   int comp, double value, double* __restrict__ x_out,
                                   double* __restrict__ values_out) {
  const BChunk ck = V.chunks[blockIdx.x];
  const BatchCell& cl = cells[ck.cell];
  const long long ctrl = cl.mech_off + 3LL * cl.g.n_red + comp;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const bool c = i == ctrl;
    x_out[i] = c ? value : factor * x[i];
    if (values_out) values_out[i] = c ? value : 0.0;
  }
}

// staggered change parts per cell: out[5c..5c+4] = ||du~||, ||u~||, max|dE|, max|E|, max|dd|
__global__ void __launch_bounds__(kThreads) b_change_mech_kernel(BVec V, const BatchCell* cells,
                                                                 const double* __restrict__ xn,
                                                                 const double* __restrict__ xo, char* red,
                                                                 double* out) {
  const BChunk ck = V.chunks[blockIdx.x];
  const BatchCell& cl = cells[ck.cell];
  const long long nu_end = cl.mech_off + 3LL * cl.g.n_red;
  double du = 0, un = 0, dE = 0, Ei = 0;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const double a = xn[i], b = a - xo[i];
    if (i < nu_end) {
      du += b * b;
      un += a * a;
    } else {
      dE = fmax(dE, fabs(b));
      Ei = fmax(Ei, fabs(a));
    }
  }
  __shared__ double sh[32];
  RedWs w = red_ws(cell_ws(red, ck.cell));
  const int nch = V.nchunk[ck.cell];
  double v = block_sum(du, sh);
  if (threadIdx.x == 0) w.part[ck.j] = v;
  v = block_sum(un, sh);
  if (threadIdx.x == 0) w.part[kMaxPartials + ck.j] = v;
  v = block_max(dE, sh);
  if (threadIdx.x == 0) w.part[2 * kMaxPartials + ck.j] = v;
  v = block_max(Ei, sh);
  if (threadIdx.x == 0) w.part[3 * kMaxPartials + ck.j] = v;
  if (arrive_last_n(w.counter, nch)) {
    double* o = out + 5 * (size_t)ck.cell;
    double t = fold_sum(w.part, nch, sh);
    if (threadIdx.x == 0) o[0] = sqrt(t);
    t = fold_sum(w.part + kMaxPartials, nch, sh);
    if (threadIdx.x == 0) o[1] = sqrt(t);
    t = fold_max(w.part + 2 * kMaxPartials, nch, sh);
    if (threadIdx.x == 0) o[2] = t;
    t = fold_max(w.part + 3 * kMaxPartials, nch, sh);
    if (threadIdx.x == 0) {
      o[3] = t;
      *w.counter = 0u;
    }
  }
}

__global__ void __launch_bounds__(kThreads) b_change_damage_kernel(BVec V, const double* __restrict__ dn,
                                                                   const double* __restrict__ dol, char* red,
                                                                   double* out) {
  const BChunk ck = V.chunks[blockIdx.x];
  double dd = 0;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) dd = fmax(dd, fabs(dn[i] - dol[i]));
  __shared__ double sh[32];
  RedWs w = red_ws(cell_ws(red, ck.cell));
  const int nch = V.nchunk[ck.cell];
  const double v = block_max(dd, sh);
  if (threadIdx.x == 0) w.part[ck.j] = v;
  if (arrive_last_n(w.counter, nch)) {
    const double t = fold_max(w.part, nch, sh);
    if (threadIdx.x == 0) {
      out[5 * (size_t)ck.cell + 4] = t;
      *w.counter = 0u;
    }
  }
}

// ------------------------------------------------------------ batched multigrid
//
// The V-cycle of gmg.cu (Chebyshev smoothing in D^-1 A, trilinear transfers,
// coarse-level mean removal, a Jacobi step on the fine E rows) on every cell of a
// packed batch at once, FP32.  Each level is a packed plan of its own (coarse
// vectors use the mechanics layout with six unused, zero entries per cell); the
// Chebyshev interval and therefore 1/theta and 1/delta differ per cell (one
// lambda_max per cell and level), the step coefficients c1 and the 2 rho of c2 do
// not.  Every kernel is guarded per cell by the Krylov engine's `active` flag.

__device__ __forceinline__ bool cell_live(const int* guard, int stride, int c) {
  return !guard || guard[(size_t)c * stride] != 0;
}

// res = b (less the cell's pending per-component mean when bsum_red is given, stored back
// into b); d = invd b / theta_c; x = d  (gmg_cheb_first_b)
__global__ void bg_first_b_kernel(BVec V, const BatchCell* cells, float* __restrict__ b,
                                  const float* __restrict__ invd, const double* __restrict__ inv_theta,
                                  float* __restrict__ res, float* __restrict__ d, float* __restrict__ x,
                                  const char* bsum_red, const int* guard, int gstride) {
  const BChunk ck = V.chunks[blockIdx.x];
  const int c = ck.cell;
  if (!cell_live(guard, gstride, c)) return;
  const BatchCell& cl = cells[c];
  const float it = float(inv_theta[c]);
  float m[3] = {0.f, 0.f, 0.f};
  if (bsum_red) {
    const double* o = cell_out(bsum_red, c);
    for (int k = 0; k < 3; ++k) m[k] = float(o[k] / cl.g.n_red);
  }
  const long long nu = cl.mech_off + 3LL * cl.g.n_red;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    float bi = b[i];
    if (bsum_red && i < nu) {
      bi -= m[(i - cl.mech_off) % 3];
      b[i] = bi;
    }
    res[i] = bi;
    const float di = invd[i] * bi * it;
    d[i] = di;
    x[i] = di;
  }
}

// res = b - Ax; d = invd res / theta_c; x += d; on the fine level (e_rows) the E rows of x get
// the Jacobi step of the macro-strain block, x_E = fixed ? 0 : b_E / diag_E  (gmg_cheb_first_res)
__global__ void bg_first_res_kernel(BVec V, const BatchCell* cells, const float* __restrict__ b,
                                    const float* __restrict__ Ax, const float* __restrict__ invd,
                                    const double* __restrict__ inv_theta, float* __restrict__ res,
                                    float* __restrict__ d, float* __restrict__ x, int e_rows,
                                    const float* __restrict__ diag, const uint8_t* __restrict__ fixed,
                                    const int* guard, int gstride) {
  const BChunk ck = V.chunks[blockIdx.x];
  const int c = ck.cell;
  if (!cell_live(guard, gstride, c)) return;
  const BatchCell& cl = cells[c];
  const float it = float(inv_theta[c]);
  const long long nu = cl.mech_off + 3LL * cl.g.n_red;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const float r = b[i] - Ax[i];
    res[i] = r;
    const float di = invd[i] * r * it;
    d[i] = di;
    if (e_rows && i >= nu)
      x[i] = fixed[i] ? 0.f : b[i] / diag[i];
    else
      x[i] = x[i] + di;
  }
}

__device__ __forceinline__ int bg_wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// r_c = P^T r_f per coarse node (full weighting, fine rows in `mask` read as zero), and each
// cell's three component sums of r_c (its mean, removed by the first coarse smoothing step).
__global__ void __launch_bounds__(kThreads) bg_restrict_kernel(BVec Vc, const BatchCell* fcells,
                                                               const BatchCell* ccells, const float* __restrict__ rf,
                                                               const uint8_t* __restrict__ mask,
                                                               float* __restrict__ rc, char* sum_red,
                                                               const int* guard, int gstride) {
  const BChunk ck = Vc.chunks[blockIdx.x];
  const int c = ck.cell;
  if (!cell_live(guard, gstride, c)) return;
  const VoxGeom& f = fcells[c].g;
  const VoxGeom& cg = ccells[c].g;
  const long long fo = fcells[c].mech_off, co = ccells[c].mech_off, no = ccells[c].node_off;
  double v[3] = {0.0, 0.0, 0.0};
  for (int n = ck.begin + threadIdx.x; n < ck.end; n += blockDim.x) {
    const int ln = (int)(n - no);
    const int I = ln % cg.rx, rem = ln / cg.rx, J = rem % cg.ry, K = rem / cg.ry;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int oz = -1; oz <= 1; ++oz) {
      const int k = bg_wrap(2 * K + oz, f.nz);
      const float wz = oz == 0 ? 1.f : 0.5f;
      for (int oy = -1; oy <= 1; ++oy) {
        const int j = bg_wrap(2 * J + oy, f.ny);
        const float wy = oy == 0 ? 1.f : 0.5f;
        for (int ox = -1; ox <= 1; ++ox) {
          const int i = bg_wrap(2 * I + ox, f.nx);
          const float wgt = (ox == 0 ? 1.f : 0.5f) * wy * wz;
          const long long fn = fo + 3LL * ((long long)i + (long long)f.rx * ((long long)j + (long long)f.ry * k));
          a0 += wgt * ((mask && mask[fn + 0]) ? 0.f : rf[fn + 0]);
          a1 += wgt * ((mask && mask[fn + 1]) ? 0.f : rf[fn + 1]);
          a2 += wgt * ((mask && mask[fn + 2]) ? 0.f : rf[fn + 2]);
        }
      }
    }
    const long long cn = co + 3LL * ln;
    rc[cn + 0] = a0;
    rc[cn + 1] = a1;
    rc[cn + 2] = a2;
    v[0] += double(a0);
    v[1] += double(a1);
    v[2] += double(a2);
  }
  seg_fold<3>(v, sum_red, ck, Vc.nchunk[c], [&](const double* f3, RedWs& w) {
    for (int k = 0; k < 3; ++k) w.out[k] = f3[k];
  });
}

// x_f += P (x_c - mean_c) per fine node, rows in `mask` untouched  (gmg_prolong_add)
__global__ void bg_prolong_kernel(BVec Vf, const BatchCell* fcells, const BatchCell* ccells,
                                  const float* __restrict__ xc, const uint8_t* __restrict__ mask,
                                  float* __restrict__ xf, const char* csum_red, const int* guard, int gstride) {
  const BChunk ck = Vf.chunks[blockIdx.x];
  const int c = ck.cell;
  if (!cell_live(guard, gstride, c)) return;
  const VoxGeom& f = fcells[c].g;
  const VoxGeom& cg = ccells[c].g;
  const long long fo = fcells[c].mech_off, co = ccells[c].mech_off, no = fcells[c].node_off;
  float m0 = 0.f, m1 = 0.f, m2 = 0.f;
  if (csum_red) {
    const double* o = cell_out(csum_red, c);
    m0 = float(o[0] / cg.n_red);
    m1 = float(o[1] / cg.n_red);
    m2 = float(o[2] / cg.n_red);
  }
  for (int n = ck.begin + threadIdx.x; n < ck.end; n += blockDim.x) {
    const int ln = (int)(n - no);
    const int i = ln % f.rx, rem = ln / f.rx, j = rem % f.ry, k = rem / f.ry;
    int I[2] = {i >> 1, 0}, J[2] = {j >> 1, 0}, K[2] = {k >> 1, 0};
    float wx[2] = {1.f, 0.f}, wy[2] = {1.f, 0.f}, wz[2] = {1.f, 0.f};
    int cx = 1, cy = 1, cz = 1;
    if (i & 1) { I[1] = bg_wrap(I[0] + 1, cg.nx); wx[0] = wx[1] = 0.5f; cx = 2; }
    if (j & 1) { J[1] = bg_wrap(J[0] + 1, cg.ny); wy[0] = wy[1] = 0.5f; cy = 2; }
    if (k & 1) { K[1] = bg_wrap(K[0] + 1, cg.nz); wz[0] = wz[1] = 0.5f; cz = 2; }
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int z = 0; z < cz; ++z)
      for (int yy = 0; yy < cy; ++yy)
        for (int xx = 0; xx < cx; ++xx) {
          const long long cn = co + 3LL * ((long long)I[xx] + (long long)cg.rx * ((long long)J[yy] + (long long)cg.ry * K[z]));
          const float wgt = wx[xx] * wy[yy] * wz[z];
          a0 += wgt * (xc[cn + 0] - m0);
          a1 += wgt * (xc[cn + 1] - m1);
          a2 += wgt * (xc[cn + 2] - m2);
        }
    const long long fn = fo + 3LL * ln;
    if (!(mask && mask[fn + 0])) xf[fn + 0] += a0;
    if (!(mask && mask[fn + 1])) xf[fn + 1] += a1;
    if (!(mask && mask[fn + 2])) xf[fn + 2] += a2;
  }
}

// each cell's three component sums of a level vector (gmg_mean3), over the level's node chunks
__global__ void __launch_bounds__(kThreads) bg_mean3_kernel(BVec Vn, const BatchCell* cells,
                                                            const float* __restrict__ x, char* red, const int* guard,
                                                            int gstride) {
  const BChunk ck = Vn.chunks[blockIdx.x];
  const int c = ck.cell;
  if (!cell_live(guard, gstride, c)) return;
  const long long mo = cells[c].mech_off, no = cells[c].node_off;
  double v[3] = {0.0, 0.0, 0.0};
  for (int n = ck.begin + threadIdx.x; n < ck.end; n += blockDim.x) {
    const long long i = mo + 3LL * (n - no);
    v[0] += double(x[i]);
    v[1] += double(x[i + 1]);
    v[2] += double(x[i + 2]);
  }
  seg_fold<3>(v, red, ck, Vn.nchunk[c], [&](const double* f3, RedWs& w) {
    for (int k = 0; k < 3; ++k) w.out[k] = f3[k];
  });
}

// power iteration for lambda_max(D^-1 A) per cell: a deterministic non-smooth start ...
__global__ void bg_power_init_kernel(BVec V, const BatchCell* cells, const uint8_t* __restrict__ mask,
                                     float* __restrict__ v) {
  const BChunk ck = V.chunks[blockIdx.x];
  const BatchCell& cl = cells[ck.cell];
  const long long nu = cl.mech_off + 3LL * cl.g.n_red;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    unsigned h = (unsigned)(i - cl.mech_off) * 2654435761u;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    v[i] = (i >= nu || (mask && mask[i])) ? 0.f : float(0.5 + (h & 0xffff) / 65536.0);
  }
}

// ... v <- D^-1 A v with its D-norm squared per cell (out[0]) ...
__global__ void __launch_bounds__(kThreads) bg_power_next_kernel(BVec V, const float* __restrict__ Av,
                                                                 const float* __restrict__ invd,
                                                                 const float* __restrict__ diag,
                                                                 float* __restrict__ v, char* red) {
  const BChunk ck = V.chunks[blockIdx.x];
  double acc[1] = {0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const float z = invd[i] * Av[i];
    v[i] = z;
    acc[0] += double(z) * double(diag[i]) * double(z);
  }
  seg_fold<1>(acc, red, ck, V.nchunk[ck.cell], [&](const double* f, RedWs& w) { w.out[0] = f[0]; });
}

// ... normalised by that norm ...
__global__ void bg_power_scale_kernel(BVec V, const char* red, float* __restrict__ v) {
  const BChunk ck = V.chunks[blockIdx.x];
  const double sm = cell_out(red, ck.cell)[0];
  const double sc = sm > 0 ? 1.0 / sqrt(sm) : 0.0;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) v[i] = float(double(v[i]) * sc);
}

// ... and the Rayleigh quotient v.Av / v.Dv over the free rows at the last step
__global__ void __launch_bounds__(kThreads) bg_power_dots_kernel(BVec V, const float* __restrict__ v,
                                                                 const float* __restrict__ Av,
                                                                 const float* __restrict__ diag,
                                                                 const uint8_t* __restrict__ mask, char* red) {
  const BChunk ck = V.chunks[blockIdx.x];
  double acc[2] = {0.0, 0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    if (mask && mask[i]) continue;
    acc[0] += double(v[i]) * double(Av[i]);
    acc[1] += double(v[i]) * double(diag[i]) * double(v[i]);
  }
  seg_fold<2>(acc, red, ck, V.nchunk[ck.cell], [&](const double* f, RedWs& w) {
    w.out[0] = f[0];
    w.out[1] = f[1];
  });
}

// per cell: lambda_max from the Rayleigh quotient (or the cached value), and the Chebyshev
// factors 1/theta and 1/delta of the interval [lmax/30, safety lmax]
__global__ void bg_cheb_factors_kernel(int n_cells, const char* red, int from_red, double* lmax, double safety,
                                       double* inv_theta, double* inv_delta) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x) {
    if (from_red) {
      const double* o = cell_out(red, c);
      lmax[c] = o[1] > 0 ? o[0] / o[1] : 1.0;
    }
    const double bmax = safety * lmax[c], amin = lmax[c] / 30.0;
    inv_theta[c] = 1.0 / (0.5 * (bmax + amin));
    inv_delta[c] = 1.0 / (0.5 * (bmax - amin));
  }
}

// fine-level mask of the multigrid: the solve's fixed rows and every E row
__global__ void bg_fine_mask_kernel(BVec V, const BatchCell* cells, const uint8_t* __restrict__ fixed,
                                    uint8_t* __restrict__ mask) {
  const BChunk ck = V.chunks[blockIdx.x];
  const BatchCell& cl = cells[ck.cell];
  const long long nu = cl.mech_off + 3LL * cl.g.n_red;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) mask[i] = fixed[i] || i >= nu;
}

// inv = mask ? 0 : 1/diag; on coarse levels the six unused entries per cell are 0 too
__global__ void bg_invert_kernel(BVec V, const BatchCell* cells, const float* __restrict__ diag,
                                 const uint8_t* __restrict__ mask, float* __restrict__ inv) {
  const BChunk ck = V.chunks[blockIdx.x];
  const BatchCell& cl = cells[ck.cell];
  const long long nu = cl.mech_off + 3LL * cl.g.n_red;
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x)
    inv[i] = ((mask && mask[i]) || (!mask && i >= nu)) ? 0.f : 1.f / diag[i];
}

// ---- batched PCG with a preconditioner (pcg_run with M): r, rr; then z = M r; rz; p = z

// r = b - Ap; rr; the start-of-solve decisions without z (rz follows once M has run)
template <typename T>
__global__ void __launch_bounds__(kThreads) bpcg_start_pre_kernel(BVec V, BPcg<T> w, const T* __restrict__ b,
                                                                  const double* abs_sq, double rel,
                                                                  const char* outer_red, const double* outer_thr_sq,
                                                                  const int* live) {
  const BChunk ck = V.chunks[blockIdx.x];
  if (live && !live[ck.cell]) {
    if (ck.j == 0 && threadIdx.x == 0) w.st[ck.cell] = PcgState{};
    return;
  }
  double v[1] = {0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    const T r = b[i] - w.Ap[i];
    w.r[i] = r;
    v[0] += double(r) * double(r);
  }
  const int c = ck.cell;
  seg_fold<1>(v, w.red, ck, V.nchunk[c], [&](const double* f, RedWs&) {
    PcgState& st = w.st[c];
    const double RR = f[0];
    st = PcgState{};
    st.rr = RR;
    st.rr0 = RR;
    const double t = rel > 0.0 ? rel * sqrt(RR) : 0.0;
    st.thr_sq = fmax(abs_sq ? abs_sq[c] : 0.0, t * t);
    st.active = 1;
    if (outer_red) st.outer_rr = cell_out(outer_red, c)[0];
    if (outer_red && isfinite(st.outer_rr) && !(st.outer_rr > outer_thr_sq[c])) {
      st.outer_done = 1;
      st.active = 0;
    } else if (!isfinite(RR) || (outer_red && !isfinite(st.outer_rr))) {
      st.nonfinite = 1;
      st.active = 0;
    } else if (!(RR > st.thr_sq)) {
      st.converged = 1;
      st.active = 0;
    }
  });
}

// rz per cell after z = M r: at the start rz itself, later beta = rz_new / rz (pcg_rz_kernel)
template <typename T>
__global__ void __launch_bounds__(kThreads) bpcg_rz_kernel(BVec V, BPcg<T> w, int start) {
  const BChunk ck = V.chunks[blockIdx.x];
  const int c = ck.cell;
  PcgState* S = w.st + c;
  if (!S->active) return;
  double v[1] = {0.0};
  for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
    v[0] += double(w.r[i]) * double(w.z[i]);
    if (start) w.p[i] = w.z[i];
  }
  seg_fold<1>(v, w.red, ck, V.nchunk[c], [&](const double* f, RedWs&) {
    PcgState& st = *S;
    const double RZ = f[0];
    if (!isfinite(RZ)) st.nonfinite = 1;
    if (start) {
      st.rz = RZ;
    } else {
      st.beta = st.rz > 0.0 ? RZ / st.rz : 0.0;
      st.rz = RZ;
    }
    if (st.nonfinite) st.active = 0;
  });
}

// alpha from the action's p.Ap; x += alpha p; r -= alpha Ap; rr and the convergence test
template <typename T>
__global__ void __launch_bounds__(kThreads) bpcg_update_pre_kernel(BVec V, BPcg<T> w, T* __restrict__ x,
                                                                   const char* dot_red) {
  const BChunk ck = V.chunks[blockIdx.x];
  const int c = ck.cell;
  PcgState* S = w.st + c;
  if (!S->active) return;
  const double PAP = cell_out(dot_red, c)[kOutDot];
  const bool ok = isfinite(PAP) && PAP > 0.0;
  const double alpha = S->rz / PAP;
  const T a = T(alpha);
  double v[1] = {0.0};
  if (ok) {
    for (int i = ck.begin + threadIdx.x; i < ck.end; i += blockDim.x) {
      x[i] = x[i] + a * w.p[i];
      const T r = w.r[i] - a * w.Ap[i];
      w.r[i] = r;
      v[0] += double(r) * double(r);
    }
  }
  seg_fold<1>(v, w.red, ck, V.nchunk[c], [&](const double* f, RedWs&) {
    PcgState& st = *S;
    const double RR = f[0];
    st.iter += 1;
    if (!ok) {
      if (!isfinite(PAP)) st.nonfinite = 1;
      if (!(PAP > 0.0)) st.breakdown = 1;
      st.active = 0;
      return;
    }
    st.alpha = alpha;
    st.steps += 1;
    if (!isfinite(RR)) st.nonfinite = 1;
    st.rr = RR;
    if (!(RR > st.thr_sq)) {
      st.converged = 1;
      st.active = 0;
    }
    if (st.nonfinite) st.active = 0;
  });
}

// ------------------------------------------------------------ workspace layout

struct Carve {
  char* p;
  size_t used = 0;
  template <typename T>
  T* take(size_t count) {
    T* r = p ? reinterpret_cast<T*>(p + used) : nullptr;
    used += align_up(sizeof(T) * count);
    return r;
  }
};

size_t n_red_ws(const phastb_batch* B) { return (size_t)B->n_cells * red_ws_bytes(); }

// every cell's reduction ticket of one per-cell workspace array back to zero
__global__ void b_reset_tickets_kernel(int n_cells, char* red) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x)
    *red_ws(cell_ws(red, c)).counter = 0u;
}

}  // namespace

// The batched elastic action: guard words per cell (stride in ints), dot: x . y per cell.
template <typename T>
int batch_mech_op(const phastb_batch* B, const VoxMat<T>& m, const uint8_t* slot, const T* d, const uint8_t* mask,
                  const T* x, T* y, char* red, const int* guard, int guard_stride, bool dot, cudaStream_t s) {
  TileBatchArgs<T> a{};
  a.cells = B->d_cells;
  a.work = B->d_work;
  a.n_blocks = (int)B->work.size();
  a.guard_stride = guard_stride;
  a.slot = slot;
  a.d = d;
  a.H = nullptr;
  a.x = x;
  a.y = y;
  a.mask = mask;
  a.ws = red;
  a.guard = guard;
  return h8_tile_batch_launch<T>(a, m, dot ? kModeDot : kModeApply, B->ox, B->oy, s);
}

int batch_damage_op(const phastb_batch* B, const VoxMat<double>& m, const uint8_t* slot, const double* H,
                    const uint8_t* mask, const double* x, double* y, char* red, const int* guard, int guard_stride,
                    bool dot, cudaStream_t s, bool scaled = true) {
  TileBatchArgs<double> a{};
  a.cells = B->d_cells;
  a.work = B->d_work;
  a.n_blocks = (int)B->work.size();
  a.guard_stride = guard_stride;
  a.slot = slot;
  a.H = H;
  a.x = x;
  a.y = y;
  a.mask = mask;
  a.ws = red;
  a.guard = guard;
  a.kappa = double(m.kappa);
  a.dscale = scaled ? 1 : 0;
  return h8_dtile_batch_launch<double>(a, m, dot, B->ox, B->oy, s);
}

int gmg_level_coefs_f32(const VoxGeom& f, const VoxGeom& c, const VoxMat<float>& m, const uint8_t* slot,
                        const float* d, const float* lam_f, const float* mu_f, float* lam_c, float* mu_c,
                        cudaStream_t s);
int gmg_coarse_diag_f32(const VoxGeom& c, const float* lam, const float* mu, float* scratch, float* diag,
                        cudaStream_t s);

namespace {

// One level of the batch's multigrid hierarchy (FP32 vectors in the level plan's layout).
struct BLevel {
  const phastb_batch* P;
  float *diag, *invd, *x, *b, *res, *dvec, *Ad, *lam, *mu;
  double *lmax, *inv_theta, *inv_delta;  // per cell
  char* red;                             // per-cell reductions of the level (means, power iteration)
  char* ared;                            // per-cell workspaces of the level's tile launches
};

struct BGmg {
  int nlev;
  BLevel L[3];
  VoxMat<float> m;
  const uint8_t* slot;
  const float* d32;
  uint8_t* mask;         // fine level: the solve's fixed rows and the E rows
  const uint8_t* fixed;  // fine level: the solve's fixed rows
  double safety;
  int deg, deg_coarse;
  const int* guard;      // the Krylov engine's per-cell active flags
  int gstride;
};

size_t bgmg_bytes(const phastb_batch* B) {
  Carve cv{nullptr};
  for (int l = 0; l < B->nlev; ++l) {
    const phastb_batch* P = l == 0 ? B : B->lev[l - 1];
    for (int k = 0; k < 7; ++k) cv.take<float>((size_t)P->n_mech);
    if (l > 0) {
      cv.take<float>(8 * (size_t)P->n_elem);
      cv.take<float>(8 * (size_t)P->n_elem);
    }
    for (int k = 0; k < 3; ++k) cv.take<double>((size_t)P->n_cells);
    cv.take<char>(n_red_ws(P));
    cv.take<char>(n_red_ws(P));
  }
  cv.take<uint8_t>((size_t)B->n_mech);
  return cv.used;
}

void bgmg_carve(BGmg& M, const phastb_batch* B, char* base) {
  Carve cv{base};
  M.nlev = B->nlev;
  for (int l = 0; l < B->nlev; ++l) {
    BLevel& L = M.L[l];
    L.P = l == 0 ? B : B->lev[l - 1];
    float** v[7] = {&L.diag, &L.invd, &L.x, &L.b, &L.res, &L.dvec, &L.Ad};
    for (auto q : v) *q = cv.take<float>((size_t)L.P->n_mech);
    L.lam = L.mu = nullptr;
    if (l > 0) {
      L.lam = cv.take<float>(8 * (size_t)L.P->n_elem);
      L.mu = cv.take<float>(8 * (size_t)L.P->n_elem);
    }
    L.lmax = cv.take<double>((size_t)L.P->n_cells);
    L.inv_theta = cv.take<double>((size_t)L.P->n_cells);
    L.inv_delta = cv.take<double>((size_t)L.P->n_cells);
    L.red = cv.take<char>(n_red_ws(L.P));
    L.ared = cv.take<char>(n_red_ws(L.P));
  }
  M.mask = cv.take<uint8_t>((size_t)B->n_mech);
}

TileBatchArgs<float> bg_args(const BGmg& M, int l, const float* x) {
  const BLevel& L = M.L[l];
  TileBatchArgs<float> a{};
  a.cells = L.P->d_cells;
  a.work = L.P->d_work;
  a.n_blocks = (int)L.P->work.size();
  a.guard = M.guard;
  a.guard_stride = M.gstride;
  a.x = x;
  a.ws = L.ared;
  if (l == 0) {
    a.slot = M.slot;
    a.d = M.d32;
    a.mask = M.mask;
  } else {
    a.lam_q = L.lam;
    a.mu_q = L.mu;
  }
  return a;
}

// y = A x on level l (the fine level's nodal block only: its smoother leaves the E rows alone)
int bg_level_apply(const BGmg& M, int l, const float* x, float* y, cudaStream_t s) {
  TileBatchArgs<float> a = bg_args(M, l, x);
  a.y = y;
  return h8_tile_batch_level_launch(a, M.m, l == 0 ? kCoefIso : kCoefQP, l == 0 ? kModeNodal : kModeApply,
                                    M.L[l].P->ox, M.L[l].P->oy, s);
}

// one fused Chebyshev step: res -= A din; dout = c1 din + c2 s_c invd res; x += dout
int bg_level_cheb(const BGmg& M, int l, const float* din, float* dout, double c1, double c2, bool scaled,
                  cudaStream_t s) {
  const BLevel& L = M.L[l];
  TileBatchArgs<float> a = bg_args(M, l, din);
  a.res = L.res;
  a.invd = L.invd;
  a.xs = L.x;
  a.d_out = dout;
  a.c1 = c1;
  a.c2 = c2;
  a.c2_scale = scaled ? L.inv_delta : nullptr;
  return h8_tile_batch_level_launch(a, M.m, l == 0 ? kCoefIso : kCoefQP, kModeCheb, L.P->ox, L.P->oy, s);
}

BVec level_mech_vec(const phastb_batch* P) { return mech_vec(P); }
BVec level_node_vec(const phastb_batch* P) { return node_vec(P); }

// Chebyshev smoothing of A x = b on level l (gmg.cu's chebyshev, per-cell interval)
int bg_chebyshev(const BGmg& M, int l, int deg, bool from_zero, bool need_res, const char* bsum_red,
                 cudaStream_t s) {
  const BLevel& L = M.L[l];
  const BVec V = level_mech_vec(L.P);
  int st;
  const double a = 1.0 / 30.0, bm = M.safety;  // interval [lmax/30, safety lmax] relative to lmax
  const double sigma = (bm + a) / (bm - a);
  if (from_zero) {
    { note_launch(); bg_first_b_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.P->d_cells, L.b, L.invd, L.inv_theta, L.res, L.dvec, L.x, bsum_red, M.guard, M.gstride); }
  } else {
    if ((st = bg_level_apply(M, l, L.x, L.Ad, s))) return st;
    { note_launch(); bg_first_res_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.P->d_cells, L.b, L.Ad, L.invd, L.inv_theta, L.res, L.dvec, L.x, l == 0, L.diag, M.fixed, M.guard, M.gstride); }
  }
  float* cur = L.dvec;
  float* oth = L.Ad;
  double rho_old = 1.0 / sigma;
  for (int k = 1; k < deg; ++k) {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    if ((st = bg_level_cheb(M, l, cur, oth, rho * rho_old, 2.0 * rho, true, s))) return st;
    std::swap(cur, oth);
    rho_old = rho;
  }
  if (need_res && (st = bg_level_cheb(M, l, cur, oth, 0.0, 0.0, false, s))) return st;
  return last_launch_status();
}

// V-cycle from level l; bsum_red: the pending mean of L.b summed by the parent's restriction;
// on coarse levels the mean of the result is left pending in L.red for the parent's prolongation
int bg_vcycle(const BGmg& M, int l, const char* bsum_red, const char** xsum_red, cudaStream_t s) {
  const BLevel& L = M.L[l];
  int st;
  *xsum_red = nullptr;
  if (l == M.nlev - 1) {
    if ((st = bg_chebyshev(M, l, M.deg_coarse, true, false, bsum_red, s))) return st;
    const BVec Vn = level_node_vec(L.P);
    { note_launch(); bg_mean3_kernel<<<Vn.n_chunks, kThreads, 0, s>>>(Vn, L.P->d_cells, L.x, L.red, M.guard, M.gstride); }
    *xsum_red = L.red;
    return last_launch_status();
  }
  if ((st = bg_chebyshev(M, l, M.deg, true, true, bsum_red, s))) return st;
  const BLevel& C = M.L[l + 1];
  const BVec Vcn = level_node_vec(C.P);
  { note_launch(); bg_restrict_kernel<<<Vcn.n_chunks, kThreads, 0, s>>>(Vcn, L.P->d_cells, C.P->d_cells, L.res, l == 0 ? M.mask : nullptr, C.b, C.red, M.guard, M.gstride); }
  const char* csum = nullptr;
  if ((st = bg_vcycle(M, l + 1, C.red, &csum, s))) return st;
  const BVec Vfn = level_node_vec(L.P);
  { note_launch(); bg_prolong_kernel<<<Vfn.n_chunks, kThreads, 0, s>>>(Vfn, L.P->d_cells, C.P->d_cells, C.x, l == 0 ? M.mask : nullptr, L.x, csum, M.guard, M.gstride); }
  if ((st = bg_chebyshev(M, l, M.deg, false, false, nullptr, s))) return st;
  if (l > 0) {
    const BVec Vn = level_node_vec(L.P);
    { note_launch(); bg_mean3_kernel<<<Vn.n_chunks, kThreads, 0, s>>>(Vn, L.P->d_cells, L.x, L.red, M.guard, M.gstride); }
    *xsum_red = L.red;
  }
  return last_launch_status();
}

// z = M^-1 r for every live cell: the fine level reads r and builds z in place
int bg_precond(const BGmg& M0, const float* r, float* z, cudaStream_t s) {
  BGmg M = M0;
  M.L[0].b = const_cast<float*>(r);
  M.L[0].x = z;
  const char* xs = nullptr;
  return bg_vcycle(M, 0, nullptr, &xs, s);
}

// Hierarchy for the current damage field: fine mask and diagonal, coarse moduli and diagonals
// (per-cell setup launches), and, unless reused, lambda_max of every level and cell by power
// iteration.  Chebyshev factors per cell from lambda_max.
int bg_setup(BGmg& M, const phastb_batch* B, char* scratch, int power_iters, bool reuse_lmax, cudaStream_t s) {
  int st;
  M.guard = nullptr;
  M.gstride = 0;
  for (int l = 0; l < M.nlev; ++l) {
    const BLevel& L = M.L[l];
    float* v[7] = {L.diag, L.invd, L.x, L.b, L.res, L.dvec, L.Ad};
    for (float* q : v)
      if ((st = cuda_status(cudaMemsetAsync(q, 0, sizeof(float) * (size_t)L.P->n_mech, s)))) return st;
    for (char* r : {L.red, L.ared})
      { note_launch(); b_reset_tickets_kernel<<<(L.P->n_cells + 255) / 256, 256, 0, s>>>(L.P->n_cells, r); }
  }
  const BVec V0 = mech_vec(B);
  { note_launch(); bg_fine_mask_kernel<<<V0.n_chunks, kThreads, 0, s>>>(V0, B->d_cells, M.fixed, M.mask); }
  for (int c = 0; c < B->n_cells; ++c) {
    const BatchCell& cl = B->cells[c];
    if ((st = h8_mech_diag_t<float>(cl.g, M.m, M.slot + cl.elem_off, nullptr, M.d32 + cl.node_off,
                                    M.L[0].diag + cl.mech_off, scratch, s)))
      return st;
  }
  { note_launch(); bg_invert_kernel<<<V0.n_chunks, kThreads, 0, s>>>(V0, B->d_cells, M.L[0].diag, M.mask, M.L[0].invd); }
  for (int l = 1; l < M.nlev; ++l) {
    const BLevel& F = M.L[l - 1];
    const BLevel& Cl = M.L[l];
    for (int c = 0; c < B->n_cells; ++c) {
      const BatchCell& fc = F.P->cells[c];
      const BatchCell& cc = Cl.P->cells[c];
      if (l == 1) {
        if ((st = gmg_level_coefs_f32(fc.g, cc.g, M.m, M.slot + fc.elem_off, M.d32 + fc.node_off, nullptr, nullptr,
                                      Cl.lam + 8 * cc.elem_off, Cl.mu + 8 * cc.elem_off, s)))
          return st;
      } else if ((st = gmg_level_coefs_f32(fc.g, cc.g, M.m, nullptr, nullptr, F.lam + 8 * fc.elem_off,
                                           F.mu + 8 * fc.elem_off, Cl.lam + 8 * cc.elem_off,
                                           Cl.mu + 8 * cc.elem_off, s))) {
        return st;
      }
      if ((st = gmg_coarse_diag_f32(cc.g, Cl.lam + 8 * cc.elem_off, Cl.mu + 8 * cc.elem_off,
                                    reinterpret_cast<float*>(scratch), Cl.diag + cc.mech_off, s)))
        return st;
    }
    const BVec Vl = mech_vec(Cl.P);
    { note_launch(); bg_invert_kernel<<<Vl.n_chunks, kThreads, 0, s>>>(Vl, Cl.P->d_cells, Cl.diag, nullptr, Cl.invd); }
  }
  for (int l = 0; l < M.nlev; ++l) {
    const BLevel& L = M.L[l];
    const BVec V = mech_vec(L.P);
    const int C = L.P->n_cells;
    if (!reuse_lmax) {
      const uint8_t* mk = l == 0 ? M.mask : nullptr;
      { note_launch(); bg_power_init_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.P->d_cells, mk, L.dvec); }
      for (int k = 0; k < power_iters; ++k) {
        if ((st = bg_level_apply(M, l, L.dvec, L.Ad, s))) return st;
        if (k == power_iters - 1) {
          { note_launch(); bg_power_dots_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.dvec, L.Ad, L.diag, mk, L.red); }
        } else {
          { note_launch(); bg_power_next_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.Ad, L.invd, L.diag, L.dvec, L.red); }
          { note_launch(); bg_power_scale_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.red, L.dvec); }
        }
      }
    }
    { note_launch(); bg_cheb_factors_kernel<<<(C + 255) / 256, 256, 0, s>>>(C, L.red, reuse_lmax ? 0 : 1, L.lmax, M.safety, L.inv_theta, L.inv_delta); }
    if ((st = last_launch_status())) return st;
  }
  return PHASTB_OK;
}

// The batched PCG of bpcg_run with the multigrid V-cycle as preconditioner (pcg_run with M):
// start r = b - A x, z = M r, rz, p = z; per iteration A p (with p.Ap), x and r, z = M r, beta,
// p = z + beta p.  Chunks of check_every iterations are captured as one graph.
int bpcg_run_pre(const phastb_batch* B, const BatchOp<float>& A, const GraphKey& op_key, const BVec& V,
                 const BPcg<float>& w, const float* b, float* x, const BpcgThr& thr, const BGmg& M0, int maxiter,
                 int check_every, const char* dot_red, int* d_count, int* h_count, cudaStream_t s) {
  int st;
  if ((st = A(x, w.Ap, thr.live, 1, false, s))) return st;
  { note_launch(); bpcg_start_pre_kernel<float><<<V.n_chunks, kThreads, 0, s>>>(V, w, b, thr.abs_sq, thr.rel, thr.outer_red, thr.outer_thr_sq, thr.live); }
  if ((st = last_launch_status())) return st;
  BGmg M = M0;
  M.guard = &w.st[0].active;
  M.gstride = kStateInts;
  if ((st = bg_precond(M, w.r, w.z, s))) return st;
  { note_launch(); bpcg_rz_kernel<float><<<V.n_chunks, kThreads, 0, s>>>(V, w, 1); }
  if ((st = last_launch_status())) return st;
  const int* guard = &w.st[0].active;
  auto iterate = [&](int k_iters) -> int {
    int e;
    for (int k = 0; k < k_iters; ++k) {
      if ((e = A(w.p, w.Ap, guard, kStateInts, true, s))) return e;
      { note_launch(); bpcg_update_pre_kernel<float><<<V.n_chunks, kThreads, 0, s>>>(V, w, x, dot_red); }
      if ((e = bg_precond(M, w.r, w.z, s))) return e;
      { note_launch(); bpcg_rz_kernel<float><<<V.n_chunks, kThreads, 0, s>>>(V, w, 0); }
      { note_launch(); bpcg_dir_kernel<float><<<V.n_chunks, kThreads, 0, s>>>(V, w); }
    }
    { note_launch(); bpcg_count_kernel<<<1, 256, 0, s>>>(B->n_cells, w.st, d_count); }
    return last_launch_status();
  };
  GraphKey key = op_key;
  key_val(key, w);
  key_val(key, x);
  key_val(key, V);
  key_val(key, check_every);
  key_val(key, dot_red);
  key_val(key, d_count);
  // the hierarchy lives in the workspace: its first array, the options and the fine inputs identify it
  key_val(key, M.nlev);
  key_val(key, M.L[0].diag);
  key_val(key, M.mask);
  key_val(key, M.d32);
  key_val(key, M.slot);
  key_val(key, M.deg);
  key_val(key, M.deg_coarse);
  key_val(key, M.safety);
  long long glaunch = 0;
  cudaGraphExec_t gexec =
      maxiter >= check_every ? graph_for(key, s, [&] { return iterate(check_every); }, &glaunch) : nullptr;
  int it = 0;
  while (it < maxiter) {
    const int chunk = std::min(check_every, maxiter - it);
    if (gexec && chunk == check_every) {
      note_launch(glaunch);
      if ((st = cuda_status(cudaGraphLaunch(gexec, s)))) return st;
    } else if ((st = iterate(chunk))) {
      return st;
    }
    it += chunk;
    if ((st = cuda_status(cudaMemcpyAsync(h_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    if (*h_count == 0) break;
  }
  return PHASTB_OK;
}

}  // namespace

}  // namespace phastb

using namespace phastb;

namespace {

bool batch_ready(const phastb_batch* B) { return B && B->bound && B->n_cells > 0; }

VoxMat<double> cell_mat64(const phastb_voxel_material& m, double ell) {
  phastb_voxel_material c = m;
  c.ell = ell;
  return make_vox_mat<double>(c);
}

// Workspace of the batched mechanics solve.
struct MechLayout {
  BPcg<double> w64;
  BPcg<float> w32;
  double *xc, *bf, *x, *r64, *d64, *thr_sq, *bb, *outer_thr_sq, *inner_abs_sq;
  float *inv32, *r32, *dx32, *d32;
  double* invd64;
  char *ared, *rred, *scratch;
  int *count, *live, *live0;
  char* gmg;  // multigrid hierarchy (bgmg_bytes), when the inner solves use the V-cycle
  size_t bytes;
};

MechLayout mech_layout(const phastb_batch* B, int mixed, char* base, bool gmg = false) {
  Carve cv{base};
  MechLayout L{};
  const size_t n = (size_t)B->n_mech, C = (size_t)B->n_cells;
  L.xc = cv.take<double>(n);
  L.bf = cv.take<double>(n);
  L.x = cv.take<double>(n);
  L.r64 = cv.take<double>(n);
  L.invd64 = cv.take<double>(n);
  L.d64 = cv.take<double>((size_t)B->n_nodes);
  L.thr_sq = cv.take<double>(C);
  L.bb = cv.take<double>(C);
  L.outer_thr_sq = cv.take<double>(C);
  L.inner_abs_sq = cv.take<double>(C);
  L.ared = cv.take<char>(n_red_ws(B));
  L.rred = cv.take<char>(n_red_ws(B));
  L.count = cv.take<int>(1);
  L.live = cv.take<int>(C);
  L.live0 = cv.take<int>(C);
  L.scratch = cv.take<char>(align_up(24 * sizeof(double) * (size_t)B->max_elem) + red_ws_bytes());
  if (!mixed) {
    L.w64.r = cv.take<double>(n);
    L.w64.z = cv.take<double>(n);
    L.w64.p = cv.take<double>(n);
    L.w64.Ap = cv.take<double>(n);
    L.w64.st = cv.take<PcgState>(C);
    L.w64.red = cv.take<char>(n_red_ws(B));
  } else {
    L.w64.Ap = cv.take<double>(n);  // FP64 actions of the refinement
    L.inv32 = cv.take<float>(n);
    L.r32 = cv.take<float>(n);
    L.dx32 = cv.take<float>(n);
    L.d32 = cv.take<float>((size_t)B->n_nodes);
    L.w32.r = cv.take<float>(n);
    L.w32.z = cv.take<float>(n);
    L.w32.p = cv.take<float>(n);
    L.w32.Ap = cv.take<float>(n);
    L.w32.st = cv.take<PcgState>(C);
    L.w32.red = cv.take<char>(n_red_ws(B));
  }
  L.gmg = gmg ? cv.take<char>(bgmg_bytes(B)) : nullptr;
  L.bytes = cv.used;
  return L;
}

// Workspace of the batched box-KKT damage solve.
struct KktLayout {
  BPcg<double> w;
  double *rhs, *diag, *invd, *known, *bf, *grad, *xd, *tol, *r0, *Hw;
  uint8_t *la, *ua, *fixed;
  int *live, *live0, *status, *iters, *sets, *kkt_ok, *running, *count;
  char *ared, *rred, *kred, *scratch;
  size_t bytes;
};

KktLayout kkt_layout(const phastb_batch* B, char* base) {
  Carve cv{base};
  KktLayout L{};
  const size_t n = (size_t)B->n_nodes, C = (size_t)B->n_cells;
  L.rhs = cv.take<double>(n);
  L.diag = cv.take<double>(n);
  L.invd = cv.take<double>(n);
  L.known = cv.take<double>(n);
  L.bf = cv.take<double>(n);
  L.grad = cv.take<double>(n);
  L.xd = cv.take<double>(n);
  L.tol = cv.take<double>(C);
  L.r0 = cv.take<double>(C);
  L.Hw = cv.take<double>(8 * (size_t)B->n_elem);
  L.la = cv.take<uint8_t>(n);
  L.ua = cv.take<uint8_t>(n);
  L.fixed = cv.take<uint8_t>(n);
  L.live = cv.take<int>(C);
  L.live0 = cv.take<int>(C);
  L.status = cv.take<int>(C);
  L.iters = cv.take<int>(C);
  L.sets = cv.take<int>(C);
  L.kkt_ok = cv.take<int>(C);
  L.running = cv.take<int>(1);
  L.count = cv.take<int>(1);
  L.ared = cv.take<char>(n_red_ws(B));
  L.rred = cv.take<char>(n_red_ws(B));
  L.kred = cv.take<char>(n_red_ws(B));
  L.scratch = cv.take<char>(align_up(24 * sizeof(double) * (size_t)B->max_elem) + red_ws_bytes());
  L.w.r = cv.take<double>(n);
  L.w.z = cv.take<double>(n);
  L.w.p = cv.take<double>(n);
  L.w.Ap = cv.take<double>(n);
  L.w.st = cv.take<PcgState>(C);
  L.w.red = cv.take<char>(n_red_ws(B));
  L.bytes = cv.used;
  return L;
}

// every per-cell reduction ticket of a set of workspaces back to zero
int reset_tickets(const phastb_batch* B, std::initializer_list<char*> reds, cudaStream_t s) {
  for (char* r : reds) {
    if (!r) continue;
    { note_launch(); b_reset_tickets_kernel<<<(B->n_cells + 255) / 256, 256, 0, s>>>(B->n_cells, r); }
  }
  return last_launch_status();
}

GraphKey mech_key(const phastb_batch* B, const void* mat, size_t mat_bytes, const void* slot, const void* d,
                  const void* mask, const void* red) {
  GraphKey k;
  key_val(k, B);
  key_add(k, mat, mat_bytes);
  key_val(k, slot);
  key_val(k, d);
  key_val(k, mask);
  key_val(k, red);
  return k;
}

}  // namespace

extern "C" {

phastb_batch* phastb_batch_create(int n_cells, const phastb_voxel_grid* grids, const double* ell,
                                  const double* dscale, int ox, int oy, int kz) {
  if (n_cells < 1 || !grids || !ell || !dscale) return nullptr;
  if (!((ox == 16 && oy == 8) || (ox == 8 && oy == 8)) || kz < 1) return nullptr;
  phastb_batch* B = new phastb_batch();
  B->n_cells = n_cells;
  B->ox = ox;
  B->oy = oy;
  B->kz = kz;
  std::vector<long long> noff, nlen, moff, mlen;
  for (int c = 0; c < n_cells; ++c) {
    if (!valid_vox(&grids[c]) || !(ell[c] > 0) || !(dscale[c] > 0)) {
      delete B;
      return nullptr;
    }
    const VoxGeom v = make_vox_geom(grids[c]);
    const long long tiles =
        (long long)((v.rx + ox - 1) / ox) * ((v.ry + oy - 1) / oy) * ((v.rz + kz - 1) / kz);
    if (tiles > kMaxPartials || ox > v.rx || oy > v.ry || kz > v.rz) {
      delete B;
      return nullptr;
    }
    BatchCell cl{};
    cl.g = v;
    cl.ts = TileShape{ox, oy, kz};
    cl.nvb = (int)tiles;
    cl.node_off = B->n_nodes;
    cl.mech_off = B->n_mech;
    cl.elem_off = B->n_elem;
    cl.ell = ell[c];
    cl.dscale = dscale[c];
    const TileArgs<float> af = tile_args<float>(v, 0);
    const TileArgs<double> ad = tile_args<double>(v, 0);
    cl.kf = af.k;
    cl.kd = ad.k;
    noff.push_back(B->n_nodes);
    nlen.push_back(v.n_red);
    moff.push_back(B->n_mech);
    mlen.push_back(3LL * v.n_red + 6);
    B->n_nodes += v.n_red;
    B->n_mech += 3LL * v.n_red + 6;
    B->n_elem += v.n_elem;
    B->max_elem = std::max<long long>(B->max_elem, v.n_elem);
    B->geom.push_back(v);
    B->cells.push_back(cl);
  }
  if (8 * B->n_elem >= (1LL << 31) || B->n_mech >= (1LL << 31)) {  // chunk bounds are 32-bit
    delete B;
    return nullptr;
  }
  // bricks of the largest cells first, so the small cells fill the tail of a launch
  std::vector<int> order(n_cells);
  for (int c = 0; c < n_cells; ++c) order[c] = c;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return B->cells[a].nvb > B->cells[b].nvb; });
  for (int c : order)
    for (int t = 0; t < B->cells[c].nvb; ++t) B->work.push_back(make_int2(c, t));
  make_chunks(noff, nlen, &B->node_chunks, &B->node_nchunk);
  make_chunks(moff, mlen, &B->mech_chunks, &B->mech_nchunk);
  size_t t = 0;
  t += align_up(sizeof(BatchCell) * B->cells.size());
  t += align_up(sizeof(int2) * B->work.size());
  t += align_up(sizeof(BChunk) * B->node_chunks.size());
  t += align_up(sizeof(BChunk) * B->mech_chunks.size());
  t += align_up(sizeof(int) * n_cells) * 2;
  B->table_bytes = t;
  // the multigrid hierarchy of the batch: rediscretised cells of twice and four times the voxel size
  bool gmg = true;
  for (int c = 0; c < n_cells && gmg; ++c) {
    const phastb_voxel_grid& g = grids[c];
    gmg = g.px && g.py && g.pz && g.nx % 4 == 0 && g.ny % 4 == 0 && g.nz % 4 == 0 && g.nx >= 32 && g.ny >= 32 &&
          g.nz >= 32;
  }
  if (gmg && ox == B->ox) {
    std::vector<phastb_voxel_grid> cg(grids, grids + n_cells);
    for (int l = 0; l < 2 && gmg; ++l) {
      for (auto& g : cg) {
        g.nx /= 2;
        g.ny /= 2;
        g.nz /= 2;
        g.hx *= 2;
        g.hy *= 2;
        g.hz *= 2;
      }
      B->lev[l] = phastb_batch_create(n_cells, cg.data(), ell, dscale, 8, 8, 4);
      gmg = B->lev[l] != nullptr;
    }
    if (gmg) {
      // a coarse plan has no levels of its own
      for (int l = 0; l < 2; ++l) {
        B->lev[l]->nlev = 1;
        delete B->lev[l]->lev[0];
        delete B->lev[l]->lev[1];
        B->lev[l]->lev[0] = B->lev[l]->lev[1] = nullptr;
      }
      B->nlev = 3;
    } else {
      delete B->lev[0];
      delete B->lev[1];
      B->lev[0] = B->lev[1] = nullptr;
    }
  }
  return B;
}

void phastb_batch_destroy(phastb_batch* B) { delete B; }

int phastb_batch_sizes(const phastb_batch* B, long long* out) {
  if (!B || !out) return PHASTB_ERR_ARG;
  out[0] = B->n_nodes;
  out[1] = B->n_mech;
  out[2] = B->n_elem;
  out[3] = (long long)B->work.size();
  out[4] = (long long)B->all_table_bytes();
  out[5] = (long long)B->mech_chunks.size();
  out[6] = (long long)B->node_chunks.size();
  for (int c = 0; c < B->n_cells; ++c) {
    const BatchCell& cl = B->cells[c];
    long long* o = out + 7 + 3 * (size_t)c;
    o[0] = cl.node_off;
    o[1] = cl.mech_off;
    o[2] = cl.elem_off;
  }
  return PHASTB_OK;
}

static int bind_level(phastb_batch* B, char* tables, cudaStream_t s) {
  Carve cv{tables};
  B->d_cells = cv.take<BatchCell>(B->cells.size());
  B->d_work = cv.take<int2>(B->work.size());
  B->d_node_chunks = cv.take<BChunk>(B->node_chunks.size());
  B->d_mech_chunks = cv.take<BChunk>(B->mech_chunks.size());
  B->d_node_nchunk = cv.take<int>(B->n_cells);
  B->d_mech_nchunk = cv.take<int>(B->n_cells);
  auto put = [&](void* dst, const void* src, size_t n) {
    return cuda_status(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s));
  };
  int st;
  if ((st = put(B->d_cells, B->cells.data(), sizeof(BatchCell) * B->cells.size()))) return st;
  if ((st = put(B->d_work, B->work.data(), sizeof(int2) * B->work.size()))) return st;
  if ((st = put(B->d_node_chunks, B->node_chunks.data(), sizeof(BChunk) * B->node_chunks.size()))) return st;
  if ((st = put(B->d_mech_chunks, B->mech_chunks.data(), sizeof(BChunk) * B->mech_chunks.size()))) return st;
  if ((st = put(B->d_node_nchunk, B->node_nchunk.data(), sizeof(int) * B->n_cells))) return st;
  if ((st = put(B->d_mech_nchunk, B->mech_nchunk.data(), sizeof(int) * B->n_cells))) return st;
  B->bound = true;
  return PHASTB_OK;
}

int phastb_batch_bind(phastb_batch* B, void* tables, size_t bytes, void* stream) {
  if (!B || !tables || bytes < B->all_table_bytes()) return PHASTB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  char* p = static_cast<char*>(tables);
  int st = bind_level(B, p, s);
  p += B->table_bytes;
  for (int l = 0; l < B->nlev - 1 && !st; ++l) {
    st = bind_level(B->lev[l], p, s);
    p += B->lev[l]->table_bytes;
  }
  if (st) return st;
  return cuda_status(cudaStreamSynchronize(s));
}

size_t phastb_batch_apply_workspace_bytes(const phastb_batch* B) { return B ? n_red_ws(B) : 0; }

int phastb_batch_mech_apply(const phastb_batch* B, const phastb_voxel_material* m, const uint8_t* slot, int dtype,
                            const void* x, const void* d, const uint8_t* mask, void* y, double* rE_out,
                            void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch_ready(B) || !valid_mat(m) || !slot || !x || !y || (dtype != PHASTB_F64 && dtype != PHASTB_F32))
    return PHASTB_ERR_ARG;
  if (!m->isotropic) return PHASTB_UNSUPPORTED;
  if (!workspace || workspace_bytes < n_red_ws(B)) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* red = static_cast<char*>(workspace);
  int st;
  if ((st = reset_tickets(B, {red}, s))) return st;
  if (dtype == PHASTB_F64)
    st = batch_mech_op<double>(B, make_vox_mat<double>(*m), slot, (const double*)d, mask, (const double*)x,
                               (double*)y, red, nullptr, 0, false, s);
  else
    st = batch_mech_op<float>(B, make_vox_mat<float>(*m), slot, (const float*)d, mask, (const float*)x, (float*)y,
                              red, nullptr, 0, false, s);
  if (st || !rE_out) return st;
  for (int c = 0; c < B->n_cells; ++c) {
    RedWs w = red_ws(red + (size_t)c * red_ws_bytes());
    if ((st = cuda_status(cudaMemcpyAsync(rE_out + 6 * (size_t)c, w.out, 6 * sizeof(double), cudaMemcpyDeviceToHost,
                                          s))))
      return st;
  }
  return cuda_status(cudaStreamSynchronize(s));
}

int phastb_batch_damage_apply(const phastb_batch* B, const phastb_voxel_material* m, const uint8_t* slot,
                              const double* d, const double* H, int scaled, const uint8_t* mask, double* y,
                              void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch_ready(B) || !valid_mat(m) || !slot || !d || !y) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < n_red_ws(B)) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* red = static_cast<char*>(workspace);
  int st;
  if ((st = reset_tickets(B, {red}, s))) return st;
  return batch_damage_op(B, make_vox_mat<double>(*m), slot, H, mask, d, y, red, nullptr, 0, false, s, scaled != 0);
}

size_t phastb_batch_mech_solve_workspace_bytes(const phastb_batch* B, int mixed) {
  if (!B || (mixed != 0 && mixed != 1)) return 0;
  return mech_layout(B, mixed, nullptr).bytes;
}

}  // extern "C"

namespace {

// Multigrid options of the batched inner solves (null: Jacobi).
struct BGmgOpts {
  int smooth_degree, coarse_degree, power_iters, reuse_lmax;
  double lmax_safety;
};

int batch_mech_solve_impl(const phastb_batch* B, const phastb_voxel_material* m, const uint8_t* slot,
                          const double* d, const uint8_t* fixed, const double* fixed_values, const double* x0,
                          double rtol, double atol, int maxiter, int check_every, int mixed, double inner_rtol,
                          int max_refine, const int* live_host, double* x_out, int* info, double* rinfo,
                          void* workspace, size_t workspace_bytes, void* stream, const BGmgOpts* go) {
  if (!batch_ready(B) || !valid_mat(m) || !slot || !d || !fixed || !fixed_values || !x_out || !info || !rinfo ||
      maxiter < 1 || check_every < 1 || !(rtol >= 0) || !(atol >= 0) || (rtol == 0 && atol == 0) ||
      (mixed != 0 && mixed != 1) || (mixed && (!(inner_rtol > 0) || max_refine < 1)))
    return PHASTB_ERR_ARG;
  if (!m->isotropic) return PHASTB_UNSUPPORTED;
  if (go && (!mixed || B->nlev < 3)) return PHASTB_UNSUPPORTED;
  MechLayout L = mech_layout(B, mixed, static_cast<char*>(workspace), go != nullptr);
  if (!workspace || workspace_bytes < L.bytes) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  const int C = B->n_cells;
  const long long n = B->n_mech;
  const BVec V = mech_vec(B);
  const VoxMat<double> m64 = make_vox_mat<double>(*m);
  int st;
  if ((st = reset_tickets(B, {L.ared, L.rred, mixed ? L.w32.red : L.w64.red}, s))) return st;
  // the captured iteration chunks read the damage field from the workspace
  if ((st = cuda_status(cudaMemcpyAsync(L.d64, d, sizeof(double) * B->n_nodes, cudaMemcpyDeviceToDevice, s))))
    return st;
  d = L.d64;
  // cells that take part (live_host[c] != 0, all when NULL); the others keep x0 in x_out
  std::vector<int> live0(C, 1);
  if (live_host)
    for (int c = 0; c < C; ++c) live0[c] = live_host[c] != 0;
  if ((st = cuda_status(cudaMemcpyAsync(L.live0, live0.data(), sizeof(int) * C, cudaMemcpyHostToDevice, s))))
    return st;
  // Jacobi diagonal of every cell (a per-cell setup pass, once per solve)
  for (int c = 0; c < C; ++c) {
    const BatchCell& cl = B->cells[c];
    if (!live0[c]) continue;
    if ((st = h8_mech_diag_t<double>(cl.g, m64, slot + cl.elem_off, nullptr, d + cl.node_off,
                                     L.invd64 + cl.mech_off, L.scratch, s)))
      return st;
  }
  { note_launch(); b_mech_setup_kernel<double><<<grid_ll(n), kThreads, 0, s>>>(n, fixed, fixed_values, x0, L.xc, x_out, L.invd64); }
  // b_f = where(free, -A xc, 0) and each cell's threshold max(rtol ||b_f||, atol)
  if ((st = batch_mech_op<double>(B, m64, slot, d, nullptr, L.xc, L.r64, L.ared, nullptr, 0, false, s))) return st;
  { note_launch(); b_rhs_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, fixed, nullptr, L.r64, L.bf, nullptr, L.rred, L.bb, L.thr_sq, rtol, atol); }
  if ((st = last_launch_status())) return st;
  int h_count = 0;
  std::vector<PcgState> hs;
  std::vector<double> bb(C);
  if (!mixed) {
    GraphKey key = mech_key(B, &m64, sizeof(m64), slot, d, fixed, L.ared);
    BatchOp<double> A = [&](const double* x, double* y, const int* guard, int gs, bool dot, cudaStream_t ss) {
      return batch_mech_op<double>(B, m64, slot, d, fixed, x, y, L.ared, guard, gs, dot, ss);
    };
    BpcgThr thr;
    thr.abs_sq = L.thr_sq;
    thr.live = L.live0;
    if ((st = cuda_status(cudaMemcpyAsync(L.x, x_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)))) return st;
    if ((st = bpcg_run<double>(B, A, key, V, L.w64, L.bf, L.invd64, L.x, thr, maxiter, check_every, PCG_FREEZE,
                               L.ared, L.count, &h_count, s)))
      return st;
    { note_launch(); b_where_kernel<<<grid_ll(n), kThreads, 0, s>>>(n, fixed, L.x, L.xc, x_out); }
    if (live_host && x0) { note_launch(); b_select_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live0, x_out, x0, x_out); }
    if ((st = last_launch_status())) return st;
    if ((st = fetch_states(B, L.w64.st, &hs, s))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(bb.data(), L.bb, sizeof(double) * C, cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    int worst = PHASTB_OK;
    for (int c = 0; c < C; ++c) {
      const PcgState& S = hs[c];
      if (!live0[c]) {
        info[2 * c] = 0;
        info[2 * c + 1] = 1;
        rinfo[2 * c] = rinfo[2 * c + 1] = 0.0;
        continue;
      }
      info[2 * c] = S.converged ? S.steps : std::min(S.iter, maxiter);
      info[2 * c + 1] = S.converged;
      rinfo[2 * c] = std::sqrt(bb[c]);
      rinfo[2 * c + 1] = std::sqrt(S.rr);
      const int cs = S.nonfinite ? PHASTB_NONFINITE : S.breakdown ? PHASTB_BREAKDOWN
                                                                  : (S.converged ? PHASTB_OK : PHASTB_NONCONVERGED);
      if (cs != PHASTB_OK && worst == PHASTB_OK) worst = cs;
    }
    return worst;
  }
  // FP32 inner PCG (FP64 dot products) under FP64 iterative refinement, per cell
  const VoxMat<float> m32 = make_vox_mat<float>(*m);
  { note_launch(); b_convert_kernel<double, float><<<grid_ll(B->n_nodes), kThreads, 0, s>>>(B->n_nodes, d, L.d32); }
  { note_launch(); b_convert_kernel<double, float><<<grid_ll(n), kThreads, 0, s>>>(n, L.invd64, L.inv32); }
  if ((st = last_launch_status())) return st;
  // outer thresholds and the inner absolute floor (0.5 thr), per cell
  std::vector<double> thr_h(C), half(C);
  if ((st = cuda_status(cudaMemcpyAsync(thr_h.data(), L.thr_sq, sizeof(double) * C, cudaMemcpyDeviceToHost, s))))
    return st;
  if ((st = cuda_status(cudaMemcpyAsync(bb.data(), L.bb, sizeof(double) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
  for (int c = 0; c < C; ++c) half[c] = 0.25 * thr_h[c];
  if ((st = cuda_status(cudaMemcpyAsync(L.outer_thr_sq, L.thr_sq, sizeof(double) * C, cudaMemcpyDeviceToDevice, s))))
    return st;
  if ((st = cuda_status(cudaMemcpyAsync(L.inner_abs_sq, half.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s))))
    return st;
  GraphKey key = mech_key(B, &m32, sizeof(m32), slot, L.d32, fixed, L.ared);
  BatchOp<float> A32 = [&](const float* x, float* y, const int* guard, int gs, bool dot, cudaStream_t ss) {
    return batch_mech_op<float>(B, m32, slot, L.d32, fixed, x, y, L.ared, guard, gs, dot, ss);
  };
  // the V-cycle hierarchy for this damage field (the FP32 moduli of every level)
  BGmg G{};
  if (go) {
    bgmg_carve(G, B, L.gmg);
    G.m = m32;
    G.slot = slot;
    G.d32 = L.d32;
    G.fixed = fixed;
    G.safety = go->lmax_safety;
    G.deg = go->smooth_degree;
    G.deg_coarse = go->coarse_degree;
    if ((st = bg_setup(G, B, L.scratch, go->power_iters, go->reuse_lmax != 0, s))) return st;
  }
  std::vector<int> iters(C, 0), done(C, 0), bad(C, 0), live(live0);
  std::vector<double> rn(C, 0.0);
  for (int k = 0; k < max_refine; ++k) {
    // cells that failed or spent their iteration budget take no further part
    if ((st = cuda_status(cudaMemcpyAsync(L.live, live.data(), sizeof(int) * C, cudaMemcpyHostToDevice, s))))
      return st;
    int budget = 1;
    for (int c = 0; c < C; ++c)
      if (live[c]) budget = std::max(budget, maxiter - iters[c]);
    // FP64 residual of every cell; each inner start checks its norm first
    if ((st = batch_mech_op<double>(B, m64, slot, d, fixed, x_out, L.w64.Ap, L.ared, nullptr, 0, false, s))) return st;
    { note_launch(); b_rhs_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, fixed, L.bf, L.w64.Ap, L.r64, L.r32, L.rred, nullptr, nullptr, 0.0, 0.0); }
    if ((st = cuda_status(cudaMemsetAsync(L.dx32, 0, sizeof(float) * n, s)))) return st;
    BpcgThr thr;
    thr.abs_sq = L.inner_abs_sq;
    thr.rel = inner_rtol;
    thr.outer_red = L.rred;
    thr.outer_thr_sq = L.outer_thr_sq;
    thr.live = L.live;
    if (G.nlev > 0) {
      if ((st = bpcg_run_pre(B, A32, key, V, L.w32, L.r32, L.dx32, thr, G, budget, 2, L.ared, L.count, &h_count, s)))
        return st;
    } else if ((st = bpcg_run<float>(B, A32, key, V, L.w32, L.r32, L.inv32, L.dx32, thr, budget, check_every,
                                     PCG_FREEZE, L.ared, L.count, &h_count, s))) {
      return st;
    }
    if ((st = fetch_states(B, L.w32.st, &hs, s))) return st;
    int n_live = 0;
    for (int c = 0; c < C; ++c) {
      const PcgState& S = hs[c];
      if (!live[c]) continue;
      live[c] = 0;
      rn[c] = std::sqrt(S.outer_rr);
      if (S.outer_done) {
        done[c] = 1;
        continue;
      }
      if (S.nonfinite || !std::isfinite(rn[c])) {
        bad[c] = PHASTB_NONFINITE;
        continue;
      }
      iters[c] += S.converged ? S.steps : std::min(S.iter, budget);
      if (S.breakdown) {
        bad[c] = PHASTB_BREAKDOWN;
        continue;
      }
      if (iters[c] >= maxiter) continue;
      live[c] = 1;
      ++n_live;
    }
    // a cell that took no part left its correction at zero
    { note_launch(); b_add_kernel<<<grid_ll(n), kThreads, 0, s>>>(n, L.dx32, x_out); }
    if ((st = last_launch_status())) return st;
    if (n_live == 0) break;
  }
  // the last corrections are not yet checked: FP64 residual norms of every cell
  if ((st = batch_mech_op<double>(B, m64, slot, d, fixed, x_out, L.w64.Ap, L.ared, nullptr, 0, false, s))) return st;
  { note_launch(); b_rhs_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, fixed, L.bf, L.w64.Ap, L.r64, nullptr, L.rred, L.bb, nullptr, 0.0, 0.0); }
  { note_launch(); b_where_kernel<<<grid_ll(n), kThreads, 0, s>>>(n, fixed, x_out, L.xc, x_out); }
  if (live_host && x0) { note_launch(); b_select_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live0, x_out, x0, x_out); }
  if ((st = last_launch_status())) return st;
  std::vector<double> rr(C);
  if ((st = cuda_status(cudaMemcpyAsync(rr.data(), L.bb, sizeof(double) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
  int worst = PHASTB_OK;
  for (int c = 0; c < C; ++c) {
    if (!live0[c]) {
      info[2 * c] = 0;
      info[2 * c + 1] = 1;
      rinfo[2 * c] = rinfo[2 * c + 1] = 0.0;
      continue;
    }
    const double r = std::sqrt(rr[c]);
    const int conv = !bad[c] && r * r <= thr_h[c];
    info[2 * c] = iters[c];
    info[2 * c + 1] = conv;
    rinfo[2 * c] = std::sqrt(bb[c]);
    rinfo[2 * c + 1] = r;
    const int cs = bad[c] ? bad[c] : (conv ? PHASTB_OK : PHASTB_NONCONVERGED);
    if (cs != PHASTB_OK && worst == PHASTB_OK) worst = cs;
  }
  return worst;
}

}  // namespace

extern "C" {

int phastb_batch_mech_solve(const phastb_batch* B, const phastb_voxel_material* m, const uint8_t* slot,
                            const double* d, const uint8_t* fixed, const double* fixed_values, const double* x0,
                            double rtol, double atol, int maxiter, int check_every, int mixed, double inner_rtol,
                            int max_refine, const int* live_host, double* x_out, int* info, double* rinfo,
                            void* workspace, size_t workspace_bytes, void* stream) {
  return batch_mech_solve_impl(B, m, slot, d, fixed, fixed_values, x0, rtol, atol, maxiter, check_every, mixed,
                               inner_rtol, max_refine, live_host, x_out, info, rinfo, workspace, workspace_bytes,
                               stream, nullptr);
}

size_t phastb_batch_mech_solve_ex_workspace_bytes(const phastb_batch* B, const phastb_mech_opts* o) {
  if (!B || !o || (o->mixed != 0 && o->mixed != 1)) return 0;
  if (o->precond && (!o->mixed || B->nlev < 3 || o->levels != 3)) return 0;
  return mech_layout(B, o->mixed, nullptr, o->precond != 0).bytes;
}

int phastb_batch_mech_solve_ex(const phastb_batch* B, const phastb_voxel_material* m, const uint8_t* slot,
                               const double* d, const uint8_t* fixed, const double* fixed_values, const double* x0,
                               double rtol, double atol, int maxiter, int check_every, const phastb_mech_opts* o,
                               int reuse_lmax, const int* live_host, double* x_out, int* info, double* rinfo,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (!o || (o->precond && (o->levels != 3 || o->smooth_degree < 1 || o->coarse_degree < 1 || o->power_iters < 1 ||
                            !(o->lmax_safety > 1.0 / 30.0))))
    return PHASTB_ERR_ARG;
  BGmgOpts go{o->smooth_degree, o->coarse_degree, o->power_iters, reuse_lmax, o->lmax_safety};
  return batch_mech_solve_impl(B, m, slot, d, fixed, fixed_values, x0, rtol, atol, maxiter, check_every, o->mixed,
                               o->inner_rtol, o->max_refine, live_host, x_out, info, rinfo, workspace,
                               workspace_bytes, stream, o->precond ? &go : nullptr);
}

size_t phastb_batch_box_kkt_workspace_bytes(const phastb_batch* B) { return B ? kkt_layout(B, nullptr).bytes : 0; }

int phastb_batch_damage_box_kkt(const phastb_batch* B, const phastb_voxel_material* m, const uint8_t* slot,
                                const double* H, const double* lower, double upper, const double* initial,
                                double lin_tol, double kkt_tol, double min_tol, int tol_rule, int max_lin,
                                int max_active, const int* live_host, double* d_out, int* info, double* rinfo,
                                void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch_ready(B) || !valid_mat(m) || !slot || !lower || !initial || !d_out || !info || max_lin < 1 ||
      max_active < 1 || !(lin_tol > 0) || !(kkt_tol >= 0) || !(min_tol >= 0))
    return PHASTB_ERR_ARG;
  KktLayout L = kkt_layout(B, static_cast<char*>(workspace));
  if (!workspace || workspace_bytes < L.bytes) return PHASTB_ERR_WORKSPACE;
  ScopedStream scope((cudaStream_t)stream);
  if (scope.status()) return scope.status();
  cudaStream_t s = scope.get();
  const int C = B->n_cells;
  const long long n = B->n_nodes;
  const BVec V = node_vec(B);
  const VoxMat<double> m64 = make_vox_mat<double>(*m);
  int st;
  if ((st = reset_tickets(B, {L.ared, L.rred, L.kred, L.w.red}, s))) return st;
  if ((st = cuda_status(cudaMemsetAsync(L.la, 0, (size_t)n, s)))) return st;
  if ((st = cuda_status(cudaMemsetAsync(L.ua, 0, (size_t)n, s)))) return st;
  for (int* a : {L.status, L.iters, L.sets, L.kkt_ok})
    if ((st = cuda_status(cudaMemsetAsync(a, 0, sizeof(int) * C, s)))) return st;
  std::vector<int> live0(C, 1);
  if (live_host)
    for (int c = 0; c < C; ++c) live0[c] = live_host[c] != 0;
  if ((st = cuda_status(cudaMemcpyAsync(L.live, live0.data(), sizeof(int) * C, cudaMemcpyHostToDevice, s)))) return st;
  if ((st = cuda_status(cudaMemcpyAsync(L.live0, live0.data(), sizeof(int) * C, cudaMemcpyHostToDevice, s)))) return st;
  // the captured iteration chunks read the history from the workspace
  if (H && (st = cuda_status(cudaMemcpyAsync(L.Hw, H, sizeof(double) * 8 * B->n_elem, cudaMemcpyDeviceToDevice, s))))
    return st;
  if (H) H = L.Hw;
  // right-hand side and Jacobi diagonal of every cell's scaled system (per-cell setup pass)
  for (int c = 0; c < C; ++c) {
    const BatchCell& cl = B->cells[c];
    if (!live0[c]) continue;
    const VoxMat<double> mc = cell_mat64(*m, cl.ell);
    const double* Hc = H ? H + 8 * cl.elem_off : nullptr;
    if ((st = h8_damage_launch(cl.g, mc, slot + cl.elem_off, 1, nullptr, Hc, cl.dscale, L.rhs + cl.node_off, nullptr,
                               L.scratch, nullptr, s)))
      return st;
    if (!H && (st = cuda_status(cudaMemsetAsync(L.rhs + cl.node_off, 0, sizeof(double) * cl.g.n_red, s)))) return st;
    if ((st = h8_damage_launch(cl.g, mc, slot + cl.elem_off, 2, nullptr, Hc, cl.dscale, L.diag + cl.node_off,
                               nullptr, L.scratch, nullptr, s)))
      return st;
  }
  // per-cell linear tolerance
  if (tol_rule) {
    if ((st = batch_damage_op(B, m64, slot, H, nullptr, initial, L.w.Ap, L.ared, nullptr, 0, false, s))) return st;
    { note_launch(); b_resid_norm_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.rhs, L.w.Ap, L.rred); }
    { note_launch(); b_lin_tol_kernel<<<1, 256, 0, s>>>(C, L.rred, lin_tol, kkt_tol, min_tol, L.tol, L.r0); }
  } else {
    std::vector<double> t(C, lin_tol), z(C, 0.0);
    if ((st = cuda_status(cudaMemcpyAsync(L.tol, t.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s)))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(L.r0, z.data(), sizeof(double) * C, cudaMemcpyHostToDevice, s)))) return st;
  }
  if ((st = last_launch_status())) return st;
  const double* cinit = initial;
  GraphKey key = mech_key(B, &m64, sizeof(m64), slot, H, L.fixed, L.ared);
  BatchOp<double> Af = [&](const double* x, double* y, const int* guard, int gs, bool dot, cudaStream_t ss) {
    return batch_damage_op(B, m64, slot, H, L.fixed, x, y, L.ared, guard, gs, dot, ss);
  };
  int h_count = 0, running = 0;
  for (int c = 0; c < C; ++c) running += live0[c];
  int ai = 0;
  for (ai = 1; ai <= max_active && running > 0; ++ai) {
    { note_launch(); b_kkt_setup_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live, L.la, L.ua, lower, upper, cinit, L.diag, L.fixed, L.known, L.xd, L.invd); }
    // b_f = where(free, rhs - A known, 0) for the live cells
    if ((st = batch_damage_op(B, m64, slot, H, nullptr, L.known, L.w.Ap, L.ared, L.live, 1, false, s))) return st;
    { note_launch(); b_kkt_rhs_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live, L.fixed, L.rhs, L.w.Ap, L.bf); }
    if ((st = last_launch_status())) return st;
    // Dirichlet PCG on each live cell's free set, tolerance relative to max(||r0||, 1)
    if ((st = Af(L.xd, L.w.Ap, L.live, 1, false, s))) return st;
    { note_launch(); bpcg_start_rel_kernel<double><<<V.n_chunks, kThreads, 0, s>>>(V, L.w, L.bf, L.invd, L.tol, L.live, PCG_STRICT); }
    if ((st = last_launch_status())) return st;
    {
      const int* guard = &L.w.st[0].active;
      auto iterate = [&](int k_iters) -> int {
        int e;
        for (int k = 0; k < k_iters; ++k) {
          if ((e = Af(L.w.p, L.w.Ap, guard, kStateInts, true, s))) return e;
          { note_launch(); bpcg_update_kernel<double><<<V.n_chunks, kThreads, 0, s>>>(V, L.w, L.xd, L.invd, PCG_STRICT, L.ared); }
          { note_launch(); bpcg_dir_kernel<double><<<V.n_chunks, kThreads, 0, s>>>(V, L.w); }
        }
        { note_launch(); bpcg_count_kernel<<<1, 256, 0, s>>>(C, L.w.st, L.count); }
        return last_launch_status();
      };
      GraphKey k2 = key;
      key_val(k2, L.w);
      key_val(k2, L.xd);
      key_val(k2, L.invd);
      key_val(k2, V);
      long long glaunch = 0;
      const int ce = 10;
      cudaGraphExec_t gexec = max_lin >= ce ? graph_for(k2, s, [&] { return iterate(ce); }, &glaunch) : nullptr;
      int it = 0;
      while (it < max_lin) {
        const int chunk = std::min(ce, max_lin - it);
        if (gexec && chunk == ce) {
          note_launch(glaunch);
          if ((st = cuda_status(cudaGraphLaunch(gexec, s)))) return st;
        } else if ((st = iterate(chunk))) {
          return st;
        }
        it += chunk;
        if ((st = cuda_status(cudaMemcpyAsync(&h_count, L.count, sizeof(int), cudaMemcpyDeviceToHost, s)))) return st;
        if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
        if (h_count == 0) break;
      }
    }
    // candidate = where(fixed, known, x); gradient, set change and audit; per-cell decision
    { note_launch(); b_kkt_where_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live, L.fixed, L.xd, L.known, L.xd); }
    if ((st = batch_damage_op(B, m64, slot, H, nullptr, L.xd, L.w.Ap, L.ared, L.live, 1, false, s))) return st;
    { note_launch(); b_kkt_update_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live, L.fixed, L.xd, L.w.Ap, L.rhs, lower, upper, kkt_tol, L.la, L.ua, L.grad, L.kred); }
    { note_launch(); b_kkt_decide_kernel<<<1, 256, 0, s>>>(C, max_lin, L.w.st, L.kred, L.live, L.status, L.iters, L.sets, L.kkt_ok, kkt_tol, L.running); }
    // the next set of a live cell starts from its candidate
    { note_launch(); b_copy_live_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live, L.xd, L.grad); }
    if ((st = last_launch_status())) return st;
    if ((st = cuda_status(cudaMemcpyAsync(&running, L.running, sizeof(int), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    cinit = L.grad;
  }
  // cells that took part return their solution, the others their initial field
  { note_launch(); b_select_kernel<<<V.n_chunks, kThreads, 0, s>>>(V, L.live0, L.xd, initial, d_out); }
  if ((st = last_launch_status())) return st;
  std::vector<int> status(C), iters(C), sets(C), ok(C);
  std::vector<double> tol(C), r0(C);
  if ((st = cuda_status(cudaMemcpyAsync(status.data(), L.status, sizeof(int) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaMemcpyAsync(iters.data(), L.iters, sizeof(int) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaMemcpyAsync(sets.data(), L.sets, sizeof(int) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaMemcpyAsync(ok.data(), L.kkt_ok, sizeof(int) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaMemcpyAsync(tol.data(), L.tol, sizeof(double) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaMemcpyAsync(r0.data(), L.r0, sizeof(double) * C, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
  int worst = PHASTB_OK;
  for (int c = 0; c < C; ++c) {
    if (!live0[c]) status[c] = 1;
    const int code = status[c] == 1 ? PHASTB_OK
                     : status[c] == 3 ? PHASTB_BREAKDOWN
                     : status[c] == 4 ? PHASTB_NONFINITE
                                      : PHASTB_NONCONVERGED;  // 0 (set budget spent) or 2
    info[4 * c] = iters[c];
    info[4 * c + 1] = sets[c];
    info[4 * c + 2] = ok[c];
    info[4 * c + 3] = code;
    if (rinfo) {
      rinfo[2 * c] = r0[c];
      rinfo[2 * c + 1] = tol[c];
    }
    if (code != PHASTB_OK && worst == PHASTB_OK) worst = code;
  }
  return worst;
}

int phastb_batch_predictor(const phastb_batch* B, const double* x, double factor, int component, double value,
                           double* x_out, double* values_out, void* stream) {
  if (!batch_ready(B) || !x || !x_out || component < 0 || component > 5) return PHASTB_ERR_ARG;
  const BVec V = mech_vec(B);
  { note_launch(); b_predictor_kernel<<<V.n_chunks, kThreads, 0, (cudaStream_t)stream>>>(V, B->d_cells, x, factor, component, value, x_out, values_out); }
  return last_launch_status();
}

size_t phastb_batch_change_workspace_bytes(const phastb_batch* B) {
  return B ? 2 * n_red_ws(B) + align_up(sizeof(double) * 5 * (size_t)B->n_cells) : 0;
}

int phastb_batch_stagger_change(const phastb_batch* B, const double* x_new, const double* x_old, const double* d_new,
                                const double* d_old, double* out_host, void* workspace, size_t workspace_bytes,
                                void* stream) {
  if (!batch_ready(B) || !x_new || !x_old || !d_new || !d_old || !out_host) return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_batch_change_workspace_bytes(B)) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* r1 = static_cast<char*>(workspace);
  char* r2 = r1 + n_red_ws(B);
  double* out = reinterpret_cast<double*>(r2 + n_red_ws(B));
  int st;
  if ((st = reset_tickets(B, {r1, r2}, s))) return st;
  const BVec Vm = mech_vec(B), Vn = node_vec(B);
  { note_launch(); b_change_mech_kernel<<<Vm.n_chunks, kThreads, 0, s>>>(Vm, B->d_cells, x_new, x_old, r1, out); }
  { note_launch(); b_change_damage_kernel<<<Vn.n_chunks, kThreads, 0, s>>>(Vn, d_new, d_old, r2, out); }
  if ((st = last_launch_status())) return st;
  if ((st = cuda_status(cudaMemcpyAsync(out_host, out, sizeof(double) * 5 * B->n_cells, cudaMemcpyDeviceToHost, s))))
    return st;
  return cuda_status(cudaStreamSynchronize(s));
}

}  // extern "C"
