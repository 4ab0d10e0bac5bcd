// Anderson mixing (type II) of the staggered damage fixed point d = G(d)
// (_AndersonAccelerator, solvers/staggered_solver.py:165-255).
//
// The history of the last depth + 1 pairs lives in one device array: rows 0..depth hold the
// residuals f = G(d) - d, rows depth+1..2 depth+1 the outputs G(d), written as a ring.  One
// kernel pushes the new pair and reduces every product of the normal equations
// (dF_i . dF_j and dF_i . f_k, dF_i = f_{i+1} - f_i, oldest first) in a fixed order; the
// small regularised system is solved on the host by Gaussian elimination with partial
// pivoting; a second kernel forms d_out - sum_i dG_i gamma_i with the two norms of the
// 1.5x safeguard, and a third clamps to [floor, 1].
#include "common.cuh"
#include "reduce.cuh"
#include <cmath>

namespace phastb {
namespace {

constexpr int kMaxDepth = 6;
constexpr int kMaxProducts = kMaxDepth * (kMaxDepth + 1) / 2 + kMaxDepth;  // 27

struct Ring {
  int rows[kMaxDepth + 1];  // history rows, oldest first
  int c;                    // entries after the push
};

size_t gram_part_bytes() { return align_up(sizeof(double) * kMaxProducts * kMaxPartials); }
size_t gram_ws_bytes() { return gram_part_bytes() + 256 + align_up(sizeof(double) * kMaxProducts); }

// Push (f, G) into row r.rows[c - 1] and reduce the products of the normal equations into out.
__global__ void __launch_bounds__(kThreads) aa_gram_kernel(int n, int depth, Ring r, double* __restrict__ hist,
                                                           const double* __restrict__ d_in,
                                                           const double* __restrict__ d_out,
                                                           double* __restrict__ part, unsigned* counter,
                                                           double* __restrict__ out) {
  const int mk = r.c - 1;
  const int K = mk * (mk + 1) / 2 + mk;
  double acc[kMaxProducts];
#pragma unroll
  for (int k = 0; k < kMaxProducts; ++k) acc[k] = 0.0;
  const size_t N = (size_t)n;
  double* F = hist;
  double* G = hist + (size_t)(depth + 1) * N;
  const int head = r.rows[r.c - 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double go = d_out[i];
    const double fk = go - d_in[i];
    F[(size_t)head * N + i] = fk;
    G[(size_t)head * N + i] = go;
    double df[kMaxDepth];
#pragma unroll
    for (int a = 0; a < kMaxDepth; ++a) {
      if (a < mk) {
        const double f1 = (a + 1 == mk) ? fk : F[(size_t)r.rows[a + 1] * N + i];
        df[a] = f1 - F[(size_t)r.rows[a] * N + i];
      } else {
        df[a] = 0.0;
      }
    }
    int k = 0;
#pragma unroll
    for (int a = 0; a < kMaxDepth; ++a)
#pragma unroll
      for (int b = a; b < kMaxDepth; ++b) {
        if (b < mk) acc[k] += df[a] * df[b];
        k += (b < mk) ? 1 : 0;
      }
#pragma unroll
    for (int a = 0; a < kMaxDepth; ++a)
      if (a < mk) acc[k + a] += df[a] * fk;
  }
  __shared__ double sh[32];
  for (int k = 0; k < K; ++k) {
    const double v = block_sum(acc[k], sh);
    if (threadIdx.x == 0) part[(size_t)k * kMaxPartials + blockIdx.x] = v;
  }
  if (arrive_last(counter)) {
    for (int k = 0; k < K; ++k) {
      const double t = fold_sum(part + (size_t)k * kMaxPartials, gridDim.x, sh);
      if (threadIdx.x == 0) out[k] = t;
    }
    if (threadIdx.x == 0) *counter = 0u;
  }
}

struct Gamma {
  double g[kMaxDepth];
};

// mix = d_out - sum_i (G_{i+1} - G_i) gamma_i; ws.out = [|mix - d_in|^2, |d_out - d_in|^2]
__global__ void __launch_bounds__(kThreads) aa_mix_kernel(int n, int depth, Ring r, Gamma gm,
                                                          const double* __restrict__ hist,
                                                          const double* __restrict__ d_in,
                                                          const double* __restrict__ d_out, double* __restrict__ mix,
                                                          RedWs ws) {
  const int mk = r.c - 1;
  const size_t N = (size_t)n;
  const double* G = hist + (size_t)(depth + 1) * N;
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < kMaxDepth; ++a)
      if (a < mk) s += (G[(size_t)r.rows[a + 1] * N + i] - G[(size_t)r.rows[a] * N + i]) * gm.g[a];
    const double v = d_out[i] - s;
    mix[i] = v;
    const double e = v - d_in[i], f = d_out[i] - d_in[i];
    acc[0] += e * e;
    acc[1] += f * f;
  }
  reduce_multi<2>(acc, ws);
}

// Projected mix: mix = clamp(d_out - sum_i (G_{i+1} - G_i) gamma_i, lower, upper);
// ws.out = [entries not finite before the clamp, entries that differ from d_out].
__global__ void __launch_bounds__(kThreads) aa_pmix_kernel(int n, int depth, Ring r, Gamma gm,
                                                           const double* __restrict__ hist,
                                                           const double* __restrict__ d_out,
                                                           const double* __restrict__ lower, double upper,
                                                           double* __restrict__ mix, RedWs ws) {
  const int mk = r.c - 1;
  const size_t N = (size_t)n;
  const double* G = hist + (size_t)(depth + 1) * N;
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < kMaxDepth; ++a)
      if (a < mk) s += (G[(size_t)r.rows[a + 1] * N + i] - G[(size_t)r.rows[a] * N + i]) * gm.g[a];
    double v = d_out[i] - s;
    if (!isfinite(v)) acc[0] += 1.0;
    v = fmin(fmax(v, lower[i]), upper);
    mix[i] = v;
    if (v != d_out[i]) acc[1] += 1.0;
  }
  reduce_multi<2>(acc, ws);
}

__global__ void aa_clamp_kernel(int n, const double* __restrict__ floor, double* __restrict__ mix) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double lo = floor ? floor[i] : 0.0;
    mix[i] = fmin(fmax(mix[i], lo), 1.0);
  }
}

// Solves A x = b (m x m, row-major) by Gaussian elimination with partial pivoting; false when a
// pivot is zero or not finite.
bool solve_small(int m, double* A, double* b, double* x) {
  for (int c = 0; c < m; ++c) {
    int p = c;
    for (int r = c + 1; r < m; ++r)
      if (std::fabs(A[r * m + c]) > std::fabs(A[p * m + c])) p = r;
    if (!(std::fabs(A[p * m + c]) > 0.0) || !std::isfinite(A[p * m + c])) return false;
    if (p != c) {
      for (int j = 0; j < m; ++j) std::swap(A[c * m + j], A[p * m + j]);
      std::swap(b[c], b[p]);
    }
    for (int r = c + 1; r < m; ++r) {
      const double f = A[r * m + c] / A[c * m + c];
      for (int j = c; j < m; ++j) A[r * m + j] -= f * A[c * m + j];
      b[r] -= f * b[c];
    }
  }
  for (int r = m - 1; r >= 0; --r) {
    double s = b[r];
    for (int j = r + 1; j < m; ++j) s -= A[r * m + j] * x[j];
    x[r] = s / A[r * m + r];
  }
  return true;
}

}  // namespace
}  // namespace phastb

using namespace phastb;

extern "C" {

size_t phastb_anderson_workspace_bytes(int depth) {
  if (depth < 1 || depth > kMaxDepth) return 0;
  return gram_ws_bytes() + red_ws_bytes();
}

int phastb_anderson_step(int n, int depth, int count, int head, double* hist, const double* d_in,
                         const double* d_out, const double* floor, double reg, double* d_mix, int* used_host,
                         void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 1 || depth < 1 || depth > kMaxDepth || count < 0 || count > depth + 1 || head < 0 || head > depth ||
      !hist || !d_in || !d_out || !d_mix || !(reg >= 0.0))
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_anderson_workspace_bytes(depth)) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* p = static_cast<char*>(workspace);
  double* part = reinterpret_cast<double*>(p);
  unsigned* counter = reinterpret_cast<unsigned*>(p + gram_part_bytes());
  double* gout = reinterpret_cast<double*>(p + gram_part_bytes() + 256);
  RedWs mw = red_ws(p + gram_ws_bytes());
  Ring r{};
  r.c = std::min(count + 1, depth + 1);
  const int R = depth + 1;
  for (int i = 0; i < r.c; ++i) r.rows[i] = ((head - (r.c - 1) + i) % R + R) % R;
  const int G = grid_for(n);
  int st;
  if ((st = cuda_status(cudaMemsetAsync(counter, 0, sizeof(unsigned), s)))) return st;
  if ((st = red_ws_reset(mw, s))) return st;
  { note_launch(); aa_gram_kernel<<<G, kThreads, 0, s>>>(n, depth, r, hist, d_in, d_out, part, counter, gout); }
  if ((st = last_launch_status())) return st;
  if (used_host) *used_host = 0;
  const int mk = r.c - 1;
  auto fallback = [&]() -> int {
    // the iterate without mixing: G(d) itself
    return cuda_status(cudaMemcpyAsync(d_mix, d_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  };
  if (mk == 0) return fallback();
  const int K = mk * (mk + 1) / 2 + mk;
  double prod[kMaxProducts];
  if ((st = cuda_status(cudaMemcpyAsync(prod, gout, sizeof(double) * K, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
  double A[kMaxDepth * kMaxDepth], b[kMaxDepth], x[kMaxDepth];
  int k = 0;
  for (int a = 0; a < mk; ++a)
    for (int c = a; c < mk; ++c) {
      A[a * mk + c] = A[c * mk + a] = prod[k];
      ++k;
    }
  for (int a = 0; a < mk; ++a) {
    b[a] = prod[k + a];
    A[a * mk + a] += reg;
  }
  if (!solve_small(mk, A, b, x)) return fallback();
  Gamma gm{};
  for (int a = 0; a < mk; ++a) gm.g[a] = x[a];
  { note_launch(); aa_mix_kernel<<<G, kThreads, 0, s>>>(n, depth, r, gm, hist, d_in, d_out, d_mix, mw); }
  if ((st = last_launch_status())) return st;
  double nrm[2];
  if ((st = red_ws_fetch(mw, nrm, 2, s))) return st;
  // safeguard: reject a mix whose residual is above 1.5x that of G(d)
  if (std::sqrt(nrm[0]) > 1.5 * std::sqrt(nrm[1])) return fallback();
  { note_launch(); aa_clamp_kernel<<<G, kThreads, 0, s>>>(n, floor, d_mix); }
  if ((st = last_launch_status())) return st;
  if (used_host) *used_host = 1;
  return PHASTB_OK;
}

int phastb_anderson_projected(int n, int depth, int count, int head, double* hist, const double* d_in,
                              const double* d_out, int want_mix, const double* lower, double upper, double reg,
                              double* d_mix, int* status_host, void* workspace, size_t workspace_bytes,
                              void* stream) {
  if (n < 1 || depth < 1 || depth > kMaxDepth || count < 0 || count > depth + 1 || head < 0 || head > depth ||
      !hist || !d_in || !d_out || !status_host || !(reg >= 0.0) || (want_mix && (!lower || !d_mix)))
    return PHASTB_ERR_ARG;
  if (!workspace || workspace_bytes < phastb_anderson_workspace_bytes(depth)) return PHASTB_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* p = static_cast<char*>(workspace);
  double* part = reinterpret_cast<double*>(p);
  unsigned* counter = reinterpret_cast<unsigned*>(p + gram_part_bytes());
  double* gout = reinterpret_cast<double*>(p + gram_part_bytes() + 256);
  RedWs mw = red_ws(p + gram_ws_bytes());
  Ring r{};
  r.c = std::min(count + 1, depth + 1);
  const int R = depth + 1;
  for (int i = 0; i < r.c; ++i) r.rows[i] = ((head - (r.c - 1) + i) % R + R) % R;
  *status_host = 0;
  int st;
  if ((st = cuda_status(cudaMemsetAsync(counter, 0, sizeof(unsigned), s)))) return st;
  if ((st = red_ws_reset(mw, s))) return st;
  const int G = grid_for(n);
  // the push, with the products of the normal equations when a mix is wanted
  Ring rp = r;
  if (!want_mix || r.c < 2) {
    rp.c = 1;
    rp.rows[0] = r.rows[r.c - 1];  // the new pair's row, no products
  }
  { note_launch(); aa_gram_kernel<<<G, kThreads, 0, s>>>(n, depth, rp, hist, d_in, d_out, part, counter, gout); }
  if ((st = last_launch_status())) return st;
  if (!want_mix || r.c < 2) return cuda_status(cudaStreamSynchronize(s));
  const int mk = r.c - 1;
  const int K = mk * (mk + 1) / 2 + mk;
  double prod[kMaxProducts];
  if ((st = cuda_status(cudaMemcpyAsync(prod, gout, sizeof(double) * K, cudaMemcpyDeviceToHost, s)))) return st;
  if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
  // unit-norm columns of dF (zero columns dropped), relative regularisation on the normal equations
  double P[kMaxDepth][kMaxDepth], pf[kMaxDepth], sc[kMaxDepth];
  int k = 0;
  for (int a = 0; a < mk; ++a)
    for (int c = a; c < mk; ++c) {
      P[a][c] = P[c][a] = prod[k];
      ++k;
    }
  for (int a = 0; a < mk; ++a) pf[a] = prod[k + a];
  int keep[kMaxDepth], nk = 0;
  for (int a = 0; a < mk; ++a) {
    sc[a] = std::sqrt(std::max(P[a][a], 0.0));
    if (sc[a] > 0.0) keep[nk++] = a;
  }
  if (nk == 0) return PHASTB_OK;
  double A[kMaxDepth * kMaxDepth], b[kMaxDepth], x[kMaxDepth];
  for (int i = 0; i < nk; ++i) {
    for (int j = 0; j < nk; ++j) A[i * nk + j] = P[keep[i]][keep[j]] / (sc[keep[i]] * sc[keep[j]]);
    A[i * nk + i] += reg;
    b[i] = pf[keep[i]] / sc[keep[i]];
  }
  if (!solve_small(nk, A, b, x)) return PHASTB_OK;
  Gamma gm{};
  for (int i = 0; i < nk; ++i) gm.g[keep[i]] = x[i] / sc[keep[i]];
  { note_launch(); aa_pmix_kernel<<<G, kThreads, 0, s>>>(n, depth, r, gm, hist, d_out, lower, upper, d_mix, mw); }
  if ((st = last_launch_status())) return st;
  double cnt[2];
  if ((st = red_ws_fetch(mw, cnt, 2, s))) return st;
  if (cnt[0] > 0.0) return PHASTB_OK;  // a non-finite mix is no mix
  *status_host = cnt[1] > 0.0 ? 1 : 2;
  return PHASTB_OK;
}

}  // extern "C"
