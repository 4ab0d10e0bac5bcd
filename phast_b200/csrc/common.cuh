// Shared device helpers for the phase-field kernels (sm_100a).
//
// Reductions are deterministic: every reducing kernel writes one partial per
// block, and the last block to finish (ticket counter) folds the partials in
// a fixed order.  Grid sizes depend only on the problem size, so the same
// inputs always give the same bits.  No floating-point atomics are used.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include "../../include/phastb.h"

namespace phastb {

constexpr int kThreads = 256;        // block size of every vector/reduction kernel
constexpr int kMaxBlocks = 148 * 8;  // 8 resident blocks per SM on 148 SMs
constexpr int kMaxPartials = kMaxBlocks;

inline int grid_for(long long n, int threads = kThreads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > kMaxBlocks) b = kMaxBlocks;
  return static_cast<int>(b);
}

inline int grid_full(long long n, int threads = kThreads) {
  long long b = (n + threads - 1) / threads;
  return static_cast<int>(b < 1 ? 1 : b);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ int warp_or(int v) {
  return __any_sync(0xffffffffu, v) ? 1 : 0;
}

// Sum over a block of kThreads threads; result valid in every thread.
// `sh` must hold kThreads/32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = (l < (blockDim.x >> 5)) ? sh[l] : 0.0;
  t = warp_sum(t);
  return t;
}

__device__ __forceinline__ double block_min(double v, double* sh) {
  v = warp_min(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = (l < (blockDim.x >> 5)) ? sh[l] : INFINITY;
  t = warp_min(t);
  return t;
}

__device__ __forceinline__ double block_max(double v, double* sh) { return -block_min(-v, sh); }

__device__ __forceinline__ int block_or(int v, int* sh) {
  v = warp_or(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  int t = (l < (blockDim.x >> 5)) ? sh[l] : 0;
  return warp_or(t);
}

// Returns true in every thread of the last block to arrive.  The caller has
// already written its per-block partials; the fence publishes them.
__device__ __forceinline__ bool arrive_last(unsigned int* counter) {
  __shared__ unsigned int s_ticket;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_ticket = atomicAdd(counter, 1u);
  __syncthreads();
  const bool last = (s_ticket == gridDim.x - 1);
  if (last) __threadfence();
  return last;
}

// arrive_last for a group of `count` blocks sharing one ticket (the blocks of
// one cell in a batched launch).
__device__ __forceinline__ bool arrive_last_n(unsigned int* counter, int count) {
  __shared__ unsigned int s_ticket_n;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_ticket_n = atomicAdd(counter, 1u);
  __syncthreads();
  const bool last = (s_ticket_n == (unsigned)count - 1u);
  if (last) __threadfence();
  return last;
}

// Fold `n` partials (global) in a fixed order inside the last block.
__device__ __forceinline__ double fold_sum(const double* part, int n, double* sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += __ldcg(part + i);
  return block_sum(v, sh);
}

// K block sums at once: for each value the same summation tree as block_sum
// (so the same bits), with two barriers in all instead of two per value.
// `sh` must hold 32 * K doubles; every thread receives the K sums.
template <int K>
__device__ __forceinline__ void block_sum_multi(double (&v)[K], double* sh) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (l == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh[32 * k + w] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum((l < (blockDim.x >> 5)) ? sh[32 * k + l] : 0.0);
}

// K folds of `n` partials each (value k at part + k * stride) in one pass: the
// loads of all K are in flight together; per value the order of fold_sum.
template <int K>
__device__ __forceinline__ void fold_sum_multi(const double* part, int stride, int n, double (&out)[K], double* sh) {
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] += __ldcg(part + (size_t)k * stride + i);
  }
  block_sum_multi<K>(out, sh);
}

__device__ __forceinline__ double fold_min(const double* part, int n, double* sh) {
  double v = INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v = fmin(v, __ldcg(part + i));
  return block_min(v, sh);
}

__device__ __forceinline__ double fold_max(const double* part, int n, double* sh) {
  double v = -INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v = fmax(v, __ldcg(part + i));
  return block_max(v, sh);
}

__device__ __forceinline__ int fold_or(const int* part, int n, int* sh) {
  int v = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v |= __ldcg(part + i);
  return block_or(v, sh);
}

template <typename T> __device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// Host-side count of kernel launches issued by this library (every launch site
// is wrapped as `{ note_launch(); kernel<<<...>>>(...); }`).
void note_launch(long long n = 1);
long long launch_count();
long long thread_launch_count();

// Solver entry points run on a library-owned non-blocking stream (one per device
// and host thread), ordered after the caller's stream on entry and before it on
// exit.  Iteration chunks can then be captured in CUDA graphs, which the legacy
// default stream does not allow.
class ScopedStream {
 public:
  explicit ScopedStream(cudaStream_t caller);
  ~ScopedStream();
  cudaStream_t get() const { return s_; }
  int status() const { return st_; }

 private:
  cudaStream_t caller_ = nullptr, s_ = nullptr;
  cudaEvent_t out_ = nullptr;
  int st_ = 0;
};

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? PHASTB_OK : PHASTB_ERR_CUDA; }

inline int last_launch_status() { return cuda_status(cudaGetLastError()); }

}  // namespace phastb
