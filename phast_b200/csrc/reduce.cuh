// Deterministic multi-quantity reductions over a caller workspace.
#pragma once
#include "common.cuh"

namespace phastb {

constexpr int kRedMaxK = 16;

__host__ __device__ inline size_t align_up(size_t b, size_t a = 256) { return (b + a - 1) / a * a; }

struct RedWs {
  double* part;       // kRedMaxK * kMaxPartials
  unsigned* counter;  // ticket
  double* out;        // kRedMaxK results
};

__host__ __device__ inline size_t red_ws_bytes() {
  return align_up(sizeof(double) * kRedMaxK * kMaxPartials) + 256 + align_up(sizeof(double) * kRedMaxK);
}

__host__ __device__ inline RedWs red_ws(void* base) {
  char* p = static_cast<char*>(base);
  RedWs w;
  w.part = reinterpret_cast<double*>(p);
  p += align_up(sizeof(double) * kRedMaxK * kMaxPartials);
  w.counter = reinterpret_cast<unsigned*>(p);
  p += 256;
  w.out = reinterpret_cast<double*>(p);
  return w;
}

inline int red_ws_reset(const RedWs& w, cudaStream_t s) {
  return cuda_status(cudaMemsetAsync(w.counter, 0, sizeof(unsigned), s));
}

inline int red_ws_fetch(const RedWs& w, double* host, int k, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(host, w.out, sizeof(double) * k, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return PHASTB_ERR_CUDA;
  return cuda_status(cudaStreamSynchronize(s));
}

// Block-reduce K sums, publish partials, the last block folds them into out[]
// and resets the ticket so the workspace can be reused by the next launch.
template <int K>
__device__ __forceinline__ void reduce_multi(double (&v)[K], RedWs ws) {
  __shared__ double sh[32 * K];
  block_sum_multi<K>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) ws.part[k * kMaxPartials + blockIdx.x] = v[k];
  }
  if (arrive_last(ws.counter)) {
    double t[K];
    fold_sum_multi<K>(ws.part, kMaxPartials, gridDim.x, t, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) ws.out[k] = t[k];
      *ws.counter = 0u;
    }
  }
}

}  // namespace phastb
