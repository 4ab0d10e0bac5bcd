// Library-level entry points: version and the kernel-launch counter.
#include <atomic>

#include "common.cuh"

namespace phastb {
static std::atomic<long long> g_launches{0};
static thread_local long long t_launches = 0;  // this host thread's launches (graph capture counts)
void note_launch(long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
long long thread_launch_count() { return t_launches; }

namespace {
struct DevStreams {
  cudaStream_t s = nullptr;
  cudaEvent_t in = nullptr, out = nullptr;
};
constexpr int kMaxDev = 64;
thread_local DevStreams t_streams[kMaxDev];
}  // namespace

ScopedStream::ScopedStream(cudaStream_t caller) : caller_(caller) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
    st_ = PHASTB_ERR_CUDA;
    s_ = caller;
    return;
  }
  DevStreams& d = t_streams[dev];
  if (!d.s) {
    if (cudaStreamCreateWithFlags(&d.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&d.in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&d.out, cudaEventDisableTiming) != cudaSuccess) {
      st_ = PHASTB_ERR_CUDA;
      s_ = caller;
      d.s = nullptr;
      return;
    }
  }
  s_ = d.s;
  out_ = d.out;
  if (cudaEventRecord(d.in, caller) != cudaSuccess || cudaStreamWaitEvent(s_, d.in, 0) != cudaSuccess)
    st_ = PHASTB_ERR_CUDA;
}

ScopedStream::~ScopedStream() {
  if (s_ != caller_ && out_) {
    cudaEventRecord(out_, s_);
    cudaStreamWaitEvent(caller_, out_, 0);
  }
}
}  // namespace phastb

extern "C" {

const char* phastb_version(void) { return "phastb 0.1 sm_100a"; }

long long phastb_launch_count(void) { return phastb::g_launches.load(std::memory_order_relaxed); }

void phastb_launch_count_reset(void) { phastb::g_launches.store(0, std::memory_order_relaxed); }

}  // extern "C"
