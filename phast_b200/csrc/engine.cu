// Device-resident Krylov engines (see engine.cuh).
#include "engine.cuh"

#include <cmath>
#include <cstdlib>
#include <list>

namespace phastb {

// ================================================================= graph cache

namespace {
struct GraphEntry {
  int dev;
  GraphKey key;
  cudaGraphExec_t exec;
  long long launches;
};
constexpr size_t kGraphCacheSize = 48;
thread_local std::list<GraphEntry> t_graph_cache;
}  // namespace

cudaGraphExec_t graph_for(const GraphKey& key, cudaStream_t s, const std::function<int()>& body, long long* count) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  for (auto it = t_graph_cache.begin(); it != t_graph_cache.end(); ++it) {
    if (it->dev == dev && it->key == key) {
      t_graph_cache.splice(t_graph_cache.begin(), t_graph_cache, it);
      *count = t_graph_cache.front().launches;
      return t_graph_cache.front().exec;
    }
  }
  const long long c0 = thread_launch_count();
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const int st = body();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  const long long n = thread_launch_count() - c0;
  note_launch(-n);  // captured, not executed
  if (st != PHASTB_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return nullptr;
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0ULL);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess || !exec) {
    cudaGetLastError();
    return nullptr;
  }
  t_graph_cache.push_front(GraphEntry{dev, key, exec, n});
  while (t_graph_cache.size() > kGraphCacheSize) {
    cudaGraphExecDestroy(t_graph_cache.back().exec);
    t_graph_cache.pop_back();
  }
  *count = n;
  return exec;
}

__global__ void while_cond_kernel(cudaGraphConditionalHandle h, const int* __restrict__ active, int* trips,
                                  const int* __restrict__ max_trips) {
  const int t = ++(*trips);
  cudaGraphSetConditional(h, (*active && t < *max_trips) ? 1u : 0u);
}

cudaGraphExec_t while_graph_for(const GraphKey& key0, cudaStream_t s, const std::function<int()>& body,
                                const int* active, int* trips, const int* max_trips, long long* count) {
  GraphKey key = key0;
  const char tag[] = "while";
  key_add(key, tag, sizeof(tag));
  key_val(key, active);
  key_val(key, trips);
  key_val(key, max_trips);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  for (auto it = t_graph_cache.begin(); it != t_graph_cache.end(); ++it) {
    if (it->dev == dev && it->key == key) {
      t_graph_cache.splice(t_graph_cache.begin(), t_graph_cache, it);
      *count = t_graph_cache.front().launches;
      return t_graph_cache.front().exec;
    }
  }
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  auto fail = [&]() -> cudaGraphExec_t {
    cudaGraphDestroy(g);
    cudaGetLastError();
    return nullptr;
  };
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) return fail();
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, nullptr, 0, &p) != cudaSuccess) return fail();
  cudaGraph_t bodyg = p.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess)
    return fail();
  const long long c0 = thread_launch_count();
  int st = body();
  { note_launch(); while_cond_kernel<<<1, 1, 0, s>>>(h, active, trips, max_trips); }
  if (!st) st = last_launch_status();
  cudaGraph_t captured = bodyg;
  const cudaError_t e = cudaStreamEndCapture(s, &captured);
  const long long n = thread_launch_count() - c0;
  note_launch(-n);  // captured, not executed
  if (st != PHASTB_OK || e != cudaSuccess) return fail();
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0ULL);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess || !exec) {
    cudaGetLastError();
    return nullptr;
  }
  t_graph_cache.push_front(GraphEntry{dev, key, exec, n});
  while (t_graph_cache.size() > kGraphCacheSize) {
    cudaGraphExecDestroy(t_graph_cache.back().exec);
    t_graph_cache.pop_back();
  }
  *count = n;
  return exec;
}

// PHASTB_DEVICE_LOOP=1 runs each Krylov solve as one conditional-WHILE graph
// (one host synchronisation per solve).  Measured on the 64^3 cell it is not
// faster than the chunked loop with a host check per chunk (the default).
static bool device_loop_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PHASTB_DEVICE_LOOP");
    return e && e[0] == '1';
  }();
  return on;
}

static int launch_graph(cudaGraphExec_t g, long long count, cudaStream_t s) {
  note_launch(count);
  return cuda_status(cudaGraphLaunch(g, s));
}

// ======================================================================= PPCG

size_t ppcg_ws_bytes(int n) {
  const size_t v = align_up(sizeof(double) * (size_t)n);
  return 8 * v + align_up((size_t)n) + align_up(sizeof(double) * 4 * kMaxPartials) +
         align_up(sizeof(int) * kMaxPartials) + 256 + align_up(sizeof(PpcgState));
}

PpcgWs ppcg_ws(void* base, int n) {
  char* p = static_cast<char*>(base);
  const size_t v = align_up(sizeof(double) * (size_t)n);
  PpcgWs w;
  double** vecs[8] = {&w.r, &w.z, &w.p, &w.Ap, &w.Ad, &w.lb, &w.minv, &w.b};
  for (auto pp : vecs) {
    *pp = reinterpret_cast<double*>(p);
    p += v;
  }
  w.act = reinterpret_cast<uint8_t*>(p);
  p += align_up((size_t)n);
  w.part = reinterpret_cast<double*>(p);
  p += align_up(sizeof(double) * 4 * kMaxPartials);
  w.ipart = reinterpret_cast<int*>(p);
  p += align_up(sizeof(int) * kMaxPartials);
  w.counter = reinterpret_cast<unsigned*>(p);
  p += 256;
  w.st = reinterpret_cast<PpcgState*>(p);
  return w;
}

__device__ __forceinline__ bool ppcg_mask(double d, double lb, double r, bool fixed) {
  const double atol = 1e-14;  // bound_atol (damage_solver.py:3559)
  return ((d <= lb + atol) && (r < 0.0)) || ((d >= 1.0 - atol) && (r > 0.0)) || fixed;
}

__global__ void ppcg_setup_kernel(int n, const double* __restrict__ d_prev, const double* __restrict__ d_init,
                                  const uint8_t* __restrict__ fixed, const double* __restrict__ vals,
                                  double* __restrict__ d, double* __restrict__ lb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double dp = d_prev[i];
    double di = d_init ? d_init[i] : dp;
    if (fixed && fixed[i]) dp = di = vals[i];
    d[i] = di;
    lb[i] = dp;
  }
}

__global__ void __launch_bounds__(kThreads) ppcg_init_kernel(int n, PpcgWs w, const double* __restrict__ d,
                                                             const uint8_t* __restrict__ fixed, double tol,
                                                             int max_iter, int check_every) {
  __shared__ double sh[96];
  double rr = 0, bb = 0, rz = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool fx = fixed && fixed[i];
    const double bi = w.b[i];
    double r = bi - w.Ad[i];
    if (fx) r = 0.0;
    w.r[i] = r;
    double mi = w.minv[i];
    if (fx) {
      mi = 0.0;
      w.minv[i] = 0.0;
    }
    const bool a = ppcg_mask(d[i], w.lb[i], r, fx);
    const double rf = a ? 0.0 : r;
    double z = rf * mi;
    if (a) z = 0.0;
    w.z[i] = z;
    w.p[i] = z;
    w.act[i] = a;
    rr += r * r;
    bb += bi * bi;
    rz += rf * z;
  }
  double v3[3] = {rr, bb, rz};
  block_sum_multi<3>(v3, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) w.part[k * kMaxPartials + blockIdx.x] = v3[k];
  }
  if (arrive_last(w.counter)) {
    double f3[3];
    fold_sum_multi<3>(w.part, kMaxPartials, gridDim.x, f3, sh);
    const double RR = f3[0], BB = f3[1], RZ = f3[2];
    if (threadIdx.x == 0) {
      PpcgState& st = *w.st;
      st.r0sq = RR;
      double ref = fmax(fmax(sqrt(BB), sqrt(RR)), 1e-30);
      st.tol_sq = (tol * ref) * (tol * ref);
      st.rz = RZ;
      st.alpha = st.beta = 0.0;
      st.max_iter = max_iter;
      st.check_every = check_every;
      st.iter = 0;
      st.last_iter = max_iter;
      st.reason = 1;
      st.branch = 0;
      st.reset_dir = 0;
      st.go_resid = 0;
      st.done = max_iter <= 0;
      st.go = max_iter > 0;
      *w.counter = 0u;
    }
  }
}

__global__ void __launch_bounds__(kThreads) ppcg_dir_stats_kernel(int n, PpcgWs w, const double* __restrict__ d) {
  if (!w.st->go) return;
  __shared__ double sh[96];
  double pap = 0, up = INFINITY, dn = INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double p = w.p[i];
    pap += p * w.Ap[i];
    if (p > 0.0) up = fmin(up, (1.0 - d[i]) / p);
    if (p < 0.0) dn = fmin(dn, (w.lb[i] - d[i]) / p);
  }
  double s = block_sum(pap, sh);
  if (threadIdx.x == 0) w.part[blockIdx.x] = s;
  s = block_min(up, sh);
  if (threadIdx.x == 0) w.part[kMaxPartials + blockIdx.x] = s;
  s = block_min(dn, sh);
  if (threadIdx.x == 0) w.part[2 * kMaxPartials + blockIdx.x] = s;
  if (arrive_last(w.counter)) {
    const double PAP = fold_sum(w.part, gridDim.x, sh);
    const double UP = fold_min(w.part + kMaxPartials, gridDim.x, sh);
    const double DN = fold_min(w.part + 2 * kMaxPartials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      PpcgState& st = *w.st;
      st.iter += 1;
      const int it = st.iter;
      if (PAP <= 0.0) {  // degenerate direction: the reference breaks out
        st.done = 1;
        st.reason = 2;
        st.last_iter = it;
        st.go = 0;
        st.go_resid = 0;
      } else {
        const double acg = st.rz / (PAP + 1e-30);
        double amax = acg;
        if (UP < amax) amax = UP;
        if (DN < amax) amax = DN;
        if (amax < acg && amax >= 0.0) {
          st.branch = 1;
          st.alpha = amax;
        } else {
          st.branch = 0;
          st.alpha = acg;
        }
        st.go_resid = (st.branch == 1) || (it % st.check_every == 0);
      }
      *w.counter = 0u;
    }
  }
}

__global__ void ppcg_update_kernel(int n, PpcgWs w, double* __restrict__ d) {
  if (!w.st->go) return;
  const double a = w.st->alpha;
  const bool restart = w.st->branch == 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double dn = d[i] + a * w.p[i];
    if (restart) {
      dn = fmin(fmax(dn, w.lb[i]), 1.0);
    } else {
      w.r[i] = w.r[i] - a * w.Ap[i];
    }
    d[i] = dn;
  }
}

__global__ void __launch_bounds__(kThreads) ppcg_resid_kernel(int n, PpcgWs w, const double* __restrict__ d,
                                                              const uint8_t* __restrict__ fixed) {
  if (!w.st->go) return;
  __shared__ double sh[96];
  __shared__ int ish[32];
  const bool need = w.st->go_resid != 0;
  double rfsq = 0, rzn = 0;
  int chg = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double r = w.r[i];
    bool a = w.act[i];
    if (need) {
      const bool fx = fixed && fixed[i];
      r = w.b[i] - w.Ad[i];
      if (fx) r = 0.0;
      w.r[i] = r;
      const bool an = ppcg_mask(d[i], w.lb[i], r, fx);
      chg |= (an != a);
      a = an;
      w.act[i] = an;
    }
    const double rf = a ? 0.0 : r;
    double z = rf * w.minv[i];
    if (a) z = 0.0;
    w.z[i] = z;
    rfsq += rf * rf;
    rzn += rf * z;
  }
  double v2[2] = {rfsq, rzn};
  block_sum_multi<2>(v2, sh);
  if (threadIdx.x == 0) {
    w.part[blockIdx.x] = v2[0];
    w.part[kMaxPartials + blockIdx.x] = v2[1];
  }
  const int c = block_or(chg, ish);
  if (threadIdx.x == 0) w.ipart[blockIdx.x] = c;
  if (arrive_last(w.counter)) {
    double f2[2];
    fold_sum_multi<2>(w.part, kMaxPartials, gridDim.x, f2, sh);
    const double RF = f2[0], RZ = f2[1];
    const int CH = fold_or(w.ipart, gridDim.x, ish);
    if (threadIdx.x == 0) {
      PpcgState& st = *w.st;
      const int it = st.iter;
      int done = 0;
      if (need) {
        if (RF < st.tol_sq) {
          done = 1;
          st.reason = 0;
          st.last_iter = it;
        } else if (RF > 1e12 * fmax(st.r0sq, 1e-30)) {
          done = 1;
          st.reason = 3;
          st.last_iter = it;
        }
      }
      if (!done) {
        const int reset = (st.branch == 1) || CH;
        st.reset_dir = reset;
        if (!reset) st.beta = RZ / (st.rz + 1e-30);
        st.rz = RZ;
        if (it >= st.max_iter) {
          done = 1;
          st.reason = 1;
          st.last_iter = st.max_iter;
        }
      }
      if (done) {
        st.done = 1;
        st.go = 0;
      }
      st.go_resid = 0;
      *w.counter = 0u;
    }
  }
}

__global__ void ppcg_dir_kernel(int n, PpcgWs w) {
  if (!w.st->go) return;
  const bool reset = w.st->reset_dir != 0;
  const double beta = w.st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double z = w.z[i];
    double pn = reset ? z : beta * w.p[i] + z;
    if (w.act[i]) pn = 0.0;
    w.p[i] = pn;
  }
}

__global__ void ppcg_finish_kernel(int n, double* __restrict__ d, const double* __restrict__ lb,
                                   const uint8_t* __restrict__ fixed, const double* __restrict__ vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double dn = fmin(fmax(d[i], lb[i]), 1.0);
    if (fixed && fixed[i]) dn = vals[i];
    d[i] = dn;
  }
}

int ppcg_solve(const LinOp<double>& A, int n, const PpcgWs& w, const double* d_prev, const double* d_init,
               const uint8_t* fixed, const double* vals, double tol, int max_iter, int check_every, double* d,
               int* info, cudaStream_t s) {
  if (check_every < 1) return PHASTB_ERR_ARG;
  const int G = grid_for(n);
  int st;
  if ((st = cuda_status(cudaMemsetAsync(w.counter, 0, sizeof(unsigned), s)))) return st;
  { note_launch(); ppcg_setup_kernel<<<G, kThreads, 0, s>>>(n, d_prev, d_init, fixed, vals, d, w.lb); }
  if ((st = last_launch_status())) return st;
  if ((st = A(d, w.Ad, nullptr, s))) return st;
  { note_launch(); ppcg_init_kernel<<<G, kThreads, 0, s>>>(n, w, d, fixed, tol, max_iter, check_every); }
  if ((st = last_launch_status())) return st;
  PpcgState hs{};
  int it = 0;
  const int* go = &w.st->go;
  const int* go_resid = &w.st->go_resid;
  auto iterate = [&](int k_iters) -> int {
    int e;
    for (int k = 0; k < k_iters; ++k) {
      if ((e = A(w.p, w.Ap, go, s))) return e;
      { note_launch(); ppcg_dir_stats_kernel<<<G, kThreads, 0, s>>>(n, w, d); }
      { note_launch(); ppcg_update_kernel<<<G, kThreads, 0, s>>>(n, w, d); }
      if ((e = A(d, w.Ad, go_resid, s))) return e;
      { note_launch(); ppcg_resid_kernel<<<G, kThreads, 0, s>>>(n, w, d, fixed); }
      { note_launch(); ppcg_dir_kernel<<<G, kThreads, 0, s>>>(n, w); }
    }
    return last_launch_status();
  };
  GraphKey key;
  key_val(key, A.apply);
  key_add(key, A.ctx, A.ctx_bytes);
  key_val(key, w);
  key_val(key, d);
  key_val(key, fixed);
  key_val(key, n);
  key_val(key, check_every);
  long long glaunch = 0;
  cudaGraphExec_t gexec =
      max_iter >= check_every ? graph_for(key, s, [&] { return iterate(check_every); }, &glaunch) : nullptr;
  while (it < max_iter) {
    const int chunk = std::min(check_every, max_iter - it);
    if (gexec && chunk == check_every) {
      if ((st = launch_graph(gexec, glaunch, s))) return st;
    } else if ((st = iterate(chunk))) {
      return st;
    }
    it += chunk;
    if ((st = cuda_status(cudaMemcpyAsync(&hs, w.st, sizeof(hs), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    if (hs.done) break;
  }
  if (max_iter <= 0) {
    if ((st = cuda_status(cudaMemcpyAsync(&hs, w.st, sizeof(hs), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
  }
  { note_launch(); ppcg_finish_kernel<<<G, kThreads, 0, s>>>(n, d, w.lb, fixed, vals); }
  if ((st = last_launch_status())) return st;
  if (info) {
    info[0] = hs.done ? hs.last_iter : max_iter;
    info[1] = hs.done ? hs.reason : 1;
  }
  return PHASTB_OK;
}

// ======================================================================== PCG

template <typename T>
size_t pcg_ws_bytes(int n) {
  const size_t v = align_up(sizeof(T) * (size_t)n);
  return 4 * v + align_up(sizeof(double) * 4 * kMaxPartials) + 256 + align_up(sizeof(PcgState));
}

template <typename T>
PcgWs<T> pcg_ws(void* base, int n) {
  char* p = static_cast<char*>(base);
  const size_t v = align_up(sizeof(T) * (size_t)n);
  PcgWs<T> w;
  w.r = reinterpret_cast<T*>(p);
  p += v;
  w.z = reinterpret_cast<T*>(p);
  p += v;
  w.p = reinterpret_cast<T*>(p);
  p += v;
  w.Ap = reinterpret_cast<T*>(p);
  p += v;
  w.part = reinterpret_cast<double*>(p);
  p += align_up(sizeof(double) * 4 * kMaxPartials);
  w.counter = reinterpret_cast<unsigned*>(p);
  p += 256;
  w.st = reinterpret_cast<PcgState*>(p);
  return w;
}

// r = b - Ax (Ax already in w.Ap); Jacobi/identity z; p = z; rz, rr.
template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_start_kernel(int n, PcgWs<T> w, const T* __restrict__ b,
                                                             const T* __restrict__ inv_diag, int custom_pre,
                                                             double thr_sq, int mode, double thr_rel,
                                                             double rel_floor, const double* outer_rr,
                                                             double outer_thr_sq, int max_trips) {
  __shared__ double sh[96];
  double rz = 0, rr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T r = b[i] - w.Ap[i];
    w.r[i] = r;
    rr += double(r) * double(r);
    if (!custom_pre) {
      const T z = inv_diag ? r * inv_diag[i] : r;
      w.z[i] = z;
      w.p[i] = z;
      rz += double(r) * double(z);
    }
  }
  double v2[2] = {rz, rr};
  block_sum_multi<2>(v2, sh);
  if (threadIdx.x == 0) {
    w.part[blockIdx.x] = v2[0];
    w.part[kMaxPartials + blockIdx.x] = v2[1];
  }
  if (arrive_last(w.counter)) {
    double f2[2];
    fold_sum_multi<2>(w.part, kMaxPartials, gridDim.x, f2, sh);
    const double RZ = f2[0], RR = f2[1];
    if (threadIdx.x == 0) {
      PcgState& st = *w.st;
      st.rz = RZ;
      st.rr = RR;
      st.rr0 = RR;
      // thr_rel > 0: a threshold relative to max(||r0||, rel_floor) (box_kkt_h8._pcg
      // uses rel_floor = 1), never below the absolute one
      const double t = thr_rel > 0.0 ? thr_rel * fmax(sqrt(RR), rel_floor) : 0.0;
      st.thr_sq = fmax(thr_sq, t * t);
      st.alpha = st.beta = 0.0;
      st.breakdown = 0;
      st.nonfinite = !isfinite(RR) || (!custom_pre && !isfinite(RZ));
      st.steps = 0;
      st.iter = 0;
      st.converged = 0;
      st.active = 1;
      st.outer_done = 0;
      st.trips = 0;
      st.max_trips = max_trips;
      st.bar_count = 0u;
      st.bar_gen = 0u;
      st.grid_error = 0;
      st.outer_rr = 0.0;
      if (outer_rr) st.outer_rr = *outer_rr;
      // the checks the host used to make before the first iteration
      if (outer_rr && isfinite(st.outer_rr) && !(st.outer_rr > outer_thr_sq)) {
        st.outer_done = 1;
        st.active = 0;
      } else if (st.nonfinite || (outer_rr && !isfinite(st.outer_rr))) {
        st.nonfinite = 1;
        st.active = 0;
      } else if (mode != PCG_PERIODIC && !(RR > st.thr_sq)) {
        st.converged = 1;
        st.active = 0;
      } else if (!custom_pre && mode == PCG_STRICT && !(RZ > 0.0)) {
        st.breakdown = 1;
        st.active = 0;
      }
      *w.counter = 0u;
    }
  }
}

// With a custom preconditioner: p = z and rz = r.z after M was applied.
template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_rz_kernel(int n, PcgWs<T> w, int start, int mode) {
  if (!w.st->active) return;
  __shared__ double sh[96];
  double rz = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    rz += double(w.r[i]) * double(w.z[i]);
  double s = block_sum(rz, sh);
  if (threadIdx.x == 0) w.part[blockIdx.x] = s;
  if (arrive_last(w.counter)) {
    const double RZ = fold_sum(w.part, gridDim.x, sh);
    if (threadIdx.x == 0) {
      PcgState& st = *w.st;
      if (start) {
        st.rz = RZ;
        st.nonfinite |= !isfinite(RZ);
        if (mode == PCG_STRICT && !(RZ > 0.0)) st.breakdown = 1;
        if (st.nonfinite || st.breakdown) st.active = 0;
      } else {
        // beta of the preconditioned update (see pcg_update_kernel)
        if (!isfinite(RZ)) st.nonfinite = 1;
        if (mode == PCG_STRICT && !(RZ > 0.0)) st.breakdown = 1;
        st.beta = (mode == PCG_STRICT) ? RZ / st.rz : ((st.rz > 0.0) ? RZ / st.rz : 0.0);
        st.rz = RZ;
        if (st.breakdown || st.nonfinite) st.active = 0;
      }
      *w.counter = 0u;
    }
  }
}

template <typename T>
__global__ void pcg_copy_p_kernel(int n, PcgWs<T> w) {
  if (!w.st->active) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w.p[i] = w.z[i];
}

template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_alpha_kernel(int n, PcgWs<T> w, int mode) {
  if (!w.st->active) return;
  __shared__ double sh[96];
  double pap = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pap += double(w.p[i]) * double(w.Ap[i]);
  double s = block_sum(pap, sh);
  if (threadIdx.x == 0) w.part[blockIdx.x] = s;
  if (arrive_last(w.counter)) {
    const double PAP = fold_sum(w.part, gridDim.x, sh);
    if (threadIdx.x == 0) {
      PcgState& st = *w.st;
      st.iter += 1;
      if (mode == PCG_PERIODIC) {
        if (!isfinite(PAP) || PAP <= 1e-30) {
          st.breakdown = 1;
          st.active = 0;
        } else {
          st.alpha = st.rr / (PAP + 1e-30);
        }
      } else {
        if (!isfinite(PAP)) st.nonfinite = 1;
        if (!(PAP > 0.0)) st.breakdown = 1;
        if (st.breakdown || st.nonfinite) {
          st.active = 0;
        } else {
          st.alpha = st.rz / PAP;
          st.steps += 1;
        }
      }
      *w.counter = 0u;
    }
  }
}

// x += alpha p; r -= alpha Ap; z = M r (Jacobi/identity inline); rz, rr.
template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_update_kernel(int n, PcgWs<T> w, T* __restrict__ x,
                                                              const T* __restrict__ inv_diag, int custom_pre,
                                                              int mode, int check_every) {
  if (!w.st->active) return;
  __shared__ double sh[96];
  const T a = T(w.st->alpha);
  double rz = 0, rr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = x[i] + a * w.p[i];
    const T r = w.r[i] - a * w.Ap[i];
    w.r[i] = r;
    rr += double(r) * double(r);
    if (!custom_pre) {
      const T z = inv_diag ? r * inv_diag[i] : r;
      w.z[i] = z;
      rz += double(r) * double(z);
    }
  }
  double v2[2] = {rz, rr};
  block_sum_multi<2>(v2, sh);
  if (threadIdx.x == 0) {
    w.part[blockIdx.x] = v2[0];
    w.part[kMaxPartials + blockIdx.x] = v2[1];
  }
  if (arrive_last(w.counter)) {
    double f2[2];
    fold_sum_multi<2>(w.part, kMaxPartials, gridDim.x, f2, sh);
    const double RZ = f2[0], RR = f2[1];
    if (threadIdx.x == 0) {
      PcgState& st = *w.st;
      if (!isfinite(RR) || (!custom_pre && !isfinite(RZ))) st.nonfinite = 1;
      if (mode == PCG_PERIODIC) {
        st.beta = RR / (st.rr + 1e-30);
        st.rr = RR;
        st.rz = RR;
        if (st.iter % check_every == 0) {
          if (RR < st.thr_sq) {
            st.converged = 1;
            st.active = 0;
          } else if (RR > 1e12 * st.rr0) {
            st.active = 0;
          }
        }
      } else {
        st.rr = RR;
        if (!(RR > st.thr_sq)) {
          st.converged = 1;
          st.active = 0;
        } else if (!custom_pre) {
          if (mode == PCG_STRICT && !(RZ > 0.0)) st.breakdown = 1;
          st.beta = (mode == PCG_STRICT) ? RZ / st.rz : ((st.rz > 0.0) ? RZ / st.rz : 0.0);
          st.rz = RZ;
        }
      }
      if (st.breakdown || st.nonfinite) st.active = 0;
      *w.counter = 0u;
    }
  }
}

// pcg_alpha_kernel + pcg_update_kernel in one launch, with p . Ap produced by the
// operator (*pap).  Every block derives alpha from the same device scalars; the
// last block does the state bookkeeping of both kernels.
template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_update_dot_kernel(int n, PcgWs<T> w, T* __restrict__ x,
                                                                  const T* __restrict__ inv_diag, int custom_pre,
                                                                  int mode, int check_every,
                                                                  const double* __restrict__ pap) {
  if (!w.st->active) return;
  __shared__ double sh[96];
  const double PAP = *pap;
  bool ok;
  double alpha;
  if (mode == PCG_PERIODIC) {
    ok = isfinite(PAP) && PAP > 1e-30;
    alpha = w.st->rr / (PAP + 1e-30);
  } else {
    ok = isfinite(PAP) && PAP > 0.0;
    alpha = w.st->rz / PAP;
  }
  const T a = T(alpha);
  double rz = 0, rr = 0;
  if (ok) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      x[i] = x[i] + a * w.p[i];
      const T r = w.r[i] - a * w.Ap[i];
      w.r[i] = r;
      rr += double(r) * double(r);
      if (!custom_pre) {
        const T z = inv_diag ? r * inv_diag[i] : r;
        w.z[i] = z;
        rz += double(r) * double(z);
      }
    }
  }
  double v2[2] = {rz, rr};
  block_sum_multi<2>(v2, sh);
  if (threadIdx.x == 0) {
    w.part[blockIdx.x] = v2[0];
    w.part[kMaxPartials + blockIdx.x] = v2[1];
  }
  if (arrive_last(w.counter)) {
    double f2[2];
    fold_sum_multi<2>(w.part, kMaxPartials, gridDim.x, f2, sh);
    const double RZ = f2[0], RR = f2[1];
    if (threadIdx.x == 0) {
      PcgState& st = *w.st;
      st.iter += 1;
      if (!ok) {
        if (mode == PCG_PERIODIC) {
          st.breakdown = 1;
        } else {
          if (!isfinite(PAP)) st.nonfinite = 1;
          if (!(PAP > 0.0)) st.breakdown = 1;
        }
        st.active = 0;
      } else {
        st.alpha = alpha;
        if (mode != PCG_PERIODIC) st.steps += 1;
        if (!isfinite(RR) || (!custom_pre && !isfinite(RZ))) st.nonfinite = 1;
        if (mode == PCG_PERIODIC) {
          st.beta = RR / (st.rr + 1e-30);
          st.rr = RR;
          st.rz = RR;
          if (st.iter % check_every == 0) {
            if (RR < st.thr_sq) {
              st.converged = 1;
              st.active = 0;
            } else if (RR > 1e12 * st.rr0) {
              st.active = 0;
            }
          }
        } else {
          st.rr = RR;
          if (!(RR > st.thr_sq)) {
            st.converged = 1;
            st.active = 0;
          } else if (!custom_pre) {
            if (mode == PCG_STRICT && !(RZ > 0.0)) st.breakdown = 1;
            st.beta = (mode == PCG_STRICT) ? RZ / st.rz : ((st.rz > 0.0) ? RZ / st.rz : 0.0);
            st.rz = RZ;
          }
        }
        if (st.breakdown || st.nonfinite) st.active = 0;
      }
      *w.counter = 0u;
    }
  }
}

template <typename T>
__global__ void pcg_dir_kernel(int n, PcgWs<T> w) {
  if (!w.st->active) return;
  const T beta = T(w.st->beta);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    w.p[i] = w.z[i] + beta * w.p[i];
}

template <typename T>
int pcg_run(const LinOp<T>& A, int n, const PcgWs<T>& w, const T* b, const T* inv_diag, const Precond<T>* M, T* x,
            double thr, int maxiter, int check_every, PcgMode mode, double, PcgResult* out, cudaStream_t s,
            const PcgLoop* loop) {
  PcgThreshold t;
  if (thr >= 0.0) {
    t.abs = thr;
  } else {  // relative to max(||r0||, 1)
    t.rel = -thr;
    t.rel_floor = 1.0;
  }
  return pcg_run_thr<T>(A, n, w, b, inv_diag, M, x, t, maxiter, check_every, mode, out, s, loop);
}

template <typename T>
int pcg_run_thr(const LinOp<T>& A, int n, const PcgWs<T>& w, const T* b, const T* inv_diag, const Precond<T>* M,
                T* x, const PcgThreshold& thr, int maxiter, int check_every, PcgMode mode, PcgResult* out,
                cudaStream_t s, const PcgLoop* loop) {
  if (check_every < 1 || maxiter < 1) return PHASTB_ERR_ARG;
  const int G = grid_for(n);
  int st;
  const int custom = M != nullptr && M->apply != nullptr;
  if ((st = cuda_status(cudaMemsetAsync(w.counter, 0, sizeof(unsigned), s)))) return st;
  if ((st = A(x, w.Ap, nullptr, s))) return st;
  // The start-of-solve decisions (relative threshold, already converged,
  // non-finite, non-positive curvature) are taken on the device: no host
  // round trip before the first chunk.
  { note_launch(); pcg_start_kernel<T><<<G, kThreads, 0, s>>>(n, w, b, inv_diag, custom, thr.abs * thr.abs, mode, thr.rel, thr.rel_floor, thr.outer_rr, thr.outer_thr * thr.outer_thr, (maxiter + check_every - 1) / check_every); }
  if ((st = last_launch_status())) return st;
  const int* active = &w.st->active;
  if (custom) {
    if ((st = M->apply(M->ctx, w.r, w.z, active, s))) return st;
    { note_launch(); pcg_rz_kernel<T><<<G, kThreads, 0, s>>>(n, w, 1, mode); }
    { note_launch(); pcg_copy_p_kernel<T><<<G, kThreads, 0, s>>>(n, w); }
    if ((st = last_launch_status())) return st;
  }
  PcgState hs{};
  int it = 0;
  bool looped = false;
  if (loop && !custom) {
    const int ls = (*loop)(maxiter);
    if (ls == PHASTB_OK) {
      if ((st = cuda_status(cudaMemcpyAsync(&hs, w.st, sizeof(hs), cudaMemcpyDeviceToHost, s)))) return st;
      if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
      if (hs.grid_error) return PHASTB_ERR_CUDA;
      looped = true;
    } else if (ls != PHASTB_UNSUPPORTED) {
      return ls;
    }
  }
  auto iterate = [&](int k_iters) -> int {
    int e;
    for (int k = 0; k < k_iters; ++k) {
      if (A.apply_dot) {
        if ((e = A.apply_dot(A.ctx, w.p, w.Ap, active, s))) return e;
        { note_launch(); pcg_update_dot_kernel<T><<<G, kThreads, 0, s>>>(n, w, x, inv_diag, custom, mode, check_every, A.dot_out); }
      } else {
        if ((e = A(w.p, w.Ap, active, s))) return e;
        { note_launch(); pcg_alpha_kernel<T><<<G, kThreads, 0, s>>>(n, w, mode); }
        { note_launch(); pcg_update_kernel<T><<<G, kThreads, 0, s>>>(n, w, x, inv_diag, custom, mode, check_every); }
      }
      if (custom) {
        if ((e = M->apply(M->ctx, w.r, w.z, active, s))) return e;
        { note_launch(); pcg_rz_kernel<T><<<G, kThreads, 0, s>>>(n, w, 0, mode); }
      }
      { note_launch(); pcg_dir_kernel<T><<<G, kThreads, 0, s>>>(n, w); }
    }
    return last_launch_status();
  };
  GraphKey key;
  key_val(key, A.apply);
  key_val(key, A.apply_dot);
  key_val(key, A.dot_out);
  key_add(key, A.ctx, A.ctx_bytes);
  key_val(key, custom);
  if (custom) {
    key_val(key, M->apply);
    key_add(key, M->ctx, M->ctx_bytes);
  }
  key_val(key, w);
  key_val(key, x);
  key_val(key, inv_diag);
  key_val(key, n);
  key_val(key, mode);
  key_val(key, check_every);
  const int size_t_ = sizeof(T);
  key_val(key, size_t_);
  long long glaunch = 0;
  // Preferred: the whole iteration loop on the device (one conditional-WHILE
  // graph, one host synchronisation per solve).  Otherwise chunks of
  // check_every iterations with a host check after each.
  cudaGraphExec_t wexec = !looped && device_loop_enabled()
                              ? while_graph_for(key, s, [&] { return iterate(check_every); }, active,
                                                &w.st->trips, &w.st->max_trips, &glaunch)
                              : nullptr;
  if (looped) {
    it = maxiter;
  } else if (wexec) {
    if ((st = cuda_status(cudaGraphLaunch(wexec, s)))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(&hs, w.st, sizeof(hs), cudaMemcpyDeviceToHost, s)))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    note_launch(glaunch * (long long)hs.trips);
    it = maxiter;
  } else {
    cudaGraphExec_t gexec =
        maxiter >= check_every ? graph_for(key, s, [&] { return iterate(check_every); }, &glaunch) : nullptr;
    while (it < maxiter) {
      const int chunk = std::min(check_every, maxiter - it);
      if (gexec && chunk == check_every) {
        if ((st = launch_graph(gexec, glaunch, s))) return st;
      } else if ((st = iterate(chunk))) {
        return st;
      }
      it += chunk;
      if ((st = cuda_status(cudaMemcpyAsync(&hs, w.st, sizeof(hs), cudaMemcpyDeviceToHost, s)))) return st;
      if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
      if (!hs.active) break;
    }
  }
  out->breakdown = hs.breakdown;
  out->nonfinite = hs.nonfinite;
  out->converged = hs.converged;
  out->rnorm = std::sqrt(hs.rr);
  out->iterations = (mode == PCG_PERIODIC) ? hs.iter : (hs.converged ? hs.steps : std::min(hs.iter, maxiter));
  out->outer_done = hs.outer_done;
  out->outer_rnorm = std::sqrt(hs.outer_rr);
  return PHASTB_OK;
}

template size_t pcg_ws_bytes<double>(int);
template size_t pcg_ws_bytes<float>(int);
template PcgWs<double> pcg_ws<double>(void*, int);
template PcgWs<float> pcg_ws<float>(void*, int);
template int pcg_run<double>(const LinOp<double>&, int, const PcgWs<double>&, const double*, const double*,
                             const Precond<double>*, double*, double, int, int, PcgMode, double, PcgResult*,
                             cudaStream_t, const PcgLoop*);
template int pcg_run<float>(const LinOp<float>&, int, const PcgWs<float>&, const float*, const float*,
                            const Precond<float>*, float*, double, int, int, PcgMode, double, PcgResult*,
                            cudaStream_t, const PcgLoop*);
template int pcg_run_thr<double>(const LinOp<double>&, int, const PcgWs<double>&, const double*, const double*,
                                 const Precond<double>*, double*, const PcgThreshold&, int, int, PcgMode, PcgResult*,
                                 cudaStream_t, const PcgLoop*);
template int pcg_run_thr<float>(const LinOp<float>&, int, const PcgWs<float>&, const float*, const float*,
                                const Precond<float>*, float*, const PcgThreshold&, int, int, PcgMode, PcgResult*,
                                cudaStream_t, const PcgLoop*);

// ================================================================ vector ops

template <typename T>
__global__ void __launch_bounds__(kThreads) norm2_kernel(const T* __restrict__ x, int n, RedWs ws) {
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] += double(x[i]) * double(x[i]);
  reduce_multi<1>(acc, ws);
}

template <typename T>
int vec_norm2(const T* x, int n, double* host, void* base, cudaStream_t s) {
  RedWs ws = red_ws(base);
  int st = red_ws_reset(ws, s);
  if (st) return st;
  { note_launch(); norm2_kernel<T><<<grid_for(n), kThreads, 0, s>>>(x, n, ws); }
  if ((st = last_launch_status())) return st;
  double v;
  if ((st = red_ws_fetch(ws, &v, 1, s))) return st;
  *host = std::sqrt(v);
  return PHASTB_OK;
}

template int vec_norm2<double>(const double*, int, double*, void*, cudaStream_t);
template int vec_norm2<float>(const float*, int, double*, void*, cudaStream_t);

}  // namespace phastb
