// Device-resident Krylov engines.
//
// The iteration state (alpha, beta, residual norms, flags) lives in device
// memory; every kernel reads it and turns into a no-op once the solve is
// finished, so the host can launch a whole chunk of iterations without
// looking at any scalar and synchronise only once per chunk.  Reductions are
// the deterministic last-block folds of common.cuh.
//
//   Ppcg   - bound-projected PCG of PhaseFieldDamageSolver._solve_projected_cg
//            (solvers/damage_solver.py:3528-3775)
//   Pcg    - Jacobi PCG with device flags of solid3d/linalg.py:pcg (freeze on
//            convergence, :99-220), of box_kkt_h8._pcg (:256-347, strict
//            curvature checks) and the unpreconditioned CG of
//            QuasiStaticSolver._cg_solve (mechanics_solver.py:1984-2043,
//            convergence looked at every 50 iterations).
#pragma once
#include "reduce.cuh"

#include <functional>
#include <vector>

namespace phastb {

// A linear operator y = A x on device vectors.  `guard` (device int, may be
// NULL) lets the operator skip work when the engine has finished.
template <typename T>
struct LinOp {
  int (*apply)(const void* ctx, const T* x, T* y, const int* guard, cudaStream_t s);
  const void* ctx;
  size_t ctx_bytes;  // size of *ctx: the bytes that identify a captured iteration graph
  // Optional: the same action that also leaves x . y (FP64, device) at *dot_out,
  // which lets CG skip its separate p . Ap reduction.
  int (*apply_dot)(const void* ctx, const T* x, T* y, const int* guard, cudaStream_t s) = nullptr;
  const double* dot_out = nullptr;
  int operator()(const T* x, T* y, const int* guard, cudaStream_t s) const { return apply(ctx, x, y, guard, s); }
};

// ---------------------------------------------------------------- PPCG

struct PpcgState {
  double rz, tol_sq, r0sq, alpha, beta;
  int go;          // iterating
  int go_resid;    // this iteration recomputes the true residual
  int done, reason, iter, last_iter;
  int branch;      // 0 full CG step, 1 capped step + restart
  int reset_dir;
  int max_iter, check_every;
};

struct PpcgWs {
  double *r, *z, *p, *Ap, *Ad, *lb, *minv, *b;
  uint8_t* act;
  double* part;      // 4 * kMaxPartials
  int* ipart;        // kMaxPartials
  unsigned* counter; // 4 tickets
  PpcgState* st;
};

size_t ppcg_ws_bytes(int n);
PpcgWs ppcg_ws(void* base, int n);

// Runs the solve; `d` holds the iterate (initialised from d_init or d_prev) and
// receives the clamped result.  Returns a PHASTB status; info[0] last_iter,
// info[1] reason.
int ppcg_solve(const LinOp<double>& A, int n, const PpcgWs& w, const double* d_prev, const double* d_init,
               const uint8_t* fixed, const double* vals, double tol, int max_iter, int check_every, double* d,
               int* info, cudaStream_t s);

// ---------------------------------------------------------------- PCG

enum PcgMode { PCG_FREEZE = 0, PCG_STRICT = 1, PCG_PERIODIC = 2 };

struct PcgState {
  double rz, rr, rr0, thr_sq, alpha, beta;
  int active;       // iterating (guard for the operator)
  int breakdown, nonfinite;
  int steps;        // iterations that moved the iterate
  int iter;
  int converged;
  double outer_rr;  // an enclosing refinement's residual norm^2, when one is checked at the start
  int outer_done;   // ... and that residual already met its threshold: nothing was iterated
  int trips;        // chunks run by the device-side loop ...
  int max_trips;    // ... which stops after this many (set per solve, not baked into the graph)
  // grid barrier of a persistent iteration kernel (reset by the start kernel)
  unsigned bar_count, bar_gen;
  int grid_error;   // a barrier wait ran out: the persistent kernel stopped early
  int pad_;
};

template <typename T>
struct PcgWs {
  T *r, *z, *p, *Ap;
  double* part;
  unsigned* counter;
  PcgState* st;
};

template <typename T>
size_t pcg_ws_bytes(int n);
template <typename T>
PcgWs<T> pcg_ws(void* base, int n);

// Preconditioner z = M^{-1} r (NULL ctx: Jacobi with inv_diag, or identity
// when inv_diag is NULL).
template <typename T>
struct Precond {
  int (*apply)(const void* ctx, const T* r, T* z, const int* guard, cudaStream_t s);
  const void* ctx;
  size_t ctx_bytes;
};

// Solves A x = b from x (initial guess held in x, zero allowed).  The caller
// has formed r = b - A x in w.r beforehand when `have_r` is set; otherwise the
// engine forms it.  thr is the absolute residual threshold on ||r||.
// iters/converged/breakdown/nonfinite are reported through `out`.
struct PcgResult {
  int iterations;
  int converged;
  int breakdown;
  int nonfinite;
  double rnorm;
  int outer_done;
  double outer_rnorm;
};

// Stopping rule of a PCG solve, evaluated on the device at the start:
// ||r|| <= max(abs, rel * max(||r0||, rel_floor)); with outer_rr set, the solve
// first checks *outer_rr <= outer_thr^2 (an enclosing refinement's FP64
// residual) and does nothing when it holds.
struct PcgThreshold {
  double abs = 0.0, rel = 0.0, rel_floor = 0.0;
  const double* outer_rr = nullptr;
  double outer_thr = 0.0;
};

// The iterations of a Jacobi- or identity-preconditioned solve run by one
// persistent launch: loop(maxiter) continues from the started state in the
// workspace with the iteration semantics of the engine and returns a status;
// PHASTB_UNSUPPORTED means it cannot run here and the engine iterates itself.
using PcgLoop = std::function<int(int maxiter)>;

template <typename T>
int pcg_run(const LinOp<T>& A, int n, const PcgWs<T>& w, const T* b, const T* inv_diag, const Precond<T>* M,
            T* x, double thr, int maxiter, int check_every, PcgMode mode, double rr0_for_div, PcgResult* out,
            cudaStream_t s, const PcgLoop* loop = nullptr);

template <typename T>
int pcg_run_thr(const LinOp<T>& A, int n, const PcgWs<T>& w, const T* b, const T* inv_diag, const Precond<T>* M,
                T* x, const PcgThreshold& thr, int maxiter, int check_every, PcgMode mode, PcgResult* out,
                cudaStream_t s, const PcgLoop* loop = nullptr);

// Vector helpers used by the drivers.
template <typename T>
int vec_norm2(const T* x, int n, double* host, void* red_ws_base, cudaStream_t s);

// CUDA-graph cache of captured iteration chunks (per host thread and device).
// `key` must hold every value the captured launches depend on.
using GraphKey = std::vector<unsigned char>;
inline void key_add(GraphKey& k, const void* p, size_t n) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  k.insert(k.end(), c, c + n);
}
template <typename V>
inline void key_val(GraphKey& k, const V& v) {
  key_add(k, &v, sizeof(V));
}
// Returns the executable graph of `body` (captured on s) or nullptr when the
// stream cannot be captured; *count receives the kernel launches per replay.
cudaGraphExec_t graph_for(const GraphKey& key, cudaStream_t s, const std::function<int()>& body, long long* count);

// A graph holding one conditional WHILE node: `body` (one chunk of solver
// iterations) then a one-thread kernel that sets the loop condition to
// *active && ++*trips < *max_trips.  The whole solve is one graph launch; the
// trip limit is read from device memory, so one graph serves every limit.
// nullptr when conditional nodes are unavailable.  *count: launches per trip.
cudaGraphExec_t while_graph_for(const GraphKey& key, cudaStream_t s, const std::function<int()>& body,
                                const int* active, int* trips, const int* max_trips, long long* count);

}  // namespace phastb
