// Tiled, z-marching voxel H8 elastic action (one kernel, no element scratch).
//
// A block owns an ox x oy x kz brick of reduced nodes and marches through its
// node layers in z.  For each element layer it stages the two bounding node
// layers (u and d) of the brick plus a one-node halo in shared memory, every
// thread computes one element of the (ox+1) x (oy+1) element tile (the halo
// row/column elements are recomputed by the neighbouring bricks), writes the
// element's lower- and upper-face nodal forces to shared memory, and each
// owned node then sums its four lower-face contributions of this layer and the
// four upper-face contributions of the previous layer in a fixed order: the
// result is deterministic and independent of the tile shape's schedule.
//
// The degradation g(d) at the Gauss points and the macro-strain E rows
// (Pt sum_q w g sigma) are fused; optionally the kernel also returns x . y
// (the p . Ap product of CG) and the elastic energy, all through the
// deterministic per-block partials of reduce.cuh.
#pragma once
#include "h8_kernels.cuh"
#include "reduce.cuh"

namespace phastb {

struct TileShape {
  int ox, oy, kz;
};

constexpr int kTileMaxThreads = 256;

inline int tile_threads(const TileShape& t) { return ((t.ox + 1) * (t.oy + 1) + 31) / 32 * 32; }

// kz = 0: the launch picks the z depth from the kernel's occupancy.
inline bool tile_ok(const TileShape& t) {
  // each thread stages at most two halo-tile nodes per layer
  return t.ox >= 1 && t.oy >= 1 && t.kz >= 0 && tile_threads(t) <= kTileMaxThreads &&
         (t.ox + 2) * (t.oy + 2) <= 2 * tile_threads(t);
}

// Byte offset, rounded up to 16, of the staged per-element arrays that follow
// node_words * nt + face_words * exy words of node and face buffers.
template <typename T>
__host__ __device__ inline size_t tile_stage_offset(int nt, int exy, int node_words, int face_words) {
  return (sizeof(T) * ((size_t)node_words * nt + (size_t)face_words * exy) + 15) / 16 * 16;
}

// Words per element staged for the next element layer: (lam_q, mu_q) of the
// per-Gauss-point coarse operators, H of the damage action.
constexpr int kStageQP = 16, kStageH = 8;

// Dynamic shared memory of h8_tile_kernel: node buffers [3][4][nt] and face
// buffers [2][12][exy]; then, 16-byte aligned, with per-Gauss-point moduli two
// element layers of staged (lam_q, mu_q), 16 words per element; then, for a
// Chebyshev step, two layers of the owned nodes' staged (res, invd, xs) [2][9][ox*oy].
// Returns the total bytes; *off_qp and *off_cheb receive the two offsets.
template <typename T>
__host__ __device__ inline size_t tile_layout(int ox, int oy, bool qp, bool cheb, size_t* off_qp, size_t* off_cheb) {
  const int nt = (ox + 2) * (oy + 2), exy = (ox + 1) * (oy + 1);
  size_t o = tile_stage_offset<T>(nt, exy, 12, 24);
  *off_qp = o;
  if (qp) o += sizeof(T) * 2 * kStageQP * (size_t)exy;
  *off_cheb = o;
  if (cheb) o += (sizeof(T) * 2 * 9 * (size_t)ox * oy + 15) / 16 * 16;
  return o;
}

// TMA staging of the node layers (h8_tile_kernel with TMA): per node layer one
// buffer of the halo tile's oy + 2 rows for u~ (3 components interleaved per
// node) and one for d, each row W (or Wd) words long.  A tiled copy must start
// on a 16-byte boundary, so the row's first word is the node column i0 - 1
// rounded down to a multiple of A = 16 / sizeof(T) words and the kernel indexes
// from the remainder (at most A - 1 words).  Three layers are in flight; every
// buffer starts on a 128-byte boundary of the (realigned) dynamic shared memory.
template <typename T>
__host__ __device__ inline int tma_wx(int ox) {
  const int A = 16 / (int)sizeof(T);
  return (3 * (ox + 2) + A - 1 + A - 1) / A * A;
}
template <typename T>
__host__ __device__ inline int tma_wd(int ox) {
  const int A = 16 / (int)sizeof(T);
  return ((ox + 2) + A - 1 + A - 1) / A * A;
}
__host__ __device__ inline size_t align128(size_t b) { return (b + 127) / 128 * 128; }
template <typename T>
__host__ __device__ inline size_t tma_xbytes(int ox, int oy) {
  return align128(sizeof(T) * (size_t)tma_wx<T>(ox) * (oy + 2));
}
template <typename T>
__host__ __device__ inline size_t tma_dbytes(int ox, int oy) {
  return align128(sizeof(T) * (size_t)tma_wd<T>(ox) * (oy + 2));
}

// Dynamic shared memory of the TMA variant, relative to the 128-byte aligned
// base: [3 u~ layer buffers][3 d layer buffers][face buffers [2][12][exy]], then
// the staged per-element arrays and Chebyshev node data as in tile_layout.
// Returns the bytes to request (128 bytes of slack for the realignment).
template <typename T>
__host__ __device__ inline size_t tile_layout_tma(int ox, int oy, bool qp, bool cheb, size_t* off_face, size_t* off_qp,
                                                  size_t* off_cheb) {
  const int exy = (ox + 1) * (oy + 1);
  size_t o = 3 * (tma_xbytes<T>(ox, oy) + tma_dbytes<T>(ox, oy));
  *off_face = o;
  o += sizeof(T) * 24 * (size_t)exy;
  o = (o + 15) / 16 * 16;
  *off_qp = o;
  if (qp) o += sizeof(T) * 2 * kStageQP * (size_t)exy;
  *off_cheb = o;
  if (cheb) o += (sizeof(T) * 2 * 9 * (size_t)ox * oy + 15) / 16 * 16;
  return o + 128;
}

// Result slots of the apply's reduction workspace (ws.out).
enum ApplyOut { kOutE = 0, kOutEnergy = 6, kOutDot = 7, kApplyOuts = 8 };

// Element coefficients: material slot with g(d) (isotropic / general Voigt), or
// per-Gauss-point isotropic moduli (multigrid coarse levels, no macro strain).
enum TileCoef { kCoefIso = 0, kCoefAniso = 1, kCoefQP = 2 };
// Node epilogue: y = A x; y and x . y; y and the energy; one Chebyshev step;
// y = A x on the nodal block only (the macro-strain E rows of x are not read,
// those of y are set to zero: a smoother's residual with the E rows masked).
enum TileMode { kModeApply = 0, kModeDot = 1, kModeEnergy = 2, kModeCheb = 3, kModeNodal = 4 };

// Gauss-point constants of the action: N1 weights with the 1/h of each axis
// folded in (the last interpolation stage of a derivative applies them).
template <typename T>
struct TileK {
  T c1, c2;                  // N1 = [[c1, c2], [c2, c1]]
  T x1, x2, y1, y2, z1, z2;  // c1/h, c2/h per axis
};

template <typename T>
struct TileArgs {
  VoxGeom g;
  TileShape ts;
  int pad_;
  const uint8_t* slot;  // kCoefIso / kCoefAniso
  const T* gq;          // optional (E, 8) degradation; else g(d) from d, else 1
  const T* d;
  const T* lam_q;       // kCoefQP: (E, 8) moduli
  const T* mu_q;
  const T* x;
  T* y;
  const uint8_t* mask;
  // kModeCheb: res -= A x;  d_out = c1 x + c2 invd res;  xs += d_out
  T* res;
  const T* invd;
  T* xs;
  T* d_out;
  double c1, c2;
  RedWs ws;
  const int* guard;
  TileK<T> k;
};

// Tile shape used for a grid, word size and coefficient class (0: material
// slots, 1: per-Gauss-point moduli): the recorded (tuned or pinned) choice when
// there is one, otherwise a heuristic.
TileShape tile_shape_for(const VoxGeom& g, int word, int cls);
bool tile_shape_lookup(const VoxGeom& g, int word, int cls, TileShape* t);

// Records a tile shape (host table, per process).
void tile_shape_record(const VoxGeom& g, int word, int cls, const TileShape& t);

template <typename T>
struct DTileArgs {
  VoxGeom g;
  TileShape ts;
  int pad_;
  const uint8_t* slot;
  T gc_ell[PHASTB_MAX_SLOTS];  // Gc / ell per material slot
  T gc_k2[PHASTB_MAX_SLOTS];   // 2 w Gc ell per material slot
  double kappa, ell, scale;
  const T* H;  // (E, 8) history, may be null
  const T* x;
  T* y;
  const uint8_t* mask;
  RedWs ws;
  const int* guard;
  TileK<T> k;
};

// Damage action y = scale [Gc (M/ell + ell L) + 2 (1-kappa) H-mass] x on the
// brick schedule (tile shapes of coefficient class 2), masked rows zero; with
// `dot` also x . y at ws.out[kOutDot].
template <typename T>
int h8_damage_tile_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* x, const T* H,
                          double scale, const uint8_t* mask, T* y, RedWs ws, const int* guard, bool dot,
                          cudaStream_t s);

template <typename T>
struct PcgWs;

// Every iteration of a Jacobi-preconditioned (inv_diag) or unpreconditioned CG
// on the masked damage operator in one cooperative launch, continuing from the
// state that pcg_start_kernel left in w (engine.cuh's PcgLoop contract); p_alt
// is a second direction buffer of n_red values.  PHASTB_UNSUPPORTED when the
// device cannot run it (or PHASTB_PERSISTENT_PCG=0): the caller iterates with
// separate launches instead.
template <typename T>
int h8_damage_pcg_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* H, double scale,
                         const uint8_t* mask, const PcgWs<T>& w, T* p_alt, T* x, const T* inv_diag, int maxiter,
                         int mode, cudaStream_t s);

// y = A(d) x with fused g(d); optional x . y (DOT) and energy (ENERGY).  ws.out
// receives the E-row sums (kOutE..), the energy and the dot.
template <typename T>
int h8_mech_tile_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* x, const T* gq,
                        const T* d, const uint8_t* mask, T* y, RedWs ws, const int* guard, bool dot, bool energy,
                        cudaStream_t s, const TileShape* force_shape = nullptr);

// Fills the geometry-derived members of a TileArgs (g, ts, k) for grid v and
// coefficient class cls.
template <typename T>
TileArgs<T> tile_args(const VoxGeom& v, int cls);

// ------------------------------------------------------------ packed cell batches
//
// Many periodic cells of different sizes in one launch: every block runs one
// brick of one cell (the same tile body as a single-grid launch, with the
// brick's index inside its cell), and each cell's reductions go to its own
// workspace with its own ticket, folded by the cell's last block.

// One cell of a packed batch: its grid, its brick schedule (the batch's ox x oy
// bricks, kz node layers deep, nvb bricks), the offsets of its data in the
// packed arrays (reduced nodes; mechanics unknowns, 3 n_red + 6 per cell;
// elements) and its phase-field length and damage-system scale.
struct BatchCell {
  VoxGeom g;
  TileShape ts;
  int nvb;
  long long node_off, mech_off, elem_off;
  double ell, dscale;
  TileK<float> kf;
  TileK<double> kd;
};

// A batched launch over the packed arrays.  Per block work[b] = (cell, brick);
// cell c's reductions use the workspace at ws + c * red_ws_bytes(); its guard
// word (an engine's `active` flag; null: none) is guard[c * guard_stride].
template <typename T>
struct TileBatchArgs {
  const BatchCell* cells;
  const int2* work;
  int n_blocks;
  int guard_stride;
  const uint8_t* slot;  // elements
  const T* d;           // nodes (null: g = 1)
  const T* H;           // damage action: (E, 8) per element (null: no history term)
  const T* x;           // elastic action: mechanics vector; damage action: nodes
  T* y;
  const uint8_t* mask;  // like x (null: none)
  char* ws;
  const int* guard;
  double kappa;         // damage action
  int dscale;           // damage action: 1 scales it by each cell's damage-system scale
  int pad_;
  // multigrid levels (kCoefQP: per-Gauss-point moduli, 8 per element, at 8 * elem_off) and the
  // Chebyshev step (kModeCheb: res -= A x; d_out = c1 x + c2 s_c invd res; xs += d_out, with the
  // per-cell factor s_c = c2_scale[c] or 1), vectors laid out like x
  const T* lam_q;
  const T* mu_q;
  T* res;
  const T* invd;
  T* xs;
  T* d_out;
  double c1, c2;
  const double* c2_scale;
};

// One multigrid-level launch of the batch: kCoefIso (the fine level: slots and g(d)) or kCoefQP
// (coarse levels) in mode kModeApply, kModeNodal or kModeCheb.  FP32, bricks 16 x 8 or 8 x 8.
int h8_tile_batch_level_launch(const TileBatchArgs<float>& b, const VoxMat<float>& m, int coef, int mode, int ox,
                               int oy, cudaStream_t s);

// y = A(d) x on every cell of the batch (MODE kModeApply or kModeDot: also
// x . y per cell at ws_c.out[kOutDot]; the E-row sums at ws_c.out[0..5]).
template <typename T>
int h8_tile_batch_launch(const TileBatchArgs<T>& b, const VoxMat<T>& m, int mode, int ox, int oy, cudaStream_t s);

// The damage action of every cell (dot: x . y per cell at ws_c.out[kOutDot]).
template <typename T>
int h8_dtile_batch_launch(const TileBatchArgs<T>& b, const VoxMat<T>& m, bool dot, int ox, int oy, cudaStream_t s);

// Launches the tile kernel for (COEF, MODE) with prepared arguments.  With
// `tune` and PHASTB_AUTOTUNE=1 in the environment, the first plain or dot
// launch for a grid with no recorded shape (outside stream capture, unguarded)
// times the candidate shapes and records the fastest; otherwise the
// deterministic heuristic shape is used.
template <typename T>
int h8_tile_launch(const TileArgs<T>& a, const VoxMat<T>& m, int coef, int mode, cudaStream_t s, bool tune = true);

}  // namespace phastb
