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

inline bool tile_ok(const TileShape& t) {
  // each thread stages at most two halo-tile nodes per layer
  return t.ox >= 1 && t.oy >= 1 && t.kz >= 1 && tile_threads(t) <= kTileMaxThreads &&
         (t.ox + 2) * (t.oy + 2) <= 2 * tile_threads(t);
}

template <typename T>
inline size_t tile_smem_bytes(const TileShape& t) {
  const size_t nt = (size_t)(t.ox + 2) * (t.oy + 2), exy = (size_t)(t.ox + 1) * (t.oy + 1);
  return sizeof(T) * (3 * 4 * nt + 2 * 12 * exy);
}

// Result slots of the apply's reduction workspace (ws.out).
enum ApplyOut { kOutE = 0, kOutEnergy = 6, kOutDot = 7, kApplyOuts = 8 };

// Tile shape used for a grid and word size: the autotuned choice when one was
// recorded for this grid, otherwise a heuristic.
TileShape tile_shape_for(const VoxGeom& g, int word);

// Records / forgets a tuned tile shape (host table, per process).
void tile_shape_record(const VoxGeom& g, int word, const TileShape& t);

// y = A(d) x with fused g(d); optional x . y (DOT) and energy (ENERGY).  ws.out
// receives the E-row sums (kOutE..), the energy and the dot.
template <typename T>
int h8_mech_tile_launch(const VoxGeom& v, const VoxMat<T>& m, const uint8_t* slot, const T* x, const T* gq,
                        const T* d, const uint8_t* mask, T* y, RedWs ws, const int* guard, bool dot, bool energy,
                        cudaStream_t s, const TileShape* force_shape = nullptr);

}  // namespace phastb
