// Persistent mode: the whole time step of one environment in one cooperative
// launch (vbd_persist.cu).
#pragma once
#include <cuda_runtime.h>

#include "vbd_internal.h"

namespace vbd {

// Device-side control of one persistent step; zeroed by launch_persist
// before every launch.
struct PersistCtl {
  unsigned long long arrivals;      // grid-barrier arrivals in this step
  unsigned long long sub_arrivals;  // arrivals at the barriers among the small-colour blocks
  unsigned long long conv[3];       // per-sweep max |dx_x+dx_y+dx_z| bits, slot = sweep % 3
  unsigned status;                  // status bits (kStat*) of every block
  unsigned abort;                   // set when a barrier wait expired
};

// Bounds of every grid-barrier wait.
struct PersistLimits {
  long long max_polls;             // polls of the arrival counter
  unsigned long long max_wait_ns;  // wall-clock limit
};

// A colour of at most kPersistSmallBlocks x (warps per block) chunks is
// "small": it runs on the first few blocks only.
constexpr int kPersistSmallBlocks = 8;

// Neighbour-scoped readiness between the colours of a sweep.  Block b, before
// its share of colour c (c > 0) of sweep k, waits until every block of
// off[b * ncolors + c] .. off[b * ncolors + c + 1] in idx has finished colour
// c - 1 of sweep k: the blocks owning a vertex that shares a tet with one of
// b's colour-c vertices.  Each block publishes its progress in epoch[b *
// kEpochStride] (phases done: sweep * ncolors + colour + 1) with a release
// store; the waits are acquire loads.  Vertices of a colour read the latest
// values of lower colours and last sweep's values of higher colours exactly
// as with a barrier between colours, because the neighbour relation is
// symmetric: a block cannot start a higher colour before every block whose
// vertices it touches has finished the lower one.  The end of a sweep stays a
// grid barrier (the convergence test needs every block's maximum).
constexpr int kEpochStride = 16;  // one 128-byte line per block
struct PersistNbr {
  const int* off;                // [blocks * ncolors + 1]
  const int* idx;
  unsigned long long* epoch;     // [blocks * kEpochStride], zeroed before every launch
};

// Largest record table (bytes) a persistent launch stages in shared memory.
constexpr int kPersistMaxTabSmem = 64 * 1024;

// Resident persist_kernel blocks per SM for `threads` threads and `smem`
// bytes of dynamic shared memory (the staged record table, or 0).
cudaError_t persist_occupancy(int prec, int material, int fmt, int tpv, int threads, size_t smem,
                              int* blocks_per_sm);

// One time step: clears *ctl and m.status[0], then a cooperative launch of
// `blocks` blocks (at most the resident count).  Writes m.iters[0] and ORs
// the step's status bits into m.status[0]; a barrier wait that expired adds
// kStatTimeout there.  `parts` holds 4 x blocks doubles (warm-start energy
// partial sums; unused without a warm-start prediction).  `smem`: bytes of the
// record table when StepParams::tab_in_smem stages it, else 0.
// `nbr`: neighbour-scoped readiness between colours (nbr.off == nullptr: a
// grid barrier between colours instead).
cudaError_t launch_persist(int prec, int material, int tpv, int threads, const DevMesh& m,
                           const StepParams* p, PersistCtl* ctl, int blocks,
                           const PersistLimits& lim, double* parts, size_t smem,
                           const PersistNbr& nbr, cudaStream_t s);

}  // namespace vbd
