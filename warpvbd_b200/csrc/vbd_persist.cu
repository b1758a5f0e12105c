// Persistent mode (one environment): the whole time step -- inertia guess,
// every colour of every sweep, the convergence test and the velocity update
// -- in ONE cooperative launch whose blocks stay resident and meet at grid
// barriers, instead of one kernel (graph node) per colour.
//
// The step loop of the reference (vbd_solver.py:509-612: initialise,
// colour loop with a host sync per launch, abs(dxs.sum(1)).max() < dx_tol
// after each sweep, velocity update) becomes:
//
//   begin     grid-stride over vertices: ut = u + dt v + dt^2 g, up = u,
//             active vertices start from ut                      | barrier
//   sweep     for each colour: warps take the colour's chunks grid-stride
//             and update their vertices (process_chunk).  Small colours (at
//             most kPersistSmallBlocks blocks' worth of chunks, e.g. the
//             107-vertex colours of a voxel cantilever) are done by the
//             first S blocks only (S = the largest small colour's chunk
//             count), one chunk per block, its slot steps split over the
//             block's warps.  Colours are separated by neighbour-scoped readiness
//             (PersistNbr, vbd_persist.h): a block waits only for the blocks
//             that own vertices sharing a tet with its own vertices of the
//             colour.  Without neighbour lists: a grid barrier between
//             colours, and inside a run of small colours a barrier among the
//             S blocks (__syncthreads when S = 1)
//             end of sweep: block max of |dx_x+dx_y+dx_z| -> atomicMax on
//             a rotating slot; the grid barrier; every block reads the slot
//             and takes the same stop decision
//   end       grid-stride velocity update; block 0 writes sweeps and status
//
// With the learned warm start (StepParams::warm and a prediction in
// DevMesh::ws_pred), between begin and the first sweep: the incremental
// potential at the inertia guess, then at inertia guess + alpha x predicted
// correction for alpha = 1, 1/2, 1/4 until one is lower (else back to the
// inertia guess).  Each potential is a grid-wide sum: every block writes its
// partial to its own slot of `parts`, and after a barrier every block adds
// the partials in block order, so all blocks take the same decision and the
// result does not depend on the order in which blocks finish.
//
// Grid barrier: one 64-bit arrival counter, zeroed before every launch;
// barrier k is passed when the counter reaches k * gridDim.x.  Arrival is a
// release reduction after __syncthreads + __threadfence, the wait an acquire
// load.  Every wait is bounded (an iteration cap and a wall-clock limit):
// on expiry the block sets the abort flag, ORs the timeout bit into the
// environment's status and returns, and every other block leaves at its
// next wait, so a launch that is not co-resident ends with VBD_ERR_TIMEOUT
// instead of hanging.  The environment's status word is zeroed before the
// launch and only ever OR-ed, so a timeout bit is never overwritten.  The
// launch is cooperative, which makes co-residency a launch-time check.
//
// Memory: vertex positions written in one colour are read by other blocks
// in later colours.  They are read with plain (weak, L1-cacheable) loads,
// never the non-coherent read-only path: every such read follows a grid
// barrier whose acquire (thread 0) and __syncthreads order it after the
// writing block's release, which the memory model makes visible (the
// acquire invalidates the SM's L1).
#include <cuda_runtime.h>

#include "vbd_device.cuh"
#include "vbd_persist.h"

namespace vbd {

namespace {

// Real4 state in global memory, plain loads (see the note on memory above).
template <typename SReal>
struct CoherentState {
  real4<SReal>* p;
  __device__ __forceinline__ real4<SReal> load(int i) const { return p[i]; }
  __device__ __forceinline__ void store(int i, const real4<SReal>& v) const { p[i] = v; }
};


__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add_u64(unsigned long long* p,
                                                    unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// This block has finished `phases` phases (sweep * ncolors + colour + 1):
// every thread's writes of them are ordered before the release store.
__device__ __forceinline__ void publish_epoch(const PersistNbr& nbr, unsigned long long phases) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release_u64(nbr.epoch + (size_t)blockIdx.x * kEpochStride, phases);
  }
}

// Waits until every neighbour block listed for (this block, colour) has
// published at least `need` phases.  The block's threads poll the list in
// parallel, each wait bounded like the grid barrier's; returns false when a
// wait expired here or elsewhere (the abort flag).
__device__ __forceinline__ bool wait_neighbours(const PersistNbr& nbr, int list,
                                                unsigned long long need, PersistCtl* ctl,
                                                const PersistLimits& lim) {
  const int b0 = __ldg(nbr.off + list), b1 = __ldg(nbr.off + list + 1);
  int ok = 1;
  for (int j = b0 + threadIdx.x; j < b1 && ok; j += blockDim.x) {
    const unsigned long long* e = nbr.epoch + (size_t)__ldg(nbr.idx + j) * kEpochStride;
    const unsigned long long t0 = globaltimer_ns();
    for (long long n = 0;; ++n) {
      if (ld_acquire_u64(e) >= need) break;
      const bool expired = n >= lim.max_polls ||
                           ((n & 255) == 255 && globaltimer_ns() - t0 > lim.max_wait_ns);
      if (expired || ld_relaxed_u32(&ctl->abort) != 0u) {
        if (expired) {
          atomicOr(&ctl->status, kStatTimeout);
          atomicExch(&ctl->abort, 1u);
        }
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
  }
  return __syncthreads_and(ok) != 0;
}

// Barrier on `counter` among the blocks that use it: passed when the counter
// reaches `target` (the number of barriers so far x the participants).
// Returns false if the launch is aborting (this block's wait expired, or
// another block's did).
__device__ __forceinline__ bool counter_sync(PersistCtl* ctl, unsigned long long* counter,
                                             unsigned long long target,
                                             const PersistLimits& lim, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    red_release_add_u64(counter, 1ull);
    const unsigned long long t0 = globaltimer_ns();
    for (long long n = 0;; ++n) {
      if (ld_acquire_u64(counter) >= target) break;
      const bool expired = n >= lim.max_polls ||
                           ((n & 255) == 255 && globaltimer_ns() - t0 > lim.max_wait_ns);
      if (expired || ld_relaxed_u32(&ctl->abort) != 0u) {
        if (expired) {
          atomicOr(&ctl->status, kStatTimeout);
          atomicExch(&ctl->abort, 1u);
        }
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Grid barrier number target / gridDim.x.
__device__ __forceinline__ bool grid_sync(PersistCtl* ctl, unsigned long long target,
                                          const PersistLimits& lim, int* s_ok) {
  if (gridDim.x == 1) {  // one block: __syncthreads is the barrier
    __syncthreads();
    return true;
  }
  return counter_sync(ctl, &ctl->arrivals, target, lim, s_ok);
}

template <typename Real, typename SReal, int TPV, int MAT, int FMT>
__global__ void __launch_bounds__(512) persist_kernel(DevMesh m,
                                                      const StepParams* __restrict__ pp,
                                                      PersistCtl* ctl, PersistLimits lim,
                                                      double* __restrict__ parts,
                                                      PersistNbr nbr) {
  using S4 = real4<SReal>;
  __shared__ unsigned long long s_red[16];
  __shared__ double s_dsum[16];
  __shared__ double s_total;
  __shared__ int s_ok;
  // per-part sums of a small colour's chunk (see the sweep loop)
  constexpr int kPartFloats = SplitBuf<TPV>::per_part;
  __shared__ Real s_split[Prefetch<TPV>::steps * kPartFloats];
  const StepConst sc = make_const(*pp);
  const double tol = pp->tol;
  const int max_iter = pp->max_iter;
  const EnvInfo e = m.env[0];
  const int nb = gridDim.x;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = nb * blockDim.x;
  S4* U = reinterpret_cast<S4*>(m.u);
  const CoherentState<SReal> state{U};
  unsigned long long bar = 0ull;  // arrivals that complete the next barrier
  // the mesh's record table: staged in this block's shared memory when the
  // launch reserved room for it (visible after the first barrier), else read
  // from global memory
  using R4 = real4<Real>;
  extern __shared__ __align__(16) unsigned char psmem[];
  const R4* tab = reinterpret_cast<const R4*>(m.rec_tab);
  if (pp->tab_in_smem) {
    R4* stab = reinterpret_cast<R4*>(psmem);
    for (int i = threadIdx.x; i < 3 * e.nrec; i += blockDim.x) stab[i] = ldg4(tab + i);
    tab = stab;
  }

#define VBD_GRID_SYNC()                                       \
  do {                                                        \
    bar += nb;                                                \
    if (!grid_sync(ctl, bar, lim, &s_ok)) {                   \
      if (threadIdx.x == 0) atomicOr(m.status, kStatTimeout); \
      return;                                                 \
    }                                                         \
  } while (0)

  // begin: inertia target and initial guess
  for (int i = tid; i < e.nv; i += nthreads)
    U[e.vbase + i] = begin_vertex<SReal>(m, e.vbase + i, i < e.nact, sc, true);
  VBD_GRID_SYNC();

  unsigned stat = 0u;
  if (pp->warm && m.ws_pred) {
    const S4* UT = reinterpret_cast<const S4*>(m.ut) + e.vbase;
    // grid-wide sums of per-block partials: each block writes its partial to
    // parts[slot * nb + block]; after a barrier every block adds them in block
    // order, so all blocks see the same total
    auto grid_sum = [&](double acc, int slot, bool& ok) -> double {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) s_dsum[warp] = acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        double v = 0.0;
        for (int i = 0; i < nwarps; ++i) v += s_dsum[i];
        parts[slot * nb + blockIdx.x] = v;
      }
      bar += nb;
      ok = grid_sync(ctl, bar, lim, &s_ok);
      if (ok && threadIdx.x == 0) {
        double v = 0.0;
        for (int b = 0; b < nb; ++b) v += __ldcg(parts + slot * nb + b);
        s_total = v;
      }
      __syncthreads();
      const double total = s_total;
      __syncthreads();  // s_total is reused by the next sum
      return total;
    };
    // incremental potential of the current U: the tets' strain energy (each
    // tet once, from the mesh's tet list) plus the solved vertices' inertia
    auto grid_energy = [&](int slot, bool& ok) -> double {
      double acc = tet_energy<Real, SReal, MAT>(m, e, state, tab, tid, nthreads, false).x;
      acc += inertia_energy<SReal>(m, e, state, sc, tid, nthreads, false);
      return grid_sum(acc, slot, ok);
    };
    auto place = [&](SReal alpha) {
      for (int i = tid; i < e.nsolved; i += nthreads) {
        const float4 d = m.ws_pred[e.vbase + i];
        if (d.w > 0.f) {
          S4 v = ldcg4(UT + i);
          v.x += alpha * SReal(d.x);
          v.y += alpha * SReal(d.y);
          v.z += alpha * SReal(d.z);
          U[e.vbase + i] = v;
        }
      }
    };
    // the potential at the inertia guess (U; its inertia energy is zero) and
    // at the full prediction in one pass (tet_energy forms the shifted
    // positions exactly as place(1) stores them)
    bool ok = true;
    double e0, e1;
    {
      const double2 el = tet_energy<Real, SReal, MAT>(m, e, state, tab, tid, nthreads, true);
      const double in1 = inertia_energy<SReal>(m, e, state, sc, tid, nthreads, true);
      e0 = grid_sum(el.x, 0, ok);
      e1 = ok ? grid_sum(el.y + in1, 1, ok) : 0.0;
    }
    bool used = ok && e1 < e0;  // false on NaN as well
    if (used) {
      place(SReal(1));
      bar += nb;
      ok = grid_sync(ctl, bar, lim, &s_ok);
    }
    // backtracking: half and a quarter of the prediction
    for (int trial = 1; trial < 3 && ok && !used; ++trial) {
      place(SReal(1.0 / double(1 << trial)));
      bar += nb;
      ok = grid_sync(ctl, bar, lim, &s_ok);
      if (!ok) break;
      const double et = grid_energy(1 + trial, ok);
      used = ok && et < e0;
    }
    if (!ok) {
      if (threadIdx.x == 0) atomicOr(m.status, kStatTimeout);
      return;
    }
    if (used) {
      stat |= kStatWarmUsed;
    } else {
      for (int i = tid; i < e.nsolved; i += nthreads) U[e.vbase + i] = ldcg4(UT + i);
      VBD_GRID_SYNC();
    }
  }
  // small colours run on the first nsb blocks, one chunk per block at a time
  // (as many blocks as the largest of them has chunks): the block's warps
  // split the chunk's slot steps (process_chunk_part) and warp 0 adds the
  // parts in part order -- a small colour's time is one chunk's dependent
  // chain, so a shorter chain is what shortens it
  auto is_small = [&](int nch) { return nb > 1 && nch <= kPersistSmallBlocks * nwarps; };
  const bool scoped = nb > 1 && nbr.off != nullptr;
  int nsb = 1;
  for (int c = 0; c < e.ncolors; ++c) {
    const int nch = m.color[e.cbase + c].chunk_end - m.color[e.cbase + c].chunk_begin;
    if (is_small(nch)) nsb = max(nsb, nch);
  }
  nsb = min(nsb, nb);
  constexpr int kParts = Prefetch<TPV>::steps;  // parts per chunk at most
  const int W = min(nwarps, kParts);
  unsigned long long sub_bar = 0ull;  // arrivals that complete the next small-colour barrier
  int it = 0;
  bool conv = false, nan = false;
  for (;;) {
    unsigned long long cmax = 0ull;
    unsigned long long* dxrec = it + 1 == max_iter ? m.dxmax : nullptr;
    for (int c = 0; c < e.ncolors; ++c) {
      const ColorInfo ci = m.color[e.cbase + c];
      const bool small = is_small(ci.chunk_end - ci.chunk_begin);
      const int span = small ? nsb : nb;  // blocks that take this colour
      const unsigned long long phase = (unsigned long long)it * e.ncolors + c;
      // the first colour follows the end-of-sweep grid barrier
      if (scoped && c > 0 &&
          !wait_neighbours(nbr, blockIdx.x * e.ncolors + c, phase, ctl, lim)) {
        if (threadIdx.x == 0) atomicOr(m.status, kStatTimeout);
        return;
      }
      if (small) {
        if (blockIdx.x < span)
          for (int q = ci.chunk_begin + blockIdx.x; q < ci.chunk_end; q += span) {
            if (warp < W)
              process_chunk_part<Real, SReal, TPV, MAT, FMT>(m, e.vbase, ci, q, lane, state, stat,
                                                             tab, warp, W,
                                                             s_split + warp * kPartFloats);
            __syncthreads();
            if (warp == 0)
              finish_split_chunk<Real, SReal, TPV>(m, e.vbase, ci, q, lane, state, sc, cmax,
                                                   stat, dxrec, s_split, W);
            __syncthreads();  // s_split is rewritten by the next chunk
          }
      } else if (blockIdx.x < span) {
        for (int q = ci.chunk_begin + blockIdx.x * nwarps + warp; q < ci.chunk_end;
             q += span * nwarps)
          process_chunk<Real, SReal, TPV, MAT, FMT>(m, e.vbase, ci, q, lane, state, sc, cmax,
                                                    stat, tab, dxrec);
      }
      if (c + 1 == e.ncolors) break;
      if (scoped) {
        publish_epoch(nbr, phase + 1);
        continue;
      }
      const ColorInfo cn = m.color[e.cbase + c + 1];
      if (small && is_small(cn.chunk_end - cn.chunk_begin)) {
        // both colours ran on the small-colour blocks only: they meet among
        // themselves (block 0 alone: its writes are block-visible)
        if (nsb == 1) {
          __syncthreads();
        } else if (blockIdx.x < nsb) {
          sub_bar += nsb;
          if (!counter_sync(ctl, &ctl->sub_arrivals, sub_bar, lim, &s_ok)) {
            if (threadIdx.x == 0) atomicOr(m.status, kStatTimeout);
            return;
          }
        }
      } else {
        VBD_GRID_SYNC();
      }
    }
    // end of sweep: convergence test over the whole grid
    cmax = warp_max_u64(cmax);
    const unsigned wst = __reduce_or_sync(0xffffffffu, stat);
    if (lane == 0) {
      s_red[warp] = cmax;
      if (wst) atomicOr(&ctl->status, wst);
    }
    __syncthreads();
    if (warp == 0) {
      unsigned long long v = lane < nwarps ? s_red[lane] : 0ull;
      v = warp_max_u64(v);
      if (lane == 0 && v) atomicMax(&ctl->conv[it % 3], v);
    }
    VBD_GRID_SYNC();
    const unsigned long long v = ld_relaxed_u64(&ctl->conv[it % 3]);
    // the slot of two sweeps ago: every block read it before this barrier,
    // and it is next written after the following one
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->conv[(it + 2) % 3] = 0ull;
    ++it;
    nan = v > 0x7ff0000000000000ull;
    conv = !nan && __longlong_as_double((long long)v) < tol;
    if (conv || nan || it >= max_iter) break;
  }

  // end: velocity update
  for (int i = tid; i < e.nv; i += nthreads) end_vertex<SReal>(m, e.vbase + i, U[e.vbase + i], sc);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned st = ld_relaxed_u32(&ctl->status);
    if (nan) st |= kStatNonFinite;
    if (!conv) st |= kStatIterCap;
    m.iters[0] = it;
    atomicOr(m.status, st);
  }
#undef VBD_GRID_SYNC
}

cudaLaunchConfig_t persist_config(int blocks, int threads, size_t smem, cudaStream_t s,
                                  cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// The staged record table may exceed the default 48 KB of dynamic shared
// memory: raise the kernel's limit once per device.
template <typename Real, typename SReal, int TPV, int MAT, int FMT>
cudaError_t configure() {
  static int configured_device = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured_device == dev) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(persist_kernel<Real, SReal, TPV, MAT, FMT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kPersistMaxTabSmem);
  if (e == cudaSuccess) configured_device = dev;
  return e;
}

struct PersistLaunch {
  int blocks, threads;
  const DevMesh& m;
  const StepParams* p;
  PersistCtl* ctl;
  PersistLimits lim;
  double* parts;
  size_t smem;
  cudaStream_t s;
  PersistNbr nbr;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    cudaError_t e = configure<Real, SReal, TPV, MAT, FMT>();
    if (e != cudaSuccess) return e;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = persist_config(blocks, threads, smem, s, attr);
    return cudaLaunchKernelEx(&cfg, persist_kernel<Real, SReal, TPV, MAT, FMT>, m, p, ctl, lim,
                              parts, nbr);
  }
};

struct PersistOccupancy {
  int threads;
  size_t smem;
  int* out;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    cudaError_t e = configure<Real, SReal, TPV, MAT, FMT>();
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        out, persist_kernel<Real, SReal, TPV, MAT, FMT>, threads, smem);
  }
};

}  // namespace

cudaError_t persist_occupancy(int prec, int material, int fmt, int tpv, int threads, size_t smem,
                              int* blocks_per_sm) {
  if (threads < 32 || threads > 512 || threads % 32) return cudaErrorInvalidValue;
  PersistOccupancy f{threads, smem, blocks_per_sm};
  return dispatch(prec, material, fmt, tpv, f);
}

cudaError_t launch_persist(int prec, int material, int tpv, int threads, const DevMesh& m,
                           const StepParams* p, PersistCtl* ctl, int blocks,
                           const PersistLimits& lim, double* parts, size_t smem,
                           const PersistNbr& nbr, cudaStream_t s) {
  if (threads < 32 || threads > 512 || threads % 32 || blocks < 1) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(PersistCtl), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(m.status, 0, sizeof(unsigned), s);
  if (e == cudaSuccess && nbr.epoch)
    e = cudaMemsetAsync(nbr.epoch, 0, sizeof(unsigned long long) * kEpochStride * blocks, s);
  if (e != cudaSuccess) return e;
  if (smem > (size_t)kPersistMaxTabSmem) return cudaErrorInvalidValue;
  PersistLaunch f{blocks, threads, m, p, ctl, lim, parts, smem, s, nbr};
  return dispatch(prec, material, m.fmt, tpv, f);
}

}  // namespace vbd
