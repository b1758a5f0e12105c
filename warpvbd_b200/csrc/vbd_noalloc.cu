// vbd_step_noalloc: a VBD time step that allocates no memory.
//
// Who needs it: callers that must not allocate GPU memory while they step a
// solver -- an application that reserves its whole device-memory budget at
// start-up (so a later cudaMalloc, or the graph instantiation the graph-mode
// vbd_step performs on its first call, may fail or is forbidden), or a
// real-time control loop whose per-step code may not call an allocator.
// Those callers create the solver once at start-up and then call this entry
// point, which calls no cudaMalloc, cudaFree, graph instantiation or other
// allocating routine.
//
// It runs the same per-colour sweep as the grid-mode step (process_chunk of
// vbd_kernels.cu), driven by the host one sweep at a time.  The scratch the
// sweep needs -- the step parameters, the loop control and one convergence
// partial per thread block -- lives in the file-scope array g_noalloc_scratch
// below instead of in the solver's own buffers.  Every GPU that loads the
// library holds this array (about 128 KiB) until the process exits.  Every
// call shares it and it keeps the last call's contents: the step resets the
// loop control itself, and each sweep overwrites the partials it reads.  Two
// calls whose work overlaps on the GPU (two streams, or two host threads)
// race on the array, so such calls must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/vbd_b200.h"
#include "vbd_device.cuh"
#include "vbd_internal.h"
#include "vbd_launch.h"
#include "vbd_noalloc.h"

namespace vbd {

// 16 control / parameter words + 16384 partials = 131,200 bytes per GPU
constexpr int kNoAllocMaxPartials = 16384;
constexpr int kNoAllocWords = kNoAllocPartialOffset + kNoAllocMaxPartials;
static_assert(sizeof(LoopControl) <= 8 * (kNoAllocParamOffset - kNoAllocCtlOffset), "ctl");
static_assert(sizeof(StepParams) <= 8 * (kNoAllocPartialOffset - kNoAllocParamOffset), "params");

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

int noalloc_max_partials() { return kNoAllocMaxPartials; }

// Colour sweep writing its block maximum to partial[blockIdx.x] instead of an
// atomic on the solver's loop-control word.
template <typename Real, typename SReal, int TPV, int MAT, int FMT>
__global__ void __launch_bounds__(256) noalloc_color_kernel(DevMesh m, int color,
                                                            const StepParams* __restrict__ pp,
                                                            LoopControl* ctl,
                                                            unsigned long long* partial) {
  using S4 = real4<SReal>;
  __shared__ unsigned long long s_red[8];
  const StepConst sc = make_const(*pp);
  const ColorInfo ci = m.color[color];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = ci.chunk_begin + blockIdx.x * (blockDim.x >> 5) + warp;
  unsigned long long cmax = 0ull;
  unsigned stat = 0u;
  const GlobalState<SReal> state{reinterpret_cast<S4*>(m.u)};
  unsigned long long* dxrec = ctl->iter + 1 == pp->max_iter ? m.dxmax : nullptr;
  if (q < ci.chunk_end)
    process_chunk<Real, SReal, TPV, MAT, FMT>(m, 0, ci, q, lane, state, sc, cmax, stat,
                                              reinterpret_cast<const real4<Real>*>(m.rec_tab),
                                              dxrec);
  cmax = warp_max_u64(cmax);
  const unsigned st = __reduce_or_sync(0xffffffffu, stat);
  if (lane == 0) {
    s_red[warp] = cmax;
    if (st) atomicOr(&ctl->status, st);
  }
  __syncthreads();
  if (warp == 0) {
    unsigned long long v = lane < (int)(blockDim.x >> 5) ? s_red[lane] : 0ull;
    v = warp_max_u64(v);
    if (lane == 0) partial[blockIdx.x] = v;
  }
}

// Reduces the sweep's partials into ctl->conv_bits; check_kernel then applies
// the stopping rule.
__global__ void __launch_bounds__(256) noalloc_reduce_kernel(const unsigned long long* partial,
                                                             int n, LoopControl* ctl) {
  __shared__ unsigned long long s_red[8];
  unsigned long long v = 0ull;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v = partial[i] > v ? partial[i] : v;
  v = warp_max_u64(v);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned long long w = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0ull;
    w = warp_max_u64(w);
    if (threadIdx.x == 0) ctl->conv_bits = w;
  }
}

namespace {

struct NoAllocColorLaunch {
  int blocks;
  const DevMesh& m;
  int color;
  const StepParams* p;
  LoopControl* ctl;
  unsigned long long* partial;
  cudaStream_t s;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    noalloc_color_kernel<Real, SReal, TPV, MAT, FMT><<<blocks, 256, 0, s>>>(m, color, p, ctl,
                                                                             partial);
    return cudaGetLastError();
  }
};

}  // namespace

cudaError_t launch_noalloc_color(int prec, int material, int tpv, const DevMesh& m, int color,
                                 int blocks, const StepParams* p, LoopControl* ctl,
                                 unsigned long long* partial, cudaStream_t s) {
  if (blocks == 0) return cudaSuccess;
  NoAllocColorLaunch f{blocks, m, color, p, ctl, partial, s};
  return dispatch(prec, material, m.fmt, tpv, f);
}

cudaError_t launch_noalloc_reduce(const unsigned long long* partial, int n, LoopControl* ctl,
                                  cudaStream_t s) {
  noalloc_reduce_kernel<<<1, 256, 0, s>>>(partial, n, ctl);
  return cudaGetLastError();
}

// Device address of g_noalloc_scratch on the current device.  The symbol's
// name in host code is only a host-side handle, so it is resolved once per
// device with cudaGetSymbolAddress (the first call on a device does this and
// should therefore come before any stream capture).
cudaError_t noalloc_scratch_address(unsigned long long** out) {
  static std::mutex mu;
  static unsigned long long* addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    addr[dev] = static_cast<unsigned long long*>(p);
  }
  *out = addr[dev];
  return cudaSuccess;
}

}  // namespace vbd
