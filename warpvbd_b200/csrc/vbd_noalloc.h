// Host-side helpers of the allocation-free step (defined in vbd_noalloc.cu).
#pragma once
#include <cuda_runtime.h>

#include "vbd_internal.h"

namespace vbd {

// Layout of the static scratch in 8-byte words: loop control at word 0, step
// parameters at word 4, per-block convergence partials from word 16.
constexpr int kNoAllocCtlOffset = 0;
constexpr int kNoAllocParamOffset = 4;
constexpr int kNoAllocPartialOffset = 16;

// Number of per-block convergence partials the static scratch holds.
int noalloc_max_partials();
// Device address of the static scratch on the current device (resolved and
// cached on the first call per device).
cudaError_t noalloc_scratch_address(unsigned long long** out);
// One colour of a sweep; block b writes its convergence maximum to partial[b].
cudaError_t launch_noalloc_color(int prec, int material, int tpv, const DevMesh& m, int color,
                                 int blocks, const StepParams* p, LoopControl* ctl,
                                 unsigned long long* partial, cudaStream_t s);
// Max of partial[0, n) into ctl->conv_bits.
cudaError_t launch_noalloc_reduce(const unsigned long long* partial, int n, LoopControl* ctl,
                                  cudaStream_t s);

}  // namespace vbd
