// Host-side launchers of the solver kernels (defined in vbd_kernels.cu).
//
// prec: 0 = fp32 state and arithmetic, 1 = fp64 state with fp32 arithmetic
// ("mixed"), 2 = fp64 throughout.  state64 = the state arrays hold double4.
#pragma once
#include <cuda_runtime.h>

#include "vbd_internal.h"

namespace vbd {

// Largest dynamic shared memory a block-mode step may use (bytes).
int env_kernel_max_smem();

// Block mode: work[b] = (environment, rank, group size) for block b; an
// environment runs begin, all sweeps and end on one block, or on all blocks
// of one cluster (group size = cluster).  n_blocks must be a multiple of
// cluster (padding blocks carry environment -1).
cudaError_t launch_env_step(int prec, int material, int tpv, int threads, const DevMesh& m,
                            const StepParams& p, const double* tol_env, const int4* work,
                            int n_blocks, int cluster, size_t smem_bytes, cudaStream_t s);
// Resident env_step blocks per SM (cluster == 1) or resident clusters on the
// device (cluster > 1) for this launch shape.
cudaError_t env_occupancy(int prec, int material, int fmt, int tpv, int threads, size_t smem,
                          int cluster, int* out);

// Grid mode building blocks (single environment).
cudaError_t launch_begin(bool state64, const DevMesh& m, const StepParams* p, LoopControl* ctl,
                         cudaStream_t s);
cudaError_t launch_color(int prec, int material, int tpv, int threads, const DevMesh& m,
                         int color, int n_chunks, const StepParams* p, LoopControl* ctl,
                         cudaStream_t s);
// use_handle != 0: the check clears `handle` (a CUDA-graph while node) when
// the loop must stop; otherwise it only records the state in *ctl.
cudaError_t launch_check(LoopControl* ctl, const StepParams* p, unsigned long long handle,
                         int use_handle, cudaStream_t s);
cudaError_t launch_end(bool state64, const DevMesh& m, const StepParams* p, LoopControl* ctl,
                       cudaStream_t s);

// Position / velocity exchange in the caller's vertex order (float64).
// offset = rest positions (added on gather, subtracted on scatter) or NULL.
cudaError_t launch_gather(bool state64, const double* offset, const int* new_of_old,
                          const void* state, double* out, int n, cudaStream_t s);
cudaError_t launch_scatter(bool state64, const double* offset, const int* new_of_old,
                           const double* in, void* state, int n, cudaStream_t s);
// Incremental potential of every environment at the renumbered displacements
// x (Real4 in the state precision) for a step with the parameters p from the
// current state; out: device double [n_env].
cudaError_t launch_potential(int prec, int material, const DevMesh& m, const StepParams& p,
                             const void* x, double* out, cudaStream_t s);
// Sets the xyz of every state vector to zero, keeping w.
cudaError_t launch_zero_xyz(bool state64, void* state, int n, cudaStream_t s);

}  // namespace vbd
