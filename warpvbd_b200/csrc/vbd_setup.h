// Mesh setup on the GPU (vbd_setup.cu).
#pragma once
#include <cstdint>
#include <string>

namespace vbd {

constexpr int kSetupTooManyColors = -1;
constexpr int kSetupCudaError = -2;

// The reference's greedy colouring (vertices in index order, each the
// smallest colour its lower-indexed tet neighbours leave free), computed on
// the current device.  `tets` and `coloring_out` are host arrays (4 T and nv
// entries, nv > every vertex id).  Returns the colour count,
// kSetupTooManyColors (more than 256), or kSetupCudaError (`err` says why).
// `rounds_out` (optional): parallel rounds taken.
int gpu_greedy_coloring(const int32_t* tets, int T, int nv, int32_t* coloring_out, int* rounds_out,
                        std::string* err);

}  // namespace vbd
