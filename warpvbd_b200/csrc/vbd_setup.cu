// Mesh setup on the GPU: the reference's greedy vertex colouring
// (src/coloring.py:24-72, consumed by VBDSolver.__init__ at
// src/vbd_solver.py:470-483) computed in parallel, with the same result.
//
// The greedy pass visits vertices in index order and gives each the smallest
// colour not used by its already-coloured neighbours -- the neighbours of
// lower index (vertices share an edge when they share a tet).  So a vertex's
// colour is a function of its lower neighbours' colours only, and a vertex can
// be coloured as soon as all of them are: Jones-Plassmann rounds with the
// vertex index as the priority.  Each round, every uncoloured vertex whose
// lower neighbours all have a colour takes the smallest colour they leave
// free; the lowest uncoloured vertex is always ready, so every round makes
// progress, and the colours are exactly the sequential pass's.  The rounds
// needed are the longest index-decreasing path of the vertex graph: about
// 1.5 nx for an nx-long voxel beam (240 for 160x16x16), not the vertex count.
//
//   1. count     per tet, each of its 6 edges adds one entry to the list of
//                the higher vertex (duplicates across tets are harmless)
//   2. scan      exclusive sum of the counts (CUB) -> CSR offsets
//   3. fill      the lower vertex ids into the CSR lists
//   4. rounds    as above; colours are written once, read with volatile
//                loads (a value is -1 or final), so a vertex coloured earlier
//                in the same round may already be seen
//
// Vertices that lie in no tet have no lower neighbours and take colour 0, as
// in the reference (compute_adjacency_dict covers ids 0..max(tets)).
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "vbd_setup.h"

namespace vbd {

namespace {

constexpr int kMaxColors = 256;  // coloring.py:45 (MAX_COLORS)

__global__ void count_lower_kernel(const int32_t* __restrict__ tets, int T, int* __restrict__ cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const int4 e = reinterpret_cast<const int4*>(tets)[t];
  const int v[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = a + 1; b < 4; ++b)
      if (v[a] != v[b]) atomicAdd(cnt + max(v[a], v[b]), 1);
}

__global__ void fill_lower_kernel(const int32_t* __restrict__ tets, int T,
                                  const int* __restrict__ off, int* __restrict__ cursor,
                                  int* __restrict__ low) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const int4 e = reinterpret_cast<const int4*>(tets)[t];
  const int v[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = a + 1; b < 4; ++b)
      if (v[a] != v[b]) {
        const int hi = max(v[a], v[b]), lo = min(v[a], v[b]);
        low[off[hi] + atomicAdd(cursor + hi, 1)] = lo;
      }
}

__global__ void init_kernel(int* __restrict__ col, int nv) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) col[v] = -1;
}

// One round: every uncoloured vertex whose lower neighbours are all
// coloured takes the smallest colour they leave free.  `left` counts the
// vertices still uncoloured; `overflow` is set when a vertex would need a
// colour beyond the 256 the reference allows.
__global__ void __launch_bounds__(256) jp_round_kernel(const int* __restrict__ off,
                                                       const int* __restrict__ low, int nv,
                                                       int* col, int* left, int* overflow) {
  volatile int* vc = col;
  int done = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    if (vc[v] >= 0) continue;
    uint32_t used[kMaxColors / 32];
#pragma unroll
    for (int w = 0; w < kMaxColors / 32; ++w) used[w] = 0u;
    bool ready = true;
    for (int j = off[v]; j < off[v + 1]; ++j) {
      const int c = vc[low[j]];
      if (c < 0) {
        ready = false;
        break;
      }
      used[c >> 5] |= 1u << (c & 31);
    }
    if (!ready) continue;
    int c = kMaxColors;
#pragma unroll
    for (int w = kMaxColors / 32 - 1; w >= 0; --w)
      if (used[w] != 0xffffffffu) c = w * 32 + __ffs(~used[w]) - 1;
    if (c >= kMaxColors) {
      atomicExch(overflow, 1);
      c = 0;  // keeps the rounds finite; the result is refused
    }
    vc[v] = c;
    ++done;
  }
  if (done) atomicSub(left, done);
}

int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

int gpu_greedy_coloring(const int32_t* tets, int T, int nv, int32_t* coloring_out, int* rounds_out,
                        std::string* err) {
  auto cuda_fail = [&](cudaError_t e, const char* what) {
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
  };
  if (nv <= 0) return 0;
  cudaStream_t s = nullptr;
  int *d_tets = nullptr, *d_cnt = nullptr, *d_off = nullptr, *d_low = nullptr, *d_col = nullptr,
      *d_flags = nullptr;
  void* d_tmp = nullptr;
  int result = kSetupCudaError, rounds = 0;
  cudaError_t e = cudaSuccess;
  size_t tmp_bytes = 0;
  int h_flags[2] = {0, 0};
  const size_t tet_ints = 4 * (size_t)T;
  const int grid = std::min(nblk(nv, 256), 148 * 8);
  constexpr int kBatch = 16;  // rounds between reads of the remaining count
#define VBD_SETUP_TRY(call, what) \
  do {                            \
    e = (call);                   \
    if (e != cudaSuccess) {       \
      cuda_fail(e, what);         \
      goto done;                  \
    }                             \
  } while (0)
  VBD_SETUP_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  VBD_SETUP_TRY(cudaMalloc(&d_tets, sizeof(int) * std::max<size_t>(tet_ints, 4)), "alloc");
  VBD_SETUP_TRY(cudaMalloc(&d_cnt, sizeof(int) * (nv + 1)), "alloc");
  VBD_SETUP_TRY(cudaMalloc(&d_off, sizeof(int) * (nv + 1)), "alloc");
  VBD_SETUP_TRY(cudaMalloc(&d_col, sizeof(int) * nv), "alloc");
  VBD_SETUP_TRY(cudaMalloc(&d_flags, sizeof(int) * 2), "alloc");
  if (T > 0)
    VBD_SETUP_TRY(cudaMemcpyAsync(d_tets, tets, sizeof(int) * tet_ints, cudaMemcpyHostToDevice, s),
                  "upload");
  VBD_SETUP_TRY(cudaMemsetAsync(d_cnt, 0, sizeof(int) * (nv + 1), s), "memset");
  if (T > 0) count_lower_kernel<<<nblk(T, 256), 256, 0, s>>>(d_tets, T, d_cnt);
  VBD_SETUP_TRY(cudaGetLastError(), "count");
  // exclusive sum over nv + 1 entries: off[nv] = number of list entries
  VBD_SETUP_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_cnt, d_off, nv + 1, s), "scan");
  VBD_SETUP_TRY(cudaMalloc(&d_tmp, std::max<size_t>(tmp_bytes, 16)), "alloc");
  VBD_SETUP_TRY(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_cnt, d_off, nv + 1, s), "scan");
  VBD_SETUP_TRY(cudaMalloc(&d_low, sizeof(int) * std::max<size_t>(6 * (size_t)T, 1)), "alloc");
  VBD_SETUP_TRY(cudaMemsetAsync(d_cnt, 0, sizeof(int) * (nv + 1), s), "memset");
  if (T > 0) fill_lower_kernel<<<nblk(T, 256), 256, 0, s>>>(d_tets, T, d_off, d_cnt, d_low);
  VBD_SETUP_TRY(cudaGetLastError(), "fill");
  init_kernel<<<nblk(nv, 256), 256, 0, s>>>(d_col, nv);
  VBD_SETUP_TRY(cudaGetLastError(), "init");
  h_flags[0] = nv;
  VBD_SETUP_TRY(cudaMemcpyAsync(d_flags, h_flags, sizeof h_flags, cudaMemcpyHostToDevice, s),
                "upload");
  // every round colours at least the lowest uncoloured vertex: at most nv
  // rounds; the remaining count is read back every kBatch rounds
  for (;;) {
    for (int r = 0; r < kBatch; ++r)
      jp_round_kernel<<<grid, 256, 0, s>>>(d_off, d_low, nv, d_col, d_flags, d_flags + 1);
    rounds += kBatch;
    VBD_SETUP_TRY(cudaGetLastError(), "round");
    VBD_SETUP_TRY(cudaMemcpyAsync(h_flags, d_flags, sizeof h_flags, cudaMemcpyDeviceToHost, s),
                  "download");
    VBD_SETUP_TRY(cudaStreamSynchronize(s), "sync");
    if (h_flags[0] <= 0 || h_flags[1]) break;
    if (rounds > nv + kBatch) {
      if (err) *err = "colouring rounds made no progress";
      goto done;
    }
  }
  if (h_flags[1]) {
    result = kSetupTooManyColors;
    goto done;
  }
  VBD_SETUP_TRY(
      cudaMemcpyAsync(coloring_out, d_col, sizeof(int) * nv, cudaMemcpyDeviceToHost, s),
      "download");
  VBD_SETUP_TRY(cudaStreamSynchronize(s), "sync");
  result = 0;
  for (int v = 0; v < nv; ++v) result = std::max(result, coloring_out[v] + 1);
done:
#undef VBD_SETUP_TRY
  if (s) cudaStreamSynchronize(s);
  cudaFree(d_tets);
  cudaFree(d_cnt);
  cudaFree(d_off);
  cudaFree(d_low);
  cudaFree(d_col);
  cudaFree(d_flags);
  cudaFree(d_tmp);
  if (s) cudaStreamDestroy(s);
  if (rounds_out) *rounds_out = rounds;
  return result;
}

}  // namespace vbd
