// Learned warm start: network dimensions, parameter layout and launchers
// (kernels in vbd_warmstart.cu).
#pragma once
#include <cuda_runtime.h>

#include "vbd_internal.h"

namespace vbd {

constexpr int kWsIn = 22;      // network inputs per vertex
constexpr int kWsRow = 24;     // floats per feature row (22 = scale s, 23 = solved flag)
constexpr int kWsHidden = 64;  // width of both hidden layers
constexpr int kWsOut = 3;
// parameter offsets: W1[64][22] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
constexpr int kWsW1 = 0;
constexpr int kWsB1 = kWsW1 + kWsHidden * kWsIn;
constexpr int kWsW2 = kWsB1 + kWsHidden;
constexpr int kWsB2 = kWsW2 + kWsHidden * kWsHidden;
constexpr int kWsW3 = kWsB2 + kWsHidden;
constexpr int kWsB3 = kWsW3 + kWsOut * kWsHidden;
constexpr int kWsParams = kWsB3 + kWsOut;  // 5827
// normalisation: mean[22], 1/std[22] of the inputs, std[3], mean[3] of the targets
constexpr int kWsNorm = 2 * kWsIn + 2 * kWsOut;  // 50

// `pack`: scratch of 6 floats per vertex (the packed fp32 displacement and
// velocity the neighbour sums read, rewritten by every call).
cudaError_t launch_ws_features(int prec, int tpv, const DevMesh& m, int n_chunks, double dt,
                               const double* g, int history, float* pack, float* feat,
                               cudaStream_t s);
cudaError_t launch_ws_targets(bool state64, const DevMesh& m, const float* feat, float* target,
                              cudaStream_t s);
// tensor-core inference (vbd_ws_tc.cu); *err is OR-ed with 1 if a wait ran out
cudaError_t launch_ws_infer(const float* feat, int n, const void* wbf, const float* norm,
                            const float4* wstat, float4* pred, unsigned* err, cudaStream_t s);
cudaError_t launch_to_bf16(const float* P, void* out, int n, cudaStream_t s);
cudaError_t launch_mlp_train_batch(const float* X, const float* Y, const int* idx, int batch,
                                   const float* P, float* grad, float* scratch, double* loss,
                                   cudaStream_t s);
// floats of training scratch for a minibatch: one partial gradient (and sum
// of squared errors) per 32-sample tile
size_t mlp_train_scratch_floats(int batch);
cudaError_t launch_mlp_forward(const float* X, int n, const float* P, float* out, cudaStream_t s);
cudaError_t launch_adam(float* P, const float* G, float* M, float* V, int n, float lr,
                        float beta1, float beta2, float eps, int t, cudaStream_t s);

}  // namespace vbd
