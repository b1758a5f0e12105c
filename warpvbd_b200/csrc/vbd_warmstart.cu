// Learned warm start: per-vertex features, the MLP that predicts each step's
// correction from the inertia guess, and the kernels that train it.
//
// Model (per solved vertex): 22 inputs -> 64 (SiLU) -> 64 (SiLU) -> 3.
// The output is the converged-minus-inertia displacement of the step divided
// by h s, with h the vertex's length scale and s the RMS of its
// displacement-type features (below): dividing by s makes the regression
// scale-free, so a network trained on large motions is equally accurate,
// relatively, on small ones.  Parameters (fp32, this order):
//   W1[64][22] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
// The network acts on normalised inputs and predicts normalised targets;
// inference (vbd_ws_tc.cu, tensor cores) applies the fp32 normalisation (mean
// and 1/std of every input, std and mean of every target) around bf16
// weights and activations with fp32 accumulation.  Training is fp32.
//
// Displacement-type features, divided by h and then by s = RMS of the 18:
//   0-2   inertia displacement of the coming step, v dt + g dt^2
//   3-5   previous-step displacement, v dt
//   6-8   1-ring mean of the neighbours' previous-step displacement minus the
//         vertex's own (neighbours counted once per incident tet)
//   9-11  1-ring mean of the neighbours' displacement from rest minus the
//         vertex's own (a discrete Laplacian of the displacement)
//   12-14 previous step's correction u - ut_prev (0 without history)
//   15-17 g dt^2
// Scale-free features:
//   18    log10(E dt^2 / (rho h^2)), the stiffness-to-inertia ratio
//   19    Poisson's ratio
//   20    valence / 20
//   21    log10(s)
// Row layout: 24 floats per vertex, 22 = s, 23 = 1 for a solved vertex.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>

#include "vbd_device.cuh"
#include "vbd_internal.h"
#include "vbd_warmstart.h"

namespace vbd {

__device__ __forceinline__ float silu(float a) { return a / (1.0f + expf(-a)); }
__device__ __forceinline__ float silu_grad(float a) {
  const float s = 1.0f / (1.0f + expf(-a));
  return s * (1.0f + a * (1.0f - s));
}

// ---------------------------------------------------------------------------
// Features: one warp per chunk, TPV lanes per vertex walk its slots.  The
// neighbour sums read a packed fp32 copy of every vertex's displacement and
// velocity (24 B instead of two 32 B double4 per neighbour visit, written
// once per step by ws_pack_kernel); the vertex's own values stay in the
// state precision.  fp32 differences of neighbouring displacements are far
// more accurate than the bf16 the network's inputs are rounded to.
// ---------------------------------------------------------------------------
template <typename SReal>
__global__ void ws_pack_kernel(DevMesh m, float4* __restrict__ pa, float2* __restrict__ pb) {
  using S4 = real4<SReal>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n_vertices) return;
  const S4 u = reinterpret_cast<const S4*>(m.u)[i];
  const S4 v = reinterpret_cast<const S4*>(m.vel)[i];
  pa[i] = make_float4(float(u.x), float(u.y), float(u.z), float(v.x));
  pb[i] = make_float2(float(v.y), float(v.z));
}

template <typename SReal, int TPV, int FMT>
__global__ void __launch_bounds__(256) ws_features_kernel(DevMesh m, int n_chunks, float dt,
                                                          float gx, float gy, float gz,
                                                          float log_dt2, int history,
                                                          const float4* __restrict__ pa,
                                                          const float2* __restrict__ pb,
                                                          float* __restrict__ feat) {
  using S4 = real4<SReal>;
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= n_chunks) return;  // whole warp
  const int2 own = m.chunk_owner[q];
  const ColorInfo ci = m.color[own.x];
  const int vbase = m.env[own.y].vbase;
  constexpr int CPW = 32 / TPV;
  const int vi = lane / TPV, sub = lane % TPV;
  const int gv = ci.vbegin + (q - ci.chunk_begin) * CPW + vi;
  const bool valid = gv < ci.vend;
  const S4* U = reinterpret_cast<const S4*>(m.u);
  const S4* VEL = reinterpret_cast<const S4*>(m.vel);
  const ChunkInfo ch = m.chunk[q];
  // the chunk's slot indices up to the prefetch depth first, as the sweep does
  using RS = RawSlot<FMT>;
  constexpr int PF = Prefetch<TPV>::steps;
  const size_t base = (size_t)ch.block * 32 + lane;
  typename RS::type sl[PF];
#pragma unroll
  for (int s = 0; s < PF; ++s)
    if (s < ch.steps) sl[s] = RS::load(m, base + (size_t)s * 32);
  int k = 0;
  S4 uo, vo;
  uo.x = uo.y = uo.z = uo.w = SReal(0);
  vo = uo;
  if (valid) {
    k = m.valence[gv];
    uo = U[gv];
    vo = VEL[gv];
  }
  float su[3] = {0.f, 0.f, 0.f}, sv[3] = {0.f, 0.f, 0.f};
  const float ux = float(uo.x), uy = float(uo.y), uz = float(uo.z);
  const float vx = float(vo.x), vy = float(vo.y), vz = float(vo.z);
  auto visit = [&](const int4& id) {
    const int nb[3] = {id.x, id.y, id.z};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float4 a = __ldg(pa + vbase + nb[j]);
      const float2 b = __ldg(pb + vbase + nb[j]);
      su[0] += a.x - ux;
      su[1] += a.y - uy;
      su[2] += a.z - uz;
      sv[0] += a.w - vx;
      sv[1] += b.x - vy;
      sv[2] += b.y - vz;
    }
  };
#pragma unroll
  for (int s = 0; s < PF; ++s)
    if (s < ch.steps && s * TPV + sub < k) visit(RS::unpack(sl[s]));
  for (int s = PF; s < ch.steps; ++s)
    if (s * TPV + sub < k) visit(load_slot<FMT>(m, base + (size_t)s * 32));
#pragma unroll
  for (int off = TPV / 2; off > 0; off >>= 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      su[i] += __shfl_xor_sync(0xffffffffu, su[i], off);
      sv[i] += __shfl_xor_sync(0xffffffffu, sv[i], off);
    }
  }
  if (!valid) return;
  // every lane of the vertex holds the sums now; each computes the row and
  // stores its share of the six 16-byte pieces
  const float4 ws = m.wstat[gv];
  const float ih = 1.0f / ws.x;
  const float icnt = 1.0f / float(3 * k);
  const S4 tp = reinterpret_cast<const S4*>(m.ut)[gv];  // the previous step's inertia target
  const float dt2 = dt * dt;
  const float g2[3] = {gx * dt2, gy * dt2, gz * dt2};
  const float v[3] = {vx, vy, vz};
  // the correction u - ut_prev is a difference of nearby values: take it in
  // the state precision before rounding
  const float up[3] = {float(uo.x - tp.x), float(uo.y - tp.y), float(uo.z - tp.z)};
  float r[kWsRow];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r[i] = (v[i] * dt + g2[i]) * ih;
    r[3 + i] = v[i] * dt * ih;
    r[6 + i] = sv[i] * icnt * dt * ih;
    r[9 + i] = su[i] * icnt * ih;
    r[12 + i] = history ? up[i] * ih : 0.0f;
    r[15 + i] = g2[i] * ih;
  }
  float ss = 0.0f;
#pragma unroll
  for (int i = 0; i < 18; ++i) ss += r[i] * r[i];
  const float sc = sqrtf(ss * (1.0f / 18.0f)) + 1e-30f;
  const float isc = 1.0f / sc;
#pragma unroll
  for (int i = 0; i < 18; ++i) r[i] *= isc;
  r[18] = ws.y + log_dt2;
  r[19] = ws.z;
  r[20] = ws.w;
  r[21] = log10f(sc);
  r[22] = sc;
  r[23] = 1.0f;
  float4* f = reinterpret_cast<float4*>(feat + (size_t)gv * kWsRow);
#pragma unroll
  for (int j = 0; j < kWsRow / 4; ++j)
    if (j % TPV == sub) f[j] = make_float4(r[4 * j], r[4 * j + 1], r[4 * j + 2], r[4 * j + 3]);
}

// Training target after a step: (u - ut) / (h s) for solved vertices.
template <typename SReal>
__global__ void ws_targets_kernel(DevMesh m, const float* __restrict__ feat,
                                  float* __restrict__ target) {
  using S4 = real4<SReal>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n_vertices) return;
  const S4 u = reinterpret_cast<const S4*>(m.u)[i];
  const S4 t = reinterpret_cast<const S4*>(m.ut)[i];
  const bool solved = feat[(size_t)i * kWsRow + 23] > 0.0f;
  const double ih = solved ? 1.0 / (double(m.wstat[i].x) * feat[(size_t)i * kWsRow + 22]) : 0.0;
  target[3 * (size_t)i] = solved ? float(double(u.x - t.x) * ih) : 0.0f;
  target[3 * (size_t)i + 1] = solved ? float(double(u.y - t.y) * ih) : 0.0f;
  target[3 * (size_t)i + 2] = solved ? float(double(u.z - t.z) * ih) : 0.0f;
}

// ---------------------------------------------------------------------------
// Training (fp32).  A minibatch is a list of row indices into X [N][24] and
// Y [N][3].  Per sample: forward keeping the pre-activations A1, A2; the loss
// gradient dOut = 2 (out - y) / (3 B); backward to the pre-activation
// gradients D1, D2.  Weight gradients reduce over the minibatch with one
// thread per parameter.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) mlp_forward_kernel(
    const float* __restrict__ X, const float* __restrict__ Y, const int* __restrict__ idx,
    int batch, const float* __restrict__ P, float* __restrict__ A1, float* __restrict__ A2,
    float* __restrict__ dout, double* __restrict__ loss, float* __restrict__ out_pred) {
  __shared__ float W[kWsParams];
  for (int i = threadIdx.x; i < kWsParams; i += blockDim.x) W[i] = P[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (b < batch) {
    const int r = idx ? idx[b] : b;
    const float* x = X + (size_t)r * kWsRow;
    float h1[kWsHidden];
#pragma unroll
    for (int j = 0; j < kWsHidden; ++j) {
      float a = W[kWsB1 + j];
#pragma unroll
      for (int i = 0; i < kWsIn; ++i) a += W[kWsW1 + j * kWsIn + i] * x[i];
      A1[(size_t)b * kWsHidden + j] = a;
      h1[j] = silu(a);
    }
    float o[kWsOut] = {W[kWsB3], W[kWsB3 + 1], W[kWsB3 + 2]};
    for (int j = 0; j < kWsHidden; ++j) {
      float a = W[kWsB2 + j];
#pragma unroll
      for (int i = 0; i < kWsHidden; ++i) a += W[kWsW2 + j * kWsHidden + i] * h1[i];
      A2[(size_t)b * kWsHidden + j] = a;
      const float s = silu(a);
      for (int k = 0; k < kWsOut; ++k) o[k] += W[kWsW3 + k * kWsHidden + j] * s;
    }
    for (int k = 0; k < kWsOut; ++k) {
      if (out_pred) out_pred[(size_t)b * kWsOut + k] = o[k];
      if (Y) {
        const float d = o[k] - Y[(size_t)r * kWsOut + k];
        dout[(size_t)b * kWsOut + k] = 2.0f * d / (kWsOut * batch);
        l += double(d) * d;
      }
    }
  }
  if (loss) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
  }
}

__global__ void __launch_bounds__(128) mlp_backward_kernel(int batch, const float* __restrict__ P,
                                                           const float* __restrict__ A1,
                                                           const float* __restrict__ A2,
                                                           const float* __restrict__ dout,
                                                           float* __restrict__ D1,
                                                           float* __restrict__ D2) {
  __shared__ float W[kWsParams];
  for (int i = threadIdx.x; i < kWsParams; i += blockDim.x) W[i] = P[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  float d2[kWsHidden];
  const float g0 = dout[(size_t)b * kWsOut], g1 = dout[(size_t)b * kWsOut + 1],
              g2 = dout[(size_t)b * kWsOut + 2];
#pragma unroll
  for (int j = 0; j < kWsHidden; ++j) {
    const float gh = W[kWsW3 + j] * g0 + W[kWsW3 + kWsHidden + j] * g1 +
                     W[kWsW3 + 2 * kWsHidden + j] * g2;
    d2[j] = gh * silu_grad(A2[(size_t)b * kWsHidden + j]);
    D2[(size_t)b * kWsHidden + j] = d2[j];
  }
  for (int i = 0; i < kWsHidden; ++i) {
    float gh = 0.0f;
#pragma unroll
    for (int j = 0; j < kWsHidden; ++j) gh += W[kWsW2 + j * kWsHidden + i] * d2[j];
    D1[(size_t)b * kWsHidden + i] = gh * silu_grad(A1[(size_t)b * kWsHidden + i]);
  }
}

// One thread per parameter: sum over the minibatch of its gradient terms.
__global__ void __launch_bounds__(256) mlp_wgrad_kernel(
    const float* __restrict__ X, const int* __restrict__ idx, int batch,
    const float* __restrict__ A1, const float* __restrict__ A2, const float* __restrict__ D1,
    const float* __restrict__ D2, const float* __restrict__ dout, float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kWsParams) return;
  float acc = 0.0f;
  if (p < kWsB1) {  // W1[j][i]
    const int j = p / kWsIn, i = p % kWsIn;
    for (int b = 0; b < batch; ++b) {
      const int r = idx ? idx[b] : b;
      acc += D1[(size_t)b * kWsHidden + j] * X[(size_t)r * kWsRow + i];
    }
  } else if (p < kWsW2) {  // b1[j]
    const int j = p - kWsB1;
    for (int b = 0; b < batch; ++b) acc += D1[(size_t)b * kWsHidden + j];
  } else if (p < kWsB2) {  // W2[j][i]
    const int j = (p - kWsW2) / kWsHidden, i = (p - kWsW2) % kWsHidden;
    for (int b = 0; b < batch; ++b)
      acc += D2[(size_t)b * kWsHidden + j] * silu(A1[(size_t)b * kWsHidden + i]);
  } else if (p < kWsW3) {  // b2[j]
    const int j = p - kWsB2;
    for (int b = 0; b < batch; ++b) acc += D2[(size_t)b * kWsHidden + j];
  } else if (p < kWsB3) {  // W3[k][j]
    const int k = (p - kWsW3) / kWsHidden, j = (p - kWsW3) % kWsHidden;
    for (int b = 0; b < batch; ++b)
      acc += dout[(size_t)b * kWsOut + k] * silu(A2[(size_t)b * kWsHidden + j]);
  } else {  // b3[k]
    const int k = p - kWsB3;
    for (int b = 0; b < batch; ++b) acc += dout[(size_t)b * kWsOut + k];
  }
  grad[p] = acc;
}

__global__ void adam_kernel(float* __restrict__ P, const float* __restrict__ G,
                            float* __restrict__ M, float* __restrict__ V, int n, float lr,
                            float beta1, float beta2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float m = beta1 * M[i] + (1.0f - beta1) * g;
  const float v = beta2 * V[i] + (1.0f - beta2) * g * g;
  M[i] = m;
  V[i] = v;
  P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void to_bf16_kernel(const float* __restrict__ P, __nv_bfloat16* __restrict__ out,
                               int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16(P[i]);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
namespace {
struct FeatLaunch {
  const DevMesh& m;
  int n_chunks;
  double dt, gx, gy, gz;
  int history;
  float* pack;
  float* feat;
  cudaStream_t s;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    const int blocks = (n_chunks + 7) / 8;
    if (blocks == 0) return cudaSuccess;
    float4* pa = reinterpret_cast<float4*>(pack);
    float2* pb = reinterpret_cast<float2*>(pack + 4 * (size_t)m.n_vertices);
    ws_pack_kernel<SReal><<<(m.n_vertices + 255) / 256, 256, 0, s>>>(m, pa, pb);
    ws_features_kernel<SReal, TPV, FMT><<<blocks, 256, 0, s>>>(
        m, n_chunks, float(dt), float(gx), float(gy), float(gz), float(2.0 * log10(dt)), history,
        pa, pb, feat);
    return cudaGetLastError();
  }
};
inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }
}  // namespace

cudaError_t launch_ws_features(int prec, int tpv, const DevMesh& m, int n_chunks, double dt,
                               const double* g, int history, float* pack, float* feat,
                               cudaStream_t s) {
  FeatLaunch f{m, n_chunks, dt, g[0], g[1], g[2], history, pack, feat, s};
  // the features depend on the state precision only; material is irrelevant
  return dispatch(prec, kSNH, m.fmt, tpv, f);
}

cudaError_t launch_ws_targets(bool state64, const DevMesh& m, const float* feat, float* target,
                              cudaStream_t s) {
  const int n = m.n_vertices;
  if (n <= 0) return cudaSuccess;
  if (state64)
    ws_targets_kernel<double><<<nblk(n, 256), 256, 0, s>>>(m, feat, target);
  else
    ws_targets_kernel<float><<<nblk(n, 256), 256, 0, s>>>(m, feat, target);
  return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* P, void* out, int n, cudaStream_t s) {
  to_bf16_kernel<<<nblk(n, 256), 256, 0, s>>>(P, static_cast<__nv_bfloat16*>(out), n);
  return cudaGetLastError();
}

cudaError_t launch_mlp_train_batch(const float* X, const float* Y, const int* idx, int batch,
                                   const float* P, float* grad, float* scratch, double* loss,
                                   cudaStream_t s) {
  float* A1 = scratch;
  float* A2 = A1 + (size_t)batch * kWsHidden;
  float* D1 = A2 + (size_t)batch * kWsHidden;
  float* D2 = D1 + (size_t)batch * kWsHidden;
  float* dout = D2 + (size_t)batch * kWsHidden;
  mlp_forward_kernel<<<nblk(batch, 128), 128, 0, s>>>(X, Y, idx, batch, P, A1, A2, dout, loss,
                                                      nullptr);
  mlp_backward_kernel<<<nblk(batch, 128), 128, 0, s>>>(batch, P, A1, A2, dout, D1, D2);
  mlp_wgrad_kernel<<<nblk(kWsParams, 256), 256, 0, s>>>(X, idx, batch, A1, A2, D1, D2, dout,
                                                        grad);
  return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* X, int n, const float* P, float* out,
                               float* scratch, cudaStream_t s) {
  float* A1 = scratch;
  float* A2 = A1 + (size_t)n * kWsHidden;
  mlp_forward_kernel<<<nblk(n, 128), 128, 0, s>>>(X, nullptr, nullptr, n, P, A1, A2, nullptr,
                                                  nullptr, out);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* P, const float* G, float* M, float* V, int n, float lr,
                        float beta1, float beta2, float eps, int t, cudaStream_t s) {
  const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
  adam_kernel<<<nblk(n, 256), 256, 0, s>>>(P, G, M, V, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace vbd
