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
// Forward pass (fp32, one thread per sample), for evaluation: X [n][24] ->
// out [n][3].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ X, int n,
                                                          const float* __restrict__ P,
                                                          float* __restrict__ out) {
  __shared__ float W[kWsParams];
  for (int i = threadIdx.x; i < kWsParams; i += blockDim.x) W[i] = P[i];
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const float* x = X + (size_t)b * kWsRow;
  float h1[kWsHidden];
#pragma unroll
  for (int j = 0; j < kWsHidden; ++j) {
    float a = W[kWsB1 + j];
#pragma unroll
    for (int i = 0; i < kWsIn; ++i) a += W[kWsW1 + j * kWsIn + i] * x[i];
    h1[j] = silu(a);
  }
  float o[kWsOut] = {W[kWsB3], W[kWsB3 + 1], W[kWsB3 + 2]};
  for (int j = 0; j < kWsHidden; ++j) {
    float a = W[kWsB2 + j];
#pragma unroll
    for (int i = 0; i < kWsHidden; ++i) a += W[kWsW2 + j * kWsHidden + i] * h1[i];
    const float s = silu(a);
    for (int k = 0; k < kWsOut; ++k) o[k] += W[kWsW3 + k * kWsHidden + j] * s;
  }
  for (int k = 0; k < kWsOut; ++k) out[(size_t)b * kWsOut + k] = o[k];
}

// ---------------------------------------------------------------------------
// Training step, fused per tile of kTrainTile samples (one block): forward
// with the activations kept in shared memory, the loss gradient, backward to
// the pre-activation deltas, and the tile's partial weight gradients -- each
// parameter's sum over the tile's samples.  A second kernel adds the tiles'
// partials in tile order, so the gradient is the same on every run (no
// atomics).  Mapping: thread t handles column (hidden unit) t % 64 for the
// samples t / 64, t / 64 + 4, ...; weights are staged in shared memory, W1
// and W2 transposed for the forward pass so that consecutive threads read
// consecutive words.
// ---------------------------------------------------------------------------
constexpr int kTrainTile = 32;
constexpr int kTrainThreads = 256;
constexpr int kTrainPartial = kWsParams + 1;  // + the tile's sum of squared errors
// shared-memory map (floats)
constexpr int kTsW = 0;                                   // params as stored
constexpr int kTsW1T = kTsW + kWsParams;                  // W1^T [22][64]
constexpr int kTsW2T = kTsW1T + kWsIn * kWsHidden;        // W2^T [64][64]
constexpr int kTsX = kTsW2T + kWsHidden * kWsHidden;      // X [tile][22]
constexpr int kTsS1 = kTsX + kTrainTile * kWsIn;          // silu(A1) [tile][64]
constexpr int kTsG1 = kTsS1 + kTrainTile * kWsHidden;     // silu'(A1)
constexpr int kTsS2 = kTsG1 + kTrainTile * kWsHidden;     // silu(A2)
constexpr int kTsG2 = kTsS2 + kTrainTile * kWsHidden;     // silu'(A2)
constexpr int kTsD1 = kTsG2 + kTrainTile * kWsHidden;     // dL/dA1
constexpr int kTsD2 = kTsD1 + kTrainTile * kWsHidden;     // dL/dA2
constexpr int kTsOut = kTsD2 + kTrainTile * kWsHidden;    // dL/dout [tile][3]
constexpr int kTsSse = kTsOut + kTrainTile * kWsOut;      // per-warp squared errors
constexpr int kTsFloats = kTsSse + kTrainThreads / 32;
constexpr size_t kTrainSmem = sizeof(float) * kTsFloats;

__global__ void __launch_bounds__(kTrainThreads) mlp_train_tile_kernel(
    const float* __restrict__ X, const float* __restrict__ Y, const int* __restrict__ idx,
    int batch, const float* __restrict__ P, float* __restrict__ out) {
  extern __shared__ __align__(16) float ts[];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int s0 = blockIdx.x * kTrainTile;
  const int ns = min(kTrainTile, batch - s0);
  for (int i = t; i < kWsParams; i += kTrainThreads) ts[kTsW + i] = P[i];
  for (int i = t; i < kWsHidden * kWsIn; i += kTrainThreads) {
    const int j = i / kWsIn, k = i % kWsIn;
    ts[kTsW1T + k * kWsHidden + j] = P[kWsW1 + i];
  }
  for (int i = t; i < kWsHidden * kWsHidden; i += kTrainThreads) {
    const int j = i / kWsHidden, k = i % kWsHidden;
    ts[kTsW2T + k * kWsHidden + j] = P[kWsW2 + i];
  }
  for (int i = t; i < kTrainTile * kWsIn; i += kTrainThreads) {
    const int s = i / kWsIn, k = i % kWsIn;
    float v = 0.0f;
    if (s < ns) {
      const int r = idx ? idx[s0 + s] : s0 + s;
      v = X[(size_t)r * kWsRow + k];
    }
    ts[kTsX + i] = v;
  }
  __syncthreads();
  const int j = t & (kWsHidden - 1), sg = t / kWsHidden, sstride = kTrainThreads / kWsHidden;
  // layer 1
  for (int s = sg; s < kTrainTile; s += sstride) {
    float a = ts[kTsW + kWsB1 + j];
#pragma unroll
    for (int k = 0; k < kWsIn; ++k) a += ts[kTsW1T + k * kWsHidden + j] * ts[kTsX + s * kWsIn + k];
    ts[kTsS1 + s * kWsHidden + j] = silu(a);
    ts[kTsG1 + s * kWsHidden + j] = silu_grad(a);
  }
  __syncthreads();
  // layer 2
  for (int s = sg; s < kTrainTile; s += sstride) {
    float a = ts[kTsW + kWsB2 + j];
#pragma unroll 16
    for (int k = 0; k < kWsHidden; ++k)
      a += ts[kTsW2T + k * kWsHidden + j] * ts[kTsS1 + s * kWsHidden + k];
    ts[kTsS2 + s * kWsHidden + j] = silu(a);
    ts[kTsG2 + s * kWsHidden + j] = silu_grad(a);
  }
  __syncthreads();
  // layer 3 and the loss gradient: one warp per (sample, output), two hidden
  // units per lane and a shuffle reduction
  float sse = 0.0f;
  for (int o = warp; o < kTrainTile * kWsOut; o += kTrainThreads / 32) {
    const int s = o / kWsOut, k = o % kWsOut;
    float a = ts[kTsW + kWsW3 + k * kWsHidden + lane] * ts[kTsS2 + s * kWsHidden + lane] +
              ts[kTsW + kWsW3 + k * kWsHidden + lane + 32] * ts[kTsS2 + s * kWsHidden + lane + 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    if (lane == 0) {
      float g = 0.0f;
      if (s < ns) {
        const int r = idx ? idx[s0 + s] : s0 + s;
        const float d = a + ts[kTsW + kWsB3 + k] - Y[(size_t)r * kWsOut + k];
        g = 2.0f * d / (kWsOut * batch);
        sse += d * d;
      }
      ts[kTsOut + o] = g;
    }
  }
  if (lane == 0) ts[kTsSse + warp] = sse;
  __syncthreads();
  // backward: layer-2 deltas, then layer-1 deltas
  for (int s = sg; s < kTrainTile; s += sstride) {
    float gh = 0.0f;
#pragma unroll
    for (int k = 0; k < kWsOut; ++k)
      gh += ts[kTsW + kWsW3 + k * kWsHidden + j] * ts[kTsOut + s * kWsOut + k];
    ts[kTsD2 + s * kWsHidden + j] = gh * ts[kTsG2 + s * kWsHidden + j];
  }
  __syncthreads();
  for (int s = sg; s < kTrainTile; s += sstride) {
    float gh = 0.0f;
#pragma unroll 16
    for (int k = 0; k < kWsHidden; ++k)
      gh += ts[kTsW + kWsW2 + k * kWsHidden + j] * ts[kTsD2 + s * kWsHidden + k];
    ts[kTsD1 + s * kWsHidden + j] = gh * ts[kTsG1 + s * kWsHidden + j];
  }
  __syncthreads();
  // the tile's weight gradients: each parameter summed over the tile's
  // samples (padding samples have zero deltas)
  float* dst = out + (size_t)blockIdx.x * kTrainPartial;
  for (int p = t; p < kWsParams; p += kTrainThreads) {
    const float *a, *b;
    int sa, sb;
    if (p < kWsB1) {  // W1[j][i] += D1[s][j] X[s][i]
      a = ts + kTsD1 + p / kWsIn; sa = kWsHidden;
      b = ts + kTsX + p % kWsIn; sb = kWsIn;
    } else if (p < kWsW2) {  // b1[j]
      a = ts + kTsD1 + (p - kWsB1); sa = kWsHidden; b = nullptr; sb = 0;
    } else if (p < kWsB2) {  // W2[j][i] += D2[s][j] S1[s][i]
      a = ts + kTsD2 + (p - kWsW2) / kWsHidden; sa = kWsHidden;
      b = ts + kTsS1 + (p - kWsW2) % kWsHidden; sb = kWsHidden;
    } else if (p < kWsW3) {  // b2[j]
      a = ts + kTsD2 + (p - kWsB2); sa = kWsHidden; b = nullptr; sb = 0;
    } else if (p < kWsB3) {  // W3[k][j] += dout[s][k] S2[s][j]
      a = ts + kTsOut + (p - kWsW3) / kWsHidden; sa = kWsOut;
      b = ts + kTsS2 + (p - kWsW3) % kWsHidden; sb = kWsHidden;
    } else {  // b3[k]
      a = ts + kTsOut + (p - kWsB3); sa = kWsOut; b = nullptr; sb = 0;
    }
    float acc = 0.0f;
    if (b) {
#pragma unroll 8
      for (int s = 0; s < kTrainTile; ++s) acc += a[s * sa] * b[s * sb];
    } else {
#pragma unroll 8
      for (int s = 0; s < kTrainTile; ++s) acc += a[s * sa];
    }
    dst[p] = acc;
  }
  if (t == 0) {
    float v = 0.0f;
    for (int w = 0; w < kTrainThreads / 32; ++w) v += ts[kTsSse + w];
    dst[kWsParams] = v;
  }
}

// Sum of the tiles' partial gradients in tile order (and of their squared
// errors into *loss).
__global__ void mlp_reduce_tiles_kernel(const float* __restrict__ part, int tiles,
                                        float* __restrict__ grad, double* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kWsParams) return;
  if (p == kWsParams) {
    if (loss) {
      double v = 0.0;
      for (int b = 0; b < tiles; ++b) v += double(part[(size_t)b * kTrainPartial + p]);
      *loss += v;
    }
    return;
  }
  float acc = 0.0f;
  for (int b = 0; b < tiles; ++b) acc += part[(size_t)b * kTrainPartial + p];
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

size_t mlp_train_scratch_floats(int batch) {
  return (size_t)nblk(batch, kTrainTile) * kTrainPartial;
}

cudaError_t launch_mlp_train_batch(const float* X, const float* Y, const int* idx, int batch,
                                   const float* P, float* grad, float* scratch, double* loss,
                                   cudaStream_t s) {
  static bool attr_set = false;  // per process; the attribute is per function
  if (!attr_set) {
    const cudaError_t e = cudaFuncSetAttribute(
        mlp_train_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int tiles = nblk(batch, kTrainTile);
  mlp_train_tile_kernel<<<tiles, kTrainThreads, kTrainSmem, s>>>(X, Y, idx, batch, P, scratch);
  mlp_reduce_tiles_kernel<<<nblk(kTrainPartial, 256), 256, 0, s>>>(scratch, tiles, grad, loss);
  return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* X, int n, const float* P, float* out,
                               cudaStream_t s) {
  if (n > 0) mlp_forward_kernel<<<nblk(n, 128), 128, 0, s>>>(X, n, P, out);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* P, const float* G, float* M, float* V, int n, float lr,
                        float beta1, float beta2, float eps, int t, cudaStream_t s) {
  const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
  adam_kernel<<<nblk(n, 256), 256, 0, s>>>(P, G, M, V, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace vbd
