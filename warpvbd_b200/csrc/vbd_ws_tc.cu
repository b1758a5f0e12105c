// Learned warm start: inference of the per-vertex MLP on the 5th-generation
// tensor cores (tcgen05), 128 vertices per tile.
//
//   layer 1   A1 [128 x 32] bf16 (22 normalised inputs, zero padded)
//             x W1^T [32 x 64] bf16  -> D1 [128 x 64] fp32 in TMEM columns 0-63
//   epilogue  tcgen05.ld D1, + b1, SiLU, bf16 -> A2 [128 x 64] in shared memory
//   layer 2   A2 x W2^T [64 x 64]    -> D2 [128 x 64] fp32 in TMEM columns 64-127
//   epilogue  tcgen05.ld D2, + b2, SiLU, layer 3 (64 -> 3) in registers,
//             de-normalisation, prediction = output * h * s
//
// One CTA = 4 warps = 128 threads; thread t owns vertex row t of the tile
// (TMEM lane t: warp w reads lanes 32w..32w+31).  The weight tiles are
// staged once per CTA; the CTA then walks tiles grid-stride.  One elected
// thread issues the MMAs and commits them to an mbarrier that every thread
// waits on (bounded: a wait that runs out sets the error word, the CTA
// stops, waits once more with a bound for its MMAs, frees its TMEM and
// returns; rows it did not finish get no prediction, so the step falls back
// to the inertia guess).
//
// Shared-memory operand layout (no swizzle, K-major canonical form of the
// UMMA descriptors): a [R x K] bf16 tile is stored as K/8 slabs of R rows
// x 16 bytes; inside a slab, rows of 8 form 128-byte core matrices.
//   byte offset (r, k) = (k / 8) * 16R + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// so for one K=16 step the two 8-column halves are 16R bytes apart (leading
// byte offset) and consecutive 8-row groups 128 bytes apart (stride byte
// offset).
//
// TMEM: 128 columns per CTA.  The dynamic shared memory request (48 KB, plus
// the 1 KB the driver reserves per CTA) lets at most 4 CTAs share an SM, so
// the 512 TMEM columns of an SM always suffice and tcgen05.alloc never waits.
//
// Each thread prefetches its row of the CTA's next tile into registers while
// the current tile's two MMA rounds run, so the feature loads (the kernel's
// only HBM traffic besides the predictions) overlap the tensor-core work.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "vbd_warmstart.h"

namespace vbd {

namespace {

constexpr int kTileM = 128;
constexpr int kK1 = 32;  // layer-1 K, kWsIn padded to a multiple of 16
constexpr int kTmemCols = 128;
// shared-memory map (bytes)
constexpr int kOffW1 = 0;                                // 64 x 32 bf16
constexpr int kOffW2 = kOffW1 + kWsHidden * kK1 * 2;     // 64 x 64 bf16
constexpr int kOffA1 = kOffW2 + kWsHidden * kWsHidden * 2;  // 128 x 32 bf16
constexpr int kOffA2 = kOffA1 + kTileM * kK1 * 2;           // 128 x 64 bf16
constexpr int kOffF = kOffA2 + kTileM * kWsHidden * 2;      // fp32 constants
constexpr int kNF = 64 + 64 + 3 * 64 + 4 + kWsNorm + 2;     // b1 b2 W3 b3 norm (padded)
constexpr int kOffBar = (kOffF + kNF * 4 + 15) / 16 * 16;   // mbarrier (8 B) + TMEM address
constexpr int kSmemUsed = kOffBar + 16;
constexpr int kSmemRequest = 48 * 1024;  // caps residency at 4 CTAs per SM
constexpr int kCtasPerSm = 4;
static_assert(kSmemUsed <= kSmemRequest, "shared-memory map exceeds the request");
static_assert((kCtasPerSm + 1) * (kSmemRequest + 1024) > 228 * 1024,
              "the request must keep CTAs per SM <= 4 (TMEM: 4 x 128 columns)");
static_assert(kCtasPerSm * kTmemCols <= 512, "TMEM columns per SM");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) of an R-row tile in the canonical layout
__device__ __forceinline__ int canon_off(int r, int k, int R) {
  return (k >> 3) * (16 * R) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// UMMA shared-memory descriptor: no swizzle, K-major; addresses in 16 B units
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for this architecture
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor, kind::f16: bf16 x bf16 -> fp32, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4)                       // D format: fp32
         | (1u << 7)                     // A format: bf16
         | (1u << 10)                    // B format: bf16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait on phase `parity` of the mbarrier
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int max_polls) {
  for (int n = 0; n < max_polls; ++n)
    if (mbar_try(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 64 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float* v) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
      "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
      "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
        "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]),
        "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]),
        "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]),
        "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
        "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]),
        "=r"(r[62]), "=r"(r[63])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// SiLU from the identity x sigma(x) = x/2 (1 + tanh(x/2)), with the
// hardware tanh approximation (PTX tanh.approx.f32, one special-function
// operation instead of an exponential and a reciprocal); its error, ~2^-11
// relative, is below the bf16 rounding the activations get next.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu_f(float a) {
  const float h = 0.5f * a;
  return fmaf(h, tanh_approx(h), h);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&p);
}

// eight consecutive k of row r of a canonical tile, as one 16-byte store
__device__ __forceinline__ void store8(unsigned char* tile, int R, int r, int k0, const float* v) {
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + canon_off(r, k0, R)) = q;
}

__global__ void __launch_bounds__(128, kCtasPerSm) ws_infer_tc_kernel(const float* __restrict__ feat, int n,
                                                          const __nv_bfloat16* __restrict__ wbf,
                                                          const float* __restrict__ norm,
                                                          const float4* __restrict__ wstat,
                                                          float4* __restrict__ pred,
                                                          unsigned* __restrict__ err,
                                                          int max_polls) {
  extern __shared__ __align__(1024) unsigned char smem[];
  float* F = reinterpret_cast<float*>(smem + kOffF);
  float* sB1 = F;
  float* sB2 = sB1 + 64;
  float* sW3 = sB2 + 64;
  float* sB3 = sW3 + 3 * 64;
  float* sN = sB3 + 4;
  uint64_t* bar_p = reinterpret_cast<uint64_t*>(smem + kOffBar);
  uint32_t* taddr_p = reinterpret_cast<uint32_t*>(smem + kOffBar + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t bar = smem_u32(bar_p);

  // TMEM (warp 0 allocates and later frees) and the mbarrier
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(taddr_p)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights: W1 zero-padded to K = 32, W2; fp32 biases, W3, normalisation
  for (int i = tid; i < kWsHidden * kK1; i += blockDim.x) {
    const int r = i / kK1, k = i % kK1;
    const __nv_bfloat16 w = k < kWsIn ? wbf[kWsW1 + r * kWsIn + k] : __float2bfloat16(0.0f);
    *reinterpret_cast<__nv_bfloat16*>(smem + kOffW1 + canon_off(r, k, kWsHidden)) = w;
  }
  for (int i = tid; i < kWsHidden * kWsHidden; i += blockDim.x) {
    const int r = i / kWsHidden, k = i % kWsHidden;
    *reinterpret_cast<__nv_bfloat16*>(smem + kOffW2 + canon_off(r, k, kWsHidden)) =
        wbf[kWsW2 + r * kWsHidden + k];
  }
  for (int i = tid; i < 64; i += blockDim.x) {
    sB1[i] = __bfloat162float(wbf[kWsB1 + i]);
    sB2[i] = __bfloat162float(wbf[kWsB2 + i]);
  }
  for (int i = tid; i < 3 * 64; i += blockDim.x) sW3[i] = __bfloat162float(wbf[kWsW3 + i]);
  if (tid < 3) sB3[tid] = __bfloat162float(wbf[kWsB3 + tid]);
  for (int i = tid; i < kWsNorm; i += blockDim.x) sN[i] = norm[i];
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_p;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  constexpr uint32_t idesc = instr_desc(kTileM, kWsHidden);
  const uint32_t a1 = smem_u32(smem + kOffA1), a2 = smem_u32(smem + kOffA2);
  const uint32_t w1 = smem_u32(smem + kOffW1), w2 = smem_u32(smem + kOffW2);
  unsigned char* A1 = smem + kOffA1;
  unsigned char* A2 = smem + kOffA2;
  const float* sy = sN + 2 * kWsIn;
  const float* my = sy + kWsOut;
  uint32_t phase = 0;
  bool ok = true;

  const int tiles = (n + kTileM - 1) / kTileM;
  // this thread's feature row of a tile (zeros past the end)
  auto load_row = [&](int tile, float4* r) {
    const int v = tile * kTileM + tid;
    if (tile < tiles && v < n) {
      const float4* f4 = reinterpret_cast<const float4*>(feat + (size_t)v * kWsRow);
#pragma unroll
      for (int q = 0; q < kWsRow / 4; ++q) r[q] = __ldg(f4 + q);
    } else {
#pragma unroll
      for (int q = 0; q < kWsRow / 4; ++q) r[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  float4 row[kWsRow / 4];
  load_row(blockIdx.x, row);
  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const int v = tile * kTileM + tid;
    const bool in = v < n;
    const float f22 = row[5].z, f23 = row[5].w;
    {
      // this thread's row of A1: normalised inputs in bf16, zero padded
      const float* f = reinterpret_cast<const float*>(row);
      float x[kK1];
#pragma unroll
      for (int i = 0; i < kK1; ++i) x[i] = 0.0f;
      if (in && f23 > 0.0f) {
#pragma unroll
        for (int i = 0; i < kWsIn; ++i) x[i] = (f[i] - sN[i]) * sN[kWsIn + i];
      }
#pragma unroll
      for (int k0 = 0; k0 < kK1; k0 += 8) store8(A1, kTileM, tid, k0, x + k0);
    }
    // the next tile's row, in flight during this tile's MMAs
    load_row(tile + gridDim.x, row);
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
#pragma unroll
      for (int j = 0; j < kK1 / 16; ++j)
        mma_bf16(tmem, smem_desc(a1 + j * 2 * 16 * kTileM, 16 * kTileM, 128),
                 smem_desc(w1 + j * 2 * 16 * kWsHidden, 16 * kWsHidden, 128), idesc, j > 0);
      mma_commit(bar);
    }
    // the decision is block-uniform, so no thread leaves while others wait
    ok = __syncthreads_and(mbar_wait(bar, phase, max_polls)) != 0;
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    {
      float h[64];
      tmem_ld64(lane_addr, h);
#pragma unroll
      for (int i = 0; i < 64; ++i) h[i] = silu_f(h[i] + sB1[i]);
#pragma unroll
      for (int k0 = 0; k0 < 64; k0 += 8) store8(A2, kTileM, tid, k0, h + k0);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
#pragma unroll
      for (int j = 0; j < kWsHidden / 16; ++j)
        mma_bf16(tmem + 64, smem_desc(a2 + j * 2 * 16 * kTileM, 16 * kTileM, 128),
                 smem_desc(w2 + j * 2 * 16 * kWsHidden, 16 * kWsHidden, 128), idesc, j > 0);
      mma_commit(bar);
    }
    // the decision is block-uniform, so no thread leaves while others wait
    ok = __syncthreads_and(mbar_wait(bar, phase, max_polls)) != 0;
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    {
      float h[64];
      tmem_ld64(lane_addr + 64, h);
      float o0 = sB3[0], o1 = sB3[1], o2 = sB3[2];
#pragma unroll
      for (int i = 0; i < 64; ++i) {
        const float s = silu_f(h[i] + sB2[i]);
        o0 += sW3[i] * s;
        o1 += sW3[64 + i] * s;
        o2 += sW3[128 + i] * s;
      }
      if (in) {
        if (f23 > 0.0f) {
          const float sc = wstat[v].x * f22;
          pred[v] = make_float4((o0 * sy[0] + my[0]) * sc, (o1 * sy[1] + my[1]) * sc,
                                (o2 * sy[2] + my[2]) * sc, 1.0f);
        } else {
          pred[v] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
    }
    // the next tile overwrites A1 / A2 and the accumulators: every thread's
    // TMEM reads are done before the next MMA is issued
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1u);
    // the MMAs this CTA committed may still be running: wait for them (again
    // bounded) before the accumulators are freed
    mbar_wait(bar, phase ^ 1u, max_polls);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

}  // namespace

cudaError_t launch_ws_infer(const float* feat, int n, const void* wbf, const float* norm,
                            const float4* wstat, float4* pred, unsigned* err, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  static int configured = -1;  // the attribute is per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured != dev) {
    cudaError_t e = cudaFuncSetAttribute(ws_infer_tc_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemRequest);
    // all of the SM's unified memory as shared memory, so that 4 CTAs fit
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ws_infer_tc_kernel,
                               cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    configured = dev;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = (n + kTileM - 1) / kTileM;
  const int grid = tiles < kCtasPerSm * sms ? tiles : kCtasPerSm * sms;
  ws_infer_tc_kernel<<<grid, kTileM, kSmemRequest, s>>>(
      feat, n, static_cast<const __nv_bfloat16*>(wbf), norm, wstat, pred, err, 1 << 22);
  return cudaGetLastError();
}

}  // namespace vbd
