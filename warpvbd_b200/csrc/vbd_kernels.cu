// VBD solver kernels for sm_100a.
//
// One VBD sweep visits the colours in order; inside a colour every solved
// vertex gathers the gradient and Hessian of the incremental potential over
// its incident tets and takes a guarded 3x3 Newton step.  Vertices of one
// colour share no tet, so they update in parallel without races (reference:
// accumulate_grad_hess + solve_grad_hess, mmichelis/WarpVBD
// src/vbd_solver.py:149-274; convergence test :578).
//
// Per (vertex, tet) slot the elastic terms are evaluated in closed form from
// the displacement gradient G = sum_n (u_n - u_v) b_n^T, F = I + G, where b_n
// are the gradients of the tet's linear shape functions and u the
// displacement from the rest shape.  With dF/dx_v^i = e_i b^T (b the vertex's
// own shape gradient) the reference's trace expressions
// (vbd_solver.py:116-124) reduce to
//   grad = V P b
//   Hess = V [ 2mu'/(Ic+1)^2 (F b)(F b)^T + mu' Ic/(Ic+1) |b|^2 I
//              + lambda' (cof(F) b)(cof(F) b)^T ]                     (SNH)
// and P is rewritten without cancellation at small strain:
//   P = mu' [ (Ic-3)/(4(Ic+1)) F + 3/4 (G + G^T - tr(G) I - cof(G)) ]
//       + lambda' (J-1) cof(F)
// using lambda'(alpha-1) = 3/4 mu', cof(F) = (1+tr G) I - G^T + cof(G) and
// J-1 = tr G + (tr(G)^2 - tr(G^2))/2 + det G.  StVK (vbd_solver.py:127-144)
// uses E = (G + G^T + G^T G)/2 in the same way.
#include <cuda_runtime.h>
#include <math.h>

#include "vbd_device.cuh"
#include "vbd_internal.h"
#include "vbd_launch.h"

namespace vbd {

// ---------------------------------------------------------------------------
// Block mode: blockIdx.x = environment.  The environment's displacements live
// in shared memory for the whole step; colours are separated by
// __syncthreads(); the convergence test is a block reduction.
// ---------------------------------------------------------------------------
template <typename Real, typename SReal, int TPV, int MAT>
__global__ void __launch_bounds__(512) env_step_kernel(DevMesh m, StepParams p,
                                                        const double* __restrict__ tol_env) {
  using S4 = real4<SReal>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S4* su = reinterpret_cast<S4*>(smem_raw);
  __shared__ unsigned long long s_red[32];
  __shared__ int s_done;
  __shared__ unsigned s_stat;
  const int env = blockIdx.x;
  const EnvInfo e = m.env[env];
  const StepConst sc = make_const(p);
  const double tol = tol_env ? tol_env[env] : p.tol;
  if (threadIdx.x == 0) s_stat = 0u;
  for (int i = threadIdx.x; i < e.nv; i += blockDim.x)
    su[i] = begin_vertex<SReal>(m, e.vbase + i, i < e.nact, sc);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  unsigned stat = 0u;
  int it = 0;
  bool converged = false;
  for (;;) {
    unsigned long long cmax = 0ull;
    for (int c = 0; c < e.ncolors; ++c) {
      const ColorInfo ci = m.color[e.cbase + c];
      for (int q = ci.chunk_begin + warp; q < ci.chunk_end; q += nwarps)
        process_chunk<Real, SReal, TPV, MAT, true>(m, e.vbase, ci, q, lane, su, sc, cmax, stat);
      __syncthreads();
    }
    ++it;
    cmax = warp_max_u64(cmax);
    if (lane == 0) s_red[warp] = cmax;
    __syncthreads();
    if (warp == 0) {
      unsigned long long v = lane < nwarps ? s_red[lane] : 0ull;
      v = warp_max_u64(v);
      if (lane == 0) {
        const bool nan = v > 0x7ff0000000000000ull;
        const bool conv = !nan && (__longlong_as_double((long long)v) < tol);
        s_done = (conv ? 1 : 0) | ((nan || conv || it >= p.max_iter) ? 2 : 0);
      }
    }
    __syncthreads();
    const int d = s_done;
    if (d & 2) {
      converged = d & 1;
      break;
    }
  }
  for (int i = threadIdx.x; i < e.nv; i += blockDim.x) {
    const S4 un = su[i];
    reinterpret_cast<S4*>(m.u)[e.vbase + i] = un;
    end_vertex<SReal>(m, e.vbase + i, un, sc);
  }
  if (stat) atomicOr(&s_stat, stat);
  __syncthreads();
  if (threadIdx.x == 0) {
    m.iters[env] = it;
    m.status[env] = s_stat | (converged ? 0u : kStatIterCap);
  }
}

// ---------------------------------------------------------------------------
// Grid mode (one environment): begin, colour sweeps, check, end.
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void begin_kernel(DevMesh m, const StepParams* __restrict__ pp, LoopControl* ctl) {
  const StepConst sc = make_const(*pp);
  const EnvInfo e = m.env[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    ctl->conv_bits = 0ull;
    ctl->iter = 0;
    ctl->status = 0u;
  }
  if (i < e.nv) {
    const real4<Real> un = begin_vertex<Real>(m, e.vbase + i, i < e.nact, sc);
    reinterpret_cast<real4<Real>*>(m.u)[e.vbase + i] = un;
  }
}

template <typename Real, typename SReal, int TPV, int MAT>
__global__ void __launch_bounds__(256) color_kernel(DevMesh m, int color,
                                                    const StepParams* __restrict__ pp,
                                                    LoopControl* ctl) {
  using S4 = real4<SReal>;
  __shared__ unsigned long long s_red[8];
  const StepConst sc = make_const(*pp);
  const ColorInfo ci = m.color[color];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = ci.chunk_begin + blockIdx.x * (blockDim.x >> 5) + warp;
  unsigned long long cmax = 0ull;
  unsigned stat = 0u;
  if (q < ci.chunk_end)
    process_chunk<Real, SReal, TPV, MAT, false>(m, 0, ci, q, lane, reinterpret_cast<S4*>(m.u),
                                                sc, cmax, stat);
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
    if (lane == 0 && v) atomicMax(&ctl->conv_bits, v);
  }
}

__global__ void check_kernel(LoopControl* ctl, const StepParams* __restrict__ pp,
                             cudaGraphConditionalHandle handle, int use_handle) {
  const unsigned long long v = ctl->conv_bits;
  const int it = ctl->iter + 1;
  ctl->iter = it;
  const bool nan = v > 0x7ff0000000000000ull;
  const bool conv = !nan && (__longlong_as_double((long long)v) < pp->tol);
  const bool stop = conv || nan || it >= pp->max_iter;
  if (stop && !conv) ctl->status |= kStatIterCap;
  if (nan) ctl->status |= kStatNonFinite;
  // bit 31 of status marks "loop finished" for the host-driven loop
  if (stop) ctl->status |= 0x80000000u;
  ctl->conv_bits = 0ull;
  if (use_handle && stop) cudaGraphSetConditional(handle, 0u);
}

template <typename Real>
__global__ void end_kernel(DevMesh m, const StepParams* __restrict__ pp, LoopControl* ctl) {
  const StepConst sc = make_const(*pp);
  const EnvInfo e = m.env[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < e.nv) {
    const real4<Real> un = reinterpret_cast<const real4<Real>*>(m.u)[e.vbase + i];
    end_vertex<Real>(m, e.vbase + i, un, sc);
  }
  if (i == 0) {
    m.iters[0] = ctl->iter;
    m.status[0] = ctl->status & 0x7fffffffu;
  }
}

// ---------------------------------------------------------------------------
// State exchange in the caller's vertex order.
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void gather_kernel(const double* __restrict__ off, const int* __restrict__ map,
                              const real4<Real>* __restrict__ st, double* __restrict__ out,
                              int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const real4<Real> v = st[map[i]];
  const double ox = off ? off[3 * i] : 0.0, oy = off ? off[3 * i + 1] : 0.0,
               oz = off ? off[3 * i + 2] : 0.0;
  out[3 * i] = ox + double(v.x);
  out[3 * i + 1] = oy + double(v.y);
  out[3 * i + 2] = oz + double(v.z);
}

template <typename Real>
__global__ void scatter_kernel(const double* __restrict__ off, const int* __restrict__ map,
                               const double* __restrict__ in, real4<Real>* __restrict__ st,
                               int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  real4<Real>& v = st[map[i]];
  const double ox = off ? off[3 * i] : 0.0, oy = off ? off[3 * i + 1] : 0.0,
               oz = off ? off[3 * i + 2] : 0.0;
  v.x = Real(in[3 * i] - ox);
  v.y = Real(in[3 * i + 1] - oy);
  v.z = Real(in[3 * i + 2] - oz);
}

template <typename Real>
__global__ void zero_xyz_kernel(real4<Real>* st, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  st[i].x = Real(0);
  st[i].y = Real(0);
  st[i].z = Real(0);
}

// ---------------------------------------------------------------------------
// Launchers.  prec: 0 = fp32 state and arithmetic, 1 = fp64 state with fp32
// arithmetic, 2 = fp64 throughout.
// ---------------------------------------------------------------------------
namespace {
// opt-in limit is 227 KB per block including the kernel's static shared memory
constexpr int kMaxSmem = 227 * 1024 - 2048;

template <typename Real, typename SReal, int TPV, int MAT>
cudaError_t env_launch_t(int threads, const DevMesh& m, const StepParams& p, const double* tol,
                         int n_env, size_t smem, cudaStream_t s) {
  static int configured_device = -1;  // the attribute is per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured_device != dev) {
    cudaError_t e = cudaFuncSetAttribute(env_step_kernel<Real, SReal, TPV, MAT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
    if (e != cudaSuccess) return e;
    configured_device = dev;
  }
  env_step_kernel<Real, SReal, TPV, MAT><<<n_env, threads, smem, s>>>(m, p, tol);
  return cudaGetLastError();
}

template <typename Real, typename SReal, int MAT>
cudaError_t env_launch_m(int tpv, int threads, const DevMesh& m, const StepParams& p,
                         const double* tol, int n_env, size_t smem, cudaStream_t s) {
  switch (tpv) {
    case 1: return env_launch_t<Real, SReal, 1, MAT>(threads, m, p, tol, n_env, smem, s);
    case 2: return env_launch_t<Real, SReal, 2, MAT>(threads, m, p, tol, n_env, smem, s);
    case 4: return env_launch_t<Real, SReal, 4, MAT>(threads, m, p, tol, n_env, smem, s);
    case 8: return env_launch_t<Real, SReal, 8, MAT>(threads, m, p, tol, n_env, smem, s);
    case 16: return env_launch_t<Real, SReal, 16, MAT>(threads, m, p, tol, n_env, smem, s);
    case 32: return env_launch_t<Real, SReal, 32, MAT>(threads, m, p, tol, n_env, smem, s);
    default: return cudaErrorInvalidValue;
  }
}

template <typename Real, typename SReal, int MAT>
cudaError_t color_launch_m(int tpv, int threads, const DevMesh& m, int color, int n_chunks,
                           const StepParams* p, LoopControl* ctl, cudaStream_t s) {
  const int wpb = threads / 32;
  const int blocks = (n_chunks + wpb - 1) / wpb;
  if (blocks == 0) return cudaSuccess;
#define VBD_COLOR(T)                                                                        \
  color_kernel<Real, SReal, T, MAT><<<blocks, threads, 0, s>>>(m, color, p, ctl);          \
  break
  switch (tpv) {
    case 1: VBD_COLOR(1);
    case 2: VBD_COLOR(2);
    case 4: VBD_COLOR(4);
    case 8: VBD_COLOR(8);
    case 16: VBD_COLOR(16);
    case 32: VBD_COLOR(32);
    default: return cudaErrorInvalidValue;
  }
#undef VBD_COLOR
  return cudaGetLastError();
}

template <typename Real, typename SReal>
cudaError_t env_launch_p(int material, int tpv, int threads, const DevMesh& m,
                         const StepParams& p, const double* tol, int n_env, size_t smem,
                         cudaStream_t s) {
  return material == kSNH
             ? env_launch_m<Real, SReal, kSNH>(tpv, threads, m, p, tol, n_env, smem, s)
             : env_launch_m<Real, SReal, kStVK>(tpv, threads, m, p, tol, n_env, smem, s);
}

template <typename Real, typename SReal>
cudaError_t color_launch_p(int material, int tpv, int threads, const DevMesh& m, int color,
                           int n_chunks, const StepParams* p, LoopControl* ctl,
                           cudaStream_t s) {
  return material == kSNH
             ? color_launch_m<Real, SReal, kSNH>(tpv, threads, m, color, n_chunks, p, ctl, s)
             : color_launch_m<Real, SReal, kStVK>(tpv, threads, m, color, n_chunks, p, ctl, s);
}

inline int nblk(int n, int t) { return (n + t - 1) / t; }
}  // namespace

int env_kernel_max_smem() { return kMaxSmem; }

cudaError_t launch_env_step(int prec, int material, int tpv, int threads, const DevMesh& m,
                            const StepParams& p, const double* tol_env, int n_env,
                            size_t smem, cudaStream_t s) {
  if (threads < 32 || threads > 512 || threads % 32) return cudaErrorInvalidValue;
  switch (prec) {
    case 0: return env_launch_p<float, float>(material, tpv, threads, m, p, tol_env, n_env, smem, s);
    case 1: return env_launch_p<float, double>(material, tpv, threads, m, p, tol_env, n_env, smem, s);
    case 2: return env_launch_p<double, double>(material, tpv, threads, m, p, tol_env, n_env, smem, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_color(int prec, int material, int tpv, int threads, const DevMesh& m,
                         int color, int n_chunks, const StepParams* p, LoopControl* ctl,
                         cudaStream_t s) {
  if (threads != 256) return cudaErrorInvalidValue;  // color_kernel reduces over 8 warps
  switch (prec) {
    case 0: return color_launch_p<float, float>(material, tpv, threads, m, color, n_chunks, p, ctl, s);
    case 1: return color_launch_p<float, double>(material, tpv, threads, m, color, n_chunks, p, ctl, s);
    case 2: return color_launch_p<double, double>(material, tpv, threads, m, color, n_chunks, p, ctl, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_begin(bool state64, const DevMesh& m, const StepParams* p, LoopControl* ctl,
                         cudaStream_t s) {
  const int n = m.n_vertices > 0 ? m.n_vertices : 1;
  if (state64)
    begin_kernel<double><<<nblk(n, 256), 256, 0, s>>>(m, p, ctl);
  else
    begin_kernel<float><<<nblk(n, 256), 256, 0, s>>>(m, p, ctl);
  return cudaGetLastError();
}

cudaError_t launch_check(LoopControl* ctl, const StepParams* p, unsigned long long handle,
                         int use_handle, cudaStream_t s) {
  check_kernel<<<1, 1, 0, s>>>(ctl, p, (cudaGraphConditionalHandle)handle, use_handle);
  return cudaGetLastError();
}

cudaError_t launch_end(bool state64, const DevMesh& m, const StepParams* p, LoopControl* ctl,
                       cudaStream_t s) {
  const int n = m.n_vertices > 0 ? m.n_vertices : 1;
  if (state64)
    end_kernel<double><<<nblk(n, 256), 256, 0, s>>>(m, p, ctl);
  else
    end_kernel<float><<<nblk(n, 256), 256, 0, s>>>(m, p, ctl);
  return cudaGetLastError();
}

cudaError_t launch_gather(bool state64, const double* off, const int* map, const void* st,
                          double* out, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (state64)
    gather_kernel<double><<<nblk(n, 256), 256, 0, s>>>(off, map,
                                                       static_cast<const double4*>(st), out, n);
  else
    gather_kernel<float><<<nblk(n, 256), 256, 0, s>>>(off, map, static_cast<const float4*>(st),
                                                      out, n);
  return cudaGetLastError();
}

cudaError_t launch_scatter(bool state64, const double* off, const int* map, const double* in,
                           void* st, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (state64)
    scatter_kernel<double><<<nblk(n, 256), 256, 0, s>>>(off, map, in,
                                                        static_cast<double4*>(st), n);
  else
    scatter_kernel<float><<<nblk(n, 256), 256, 0, s>>>(off, map, in, static_cast<float4*>(st),
                                                       n);
  return cudaGetLastError();
}

cudaError_t launch_zero_xyz(bool state64, void* st, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (state64)
    zero_xyz_kernel<double><<<nblk(n, 256), 256, 0, s>>>(static_cast<double4*>(st), n);
  else
    zero_xyz_kernel<float><<<nblk(n, 256), 256, 0, s>>>(static_cast<float4*>(st), n);
  return cudaGetLastError();
}

}  // namespace vbd
