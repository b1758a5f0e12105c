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
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>

#include "vbd_device.cuh"
#include "vbd_internal.h"
#include "vbd_launch.h"

namespace vbd {

// ---------------------------------------------------------------------------
// Block mode.  Work item work[blockIdx.x] = (environment, rank, group size):
// an environment runs on one thread block, or -- when it is much heavier
// than the others -- on all `group` blocks of one thread-block cluster.  Every
// block of a group holds a replica of the environment's positions (x, y, z)
// in shared memory for the whole step, updates its share of every colour
// (chunks rank, rank + group, ...) and writes each update into every replica
// through distributed shared memory.  Colours are separated by
// __syncthreads() (one block) or the cluster barrier (a group); the
// convergence test is a block reduction followed, in a group, by an exchange
// of the block maxima.  No block waits on a flag.
// ---------------------------------------------------------------------------
namespace cg = cooperative_groups;

constexpr int kMaxGroup = 16;

// Replicated environment state: loads from the block's own replica, stores
// into every replica of the group (remote replicas through distributed shared
// memory; map_shared_rank is one address-mapping instruction).
template <typename SReal>
struct GroupSmemState {
  SReal* local;
  int g, rank;
  __device__ __forceinline__ real4<SReal> load(int i) const {
    real4<SReal> v;
    v.x = local[3 * i];
    v.y = local[3 * i + 1];
    v.z = local[3 * i + 2];
    v.w = SReal(0);
    return v;
  }
  __device__ __forceinline__ void store(int i, const real4<SReal>& v) const {
    SReal* p = local + 3 * i;
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    cg::cluster_group cl = cg::this_cluster();
    for (int r = 0; r < g; ++r) {
      if (r == rank) continue;
      SReal* d = cl.map_shared_rank(p, r);
      d[0] = v.x;
      d[1] = v.y;
      d[2] = v.z;
    }
  }
};

template <bool GROUP>
__device__ __forceinline__ void group_sync(int g) {
  if (GROUP && g > 1)
    cg::this_cluster().sync();
  else
    __syncthreads();
}

// Sweeps of one environment until its convergence test passes or max_iter;
// returns the number of sweeps.
template <typename Real, typename SReal, int TPV, int MAT, int FMT, bool GROUP, class State>
__device__ __forceinline__ int env_sweeps(const DevMesh& m, const EnvInfo& e, const State& su,
                                          int rank, int g, const StepConst& sc, int max_iter,
                                          double tol, unsigned& stat, bool& converged,
                                          unsigned long long* s_red,
                                          unsigned long long (*s_conv)[kMaxGroup],
                                          int* s_done, const real4<Real>* tab,
                                          unsigned long long* dxw, Real* s_split) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  constexpr int kPart = SplitBuf<TPV>::per_part;
  int it = 0;
  for (;;) {
    unsigned long long cmax = 0ull;
    unsigned long long* dxrec = it + 1 == max_iter ? dxw : nullptr;
    for (int c = 0; c < e.ncolors; ++c) {
      const ColorInfo ci = m.color[e.cbase + c];
      const int nch = ci.chunk_end - ci.chunk_begin;
      const int W = split_ways<TPV>(nch);
      if (W == 1) {
        for (int q = ci.chunk_begin + rank + g * warp; q < ci.chunk_end; q += g * nwarps)
          process_chunk<Real, SReal, TPV, MAT, FMT>(m, e.vbase, ci, q, lane, su, sc, cmax, stat,
                                                    tab, dxrec);
      } else {
        // this block's chunks rank, rank + g, ...; W parts each (nloc x W <=
        // kSplitWarps, the size of s_split)
        const int nloc = rank < nch ? (nch - rank + g - 1) / g : 0;
        for (int pi = warp; pi < nloc * W; pi += nwarps) {
          const int q = ci.chunk_begin + rank + g * (pi / W);
          process_chunk_part<Real, SReal, TPV, MAT, FMT>(m, e.vbase, ci, q, lane, su, stat, tab,
                                                         pi % W, W, s_split + pi * kPart);
        }
        __syncthreads();
        for (int kl = warp; kl < nloc; kl += nwarps)
          finish_split_chunk<Real, SReal, TPV>(m, e.vbase, ci, ci.chunk_begin + rank + g * kl,
                                               lane, su, sc, cmax, stat, dxrec,
                                               s_split + kl * W * kPart, W);
        // s_split is reused by the next colour after the barrier below
      }
      group_sync<GROUP>(g);
    }
    ++it;
    cmax = warp_max_u64(cmax);
    if (lane == 0) s_red[warp] = cmax;
    __syncthreads();
    unsigned long long v = 0ull;
    if (warp == 0) {
      v = lane < nwarps ? s_red[lane] : 0ull;
      v = warp_max_u64(v);
    }
    if (GROUP && g > 1) {
      // exchange the block maxima (double-buffered by sweep parity)
      cg::cluster_group cl = cg::this_cluster();
      if (threadIdx.x == 0)
        for (int r = 0; r < g; ++r) *cl.map_shared_rank(&s_conv[it & 1][rank], r) = v;
      cl.sync();
      if (threadIdx.x == 0) {
        v = 0ull;
        for (int r = 0; r < g; ++r) v = s_conv[it & 1][r] > v ? s_conv[it & 1][r] : v;
      }
    }
    if (threadIdx.x == 0) {
      const bool nan = v > 0x7ff0000000000000ull;
      const bool conv = !nan && (__longlong_as_double((long long)v) < tol);
      *s_done = (conv ? 1 : 0) | ((nan || conv || it >= max_iter) ? 2 : 0);
    }
    __syncthreads();
    const int d = *s_done;
    if (d & 2) {
      converged = d & 1;
      return it;
    }
  }
}

// Incremental potential of an environment at its block's replica (tets'
// strain energy plus the solved vertices' inertia energy), summed over the
// group: every block sums its share of the tets and vertices, the block sums
// are exchanged through distributed shared memory (slot `buf` of s_esum).
template <typename Real, typename SReal, int MAT, bool GROUP>
__device__ double env_energy(const DevMesh& m, const EnvInfo& e, const SmemState<SReal>& st,
                             int rank, int g, const StepConst& sc, double* s_sum,
                             double (*s_esum)[kMaxGroup], int buf, const real4<Real>* tab) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int first = rank * blockDim.x + threadIdx.x, stride = g * blockDim.x;
  double acc = tet_energy<Real, SReal, MAT>(m, e, st, tab, first, stride, false).x;
  acc += inertia_energy<SReal>(m, e, st, sc, first, stride, false);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) s_sum[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int i = 0; i < nwarps; ++i) v += s_sum[i];
    s_sum[32] = v;
  }
  if (GROUP && g > 1) {
    cg::cluster_group cl = cg::this_cluster();
    if (threadIdx.x == 0)
      for (int r = 0; r < g; ++r) *cl.map_shared_rank(&s_esum[buf][rank], r) = s_sum[32];
    cl.sync();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int r = 0; r < g; ++r) v += s_esum[buf][r];
      s_sum[32] = v;
    }
  }
  __syncthreads();
  const double v = s_sum[32];
  __syncthreads();  // s_sum is reused by the next call
  return v;
}

// Both potentials the learned warm start compares, in one pass, summed over
// the environment (and the group): x = the strain energy at the inertia guess
// (its inertia energy is zero), y = the incremental potential at inertia guess
// + predicted correction.  Block sums are exchanged through distributed
// shared memory in s_pair (one slot per rank).
template <typename Real, typename SReal, int MAT, bool GROUP>
__device__ double2 env_energy_pair(const DevMesh& m, const EnvInfo& e, const SmemState<SReal>& st,
                                   int rank, int g, const StepConst& sc, double* s_sum,
                                   double2* s_pair, const real4<Real>* tab) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int first = rank * blockDim.x + threadIdx.x, stride = g * blockDim.x;
  const double2 el = tet_energy<Real, SReal, MAT>(m, e, st, tab, first, stride, true);
  double a = el.x;
  double b = el.y + inertia_energy<SReal>(m, e, st, sc, first, stride, true);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, off);
    b += __shfl_xor_sync(0xffffffffu, b, off);
  }
  // s_sum[0..15] and [16..31] hold the warps' two sums (at most 16 warps)
  if (lane == 0) {
    s_sum[warp] = a;
    s_sum[16 + warp] = b;
  }
  __syncthreads();
  __shared__ double2 s_tot;
  if (threadIdx.x == 0) {
    double va = 0.0, vb = 0.0;
    for (int i = 0; i < nwarps; ++i) {
      va += s_sum[i];
      vb += s_sum[16 + i];
    }
    s_tot = make_double2(va, vb);
  }
  if (GROUP && g > 1) {
    cg::cluster_group cl = cg::this_cluster();
    __syncthreads();
    if (threadIdx.x == 0)
      for (int r = 0; r < g; ++r) *cl.map_shared_rank(&s_pair[rank], r) = s_tot;
    cl.sync();
    if (threadIdx.x == 0) {
      double va = 0.0, vb = 0.0;
      for (int r = 0; r < g; ++r) {
        va += s_pair[r].x;
        vb += s_pair[r].y;
      }
      s_tot = make_double2(va, vb);
    }
  }
  __syncthreads();
  const double2 v = s_tot;
  __syncthreads();  // s_sum / s_tot are reused by the next call
  return v;
}

// Learned warm start: compare the incremental potential at the inertia guess
// (the replica's current content) with the one at inertia guess + alpha x
// predicted correction for alpha = 1, 1/2, 1/4 (a backtracking line search
// along the prediction: the next alpha is tried only when the previous one
// did not lower the potential), and keep the first that is lower, else the
// inertia guess.  The potentials are summed over the environment's tet list
// (each tet once) and its solved vertices; the first comparison (alpha = 1)
// takes one pass for both.  Every block of a group decides the same way
// from the same sums.  Returns kStatWarmUsed or 0.
template <typename Real, typename SReal, int TPV, int MAT, int FMT, bool GROUP>
__device__ unsigned warm_start_stage(const DevMesh& m, const EnvInfo& e,
                                     const SmemState<SReal>& local, int rank, int g,
                                     const StepConst& sc, double* s_sum,
                                     double (*s_esum)[kMaxGroup], double2* s_pair,
                                     const real4<Real>* tab) {
  using S4 = real4<SReal>;
  const S4* UT = reinterpret_cast<const S4*>(m.ut) + e.vbase;
  auto place = [&](SReal alpha) {
    // candidate: inertia guess + alpha x prediction, formed from ut each time
    for (int i = threadIdx.x; i < e.nsolved; i += blockDim.x) {
      const float4 d = m.ws_pred[e.vbase + i];
      if (d.w > 0.f) {
        S4 v = ldcg4(UT + i);
        v.x += alpha * SReal(d.x);
        v.y += alpha * SReal(d.y);
        v.z += alpha * SReal(d.z);
        local.store(i, v);
      }
    }
  };
  const double2 e01 =
      env_energy_pair<Real, SReal, MAT, GROUP>(m, e, local, rank, g, sc, s_sum, s_pair, tab);
  const double e0 = e01.x;
  if (e01.y < e0) {  // false on NaN as well
    place(SReal(1));
    return (unsigned)kStatWarmUsed;
  }
  int buf = 0;
  for (int trial = 1; trial < 3; ++trial) {
    place(SReal(1.0 / double(1 << trial)));
    __syncthreads();
    const double e1 =
        env_energy<Real, SReal, MAT, GROUP>(m, e, local, rank, g, sc, s_sum, s_esum, buf, tab);
    buf ^= 1;
    if (e1 < e0) return (unsigned)kStatWarmUsed;
  }
  // back to the inertia guess, exactly as begin computed it
  for (int i = threadIdx.x; i < e.nsolved; i += blockDim.x) local.store(i, ldcg4(UT + i));
  return 0u;
}

template <typename Real, typename SReal, int TPV, int MAT, int FMT, bool GROUP>
__global__ void __launch_bounds__(512) env_step_kernel(DevMesh m, StepParams p,
                                                        const double* __restrict__ tol_env,
                                                        const int4* __restrict__ work) {
  using S4 = real4<SReal>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SReal* sp = reinterpret_cast<SReal*>(smem_raw);
  __shared__ unsigned long long s_red[32];
  __shared__ unsigned long long s_conv[2][kMaxGroup];
  __shared__ double s_sum[33];
  __shared__ double s_esum[2][kMaxGroup];
  __shared__ double2 s_pair[kMaxGroup];
  __shared__ int s_done;
  __shared__ unsigned s_stat;
  // per-part sums of the split chunks of small colours (env_sweeps)
  __shared__ Real s_split[kSplitWarps * SplitBuf<TPV>::per_part];
  const int4 w = work[blockIdx.x];
  const int env = w.x, rank = w.y, g = w.z;
  if (env < 0) return;  // padding block of a cluster of single-block environments
  const unsigned long long t_start = p.trace ? globaltimer_ns() : 0ull;
  const EnvInfo e = m.env[env];
  const StepConst sc = make_const(p);
  // the environment's record table: staged in shared memory after the state
  // when the launch reserved room for it (p.tab_in_smem), else read from
  // global memory; either way a generic pointer to its 3 x nrec Real4
  using R4 = real4<Real>;
  const R4* gtab = reinterpret_cast<const R4*>(m.rec_tab) + 3 * (size_t)e.rbase;
  const R4* tab = gtab;
  if (p.tab_in_smem) {
    R4* stab = reinterpret_cast<R4*>(smem_raw + tab_smem_offset<SReal>(e.nv));
    for (int i = threadIdx.x; i < 3 * e.nrec; i += blockDim.x) stab[i] = ldg4(gtab + i);
    tab = stab;  // visible to the block after the __syncthreads / cluster barrier below
  }
  const double tol = tol_env ? tol_env[env] : p.tol;
  if (threadIdx.x == 0) s_stat = 0u;
  // every replica computes the inertia guess of every vertex; rank 0 writes
  // the step-start state back
  const SmemState<SReal> local{sp};
  for (int i = threadIdx.x; i < e.nv; i += blockDim.x)
    local.store(i, begin_vertex<SReal>(m, e.vbase + i, i < e.nact, sc, rank == 0));
  unsigned stat = 0u;
  bool converged = false;
  int it;
  if (GROUP && g > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const GroupSmemState<SReal> su{sp, g, rank};
    cl.sync();  // every block of the group has started and filled its replica
    if (p.warm && m.ws_pred) {
      stat |= warm_start_stage<Real, SReal, TPV, MAT, FMT, GROUP>(m, e, local, rank, g, sc, s_sum,
                                                                 s_esum, s_pair, tab);
      cl.sync();  // replicas settled before the first remote update
    }
    it = env_sweeps<Real, SReal, TPV, MAT, FMT, GROUP>(m, e, su, rank, g, sc, p.max_iter, tol,
                                                        stat, converged, s_red, s_conv, &s_done,
                                                        tab, m.dxmax + env, s_split);
  } else {
    __syncthreads();
    if (p.warm && m.ws_pred) {
      stat |= warm_start_stage<Real, SReal, TPV, MAT, FMT, false>(m, e, local, 0, 1, sc, s_sum,
                                                                 s_esum, s_pair, tab);
      __syncthreads();
    }
    it = env_sweeps<Real, SReal, TPV, MAT, FMT, false>(m, e, local, 0, 1, sc, p.max_iter, tol,
                                                        stat, converged, s_red, s_conv, &s_done,
                                                        tab, m.dxmax + env, s_split);
  }
  // velocity update and write-back, vertices split over the group
  for (int i = rank + g * threadIdx.x; i < e.nv; i += g * blockDim.x) {
    S4 un = local.load(i);
    un.w = reinterpret_cast<const S4*>(m.u)[e.vbase + i].w;
    reinterpret_cast<S4*>(m.u)[e.vbase + i] = un;
    end_vertex<SReal>(m, e.vbase + i, un, sc);
  }
  if (m.host_out) {
    // the environment's positions in the caller's order, one double per
    // thread and consecutive threads on consecutive doubles (the caller's
    // vertex ids of an environment are its renumbered range), written over
    // the bus while other environments still run
    double* out = m.host_out + 3 * (size_t)e.vbase;
    const double* rest = m.rest + 3 * (size_t)e.vbase;
    for (int k = rank * blockDim.x + threadIdx.x; k < 3 * e.nv; k += g * blockDim.x) {
      const int j = k / 3, c = k - 3 * j;
      const S4 un = local.load(m.map[e.vbase + j] - e.vbase);
      out[k] = rest[k] + double(c == 0 ? un.x : (c == 1 ? un.y : un.z));
    }
  }
  if (stat) atomicOr(&s_stat, stat);
  __syncthreads();
  if (GROUP && g > 1) {
    cg::cluster_group cl = cg::this_cluster();
    if (threadIdx.x == 0 && rank != 0 && s_stat)
      atomicOr(cl.map_shared_rank(&s_stat, 0), s_stat);
    cl.sync();  // also the last access of another block's shared memory
  }
  if (threadIdx.x == 0 && rank == 0) {
    m.iters[env] = it;
    m.status[env] = s_stat | (converged ? 0u : kStatIterCap);
  }
  if (p.trace && threadIdx.x == 0) {
    unsigned long long* r = p.trace + 4 * (size_t)blockIdx.x;
    r[0] = t_start;
    r[1] = globaltimer_ns();
    r[2] = ((unsigned long long)env << 32) | ((unsigned long long)rank << 16) | sm_id();
    r[3] = ((unsigned long long)it << 8) | (unsigned long long)w.w;
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
    const real4<Real> un = begin_vertex<Real>(m, e.vbase + i, i < e.nact, sc, true);
    reinterpret_cast<real4<Real>*>(m.u)[e.vbase + i] = un;
  }
}

template <typename Real, typename SReal, int TPV, int MAT, int FMT>
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
  const GlobalState<SReal> state{reinterpret_cast<S4*>(m.u)};
  // sweeps done so far: check_kernel advances it after every sweep
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
// dynamic shared memory of a block-mode block at most: 227 KB less the
// kernel's static arrays (2 KB of reductions, and the split-chunk sums: 16
// parts x 9 values x 16 vertices x 8 bytes at the largest)
constexpr int kMaxSmem = 227 * 1024 - 2048 - kSplitWarps * 9 * 16 * 8;

template <typename Real, typename SReal, int TPV, int MAT, int FMT, bool GROUP>
cudaError_t configure_env_kernel() {
  static int configured_device = -1;  // the attributes are per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured_device == dev) return cudaSuccess;
  auto* k = env_step_kernel<Real, SReal, TPV, MAT, FMT, GROUP>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  if (e == cudaSuccess && GROUP)
    e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e == cudaSuccess) configured_device = dev;
  return e;
}

struct EnvLaunch {
  int threads;
  const DevMesh& m;
  const StepParams& p;
  const double* tol;
  const int4* work;
  int n_blocks, cluster;
  size_t smem;
  cudaStream_t s;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    if (cluster <= 1) {
      cudaError_t e = configure_env_kernel<Real, SReal, TPV, MAT, FMT, false>();
      if (e != cudaSuccess) return e;
      env_step_kernel<Real, SReal, TPV, MAT, FMT, false><<<n_blocks, threads, smem, s>>>(
          m, p, tol, work);
      return cudaGetLastError();
    }
    cudaError_t e = configure_env_kernel<Real, SReal, TPV, MAT, FMT, true>();
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, env_step_kernel<Real, SReal, TPV, MAT, FMT, true>, m, p, tol,
                              work);
  }
};

// Resident blocks per SM (cluster = 1) or resident clusters on the device.
struct EnvOccupancy {
  int threads;
  size_t smem;
  int cluster;
  int* out;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    if (cluster <= 1) {
      cudaError_t e = configure_env_kernel<Real, SReal, TPV, MAT, FMT, false>();
      if (e != cudaSuccess) return e;
      return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          out, env_step_kernel<Real, SReal, TPV, MAT, FMT, false>, threads, smem);
    }
    cudaError_t e = configure_env_kernel<Real, SReal, TPV, MAT, FMT, true>();
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster * 64);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(out, env_step_kernel<Real, SReal, TPV, MAT, FMT, true>,
                                          &cfg);
  }
};

struct ColorLaunch {
  int blocks, threads;
  const DevMesh& m;
  int color;
  const StepParams* p;
  LoopControl* ctl;
  cudaStream_t s;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    color_kernel<Real, SReal, TPV, MAT, FMT><<<blocks, threads, 0, s>>>(m, color, p, ctl);
    return cudaGetLastError();
  }
};

// Incremental potential of every environment at a candidate state `x`
// (displacements, renumbered), for a step of length dt from the current state
// (u, vel): the same tet-list strain energy and inertia energy the learned
// warm start compares, with the inertia target formed as begin_vertex forms
// it (not written back).  One block per environment.
template <typename Real, typename SReal, int MAT>
__global__ void __launch_bounds__(256) potential_kernel(DevMesh m, StepParams p,
                                                        const real4<SReal>* __restrict__ x,
                                                        double* __restrict__ out) {
  using S4 = real4<SReal>;
  using R4 = real4<Real>;
  const EnvInfo e = m.env[blockIdx.x];
  const StepConst sc = make_const(p);
  const GlobalState<SReal> st{const_cast<S4*>(x) + e.vbase};  // read only
  const R4* tab = reinterpret_cast<const R4*>(m.rec_tab) + 3 * (size_t)e.rbase;
  double acc = tet_energy<Real, SReal, MAT>(m, e, st, tab, threadIdx.x, blockDim.x, false).x;
  const S4* U = reinterpret_cast<const S4*>(m.u) + e.vbase;
  const S4* V = reinterpret_cast<const S4*>(m.vel) + e.vbase;
  const S4* UT = reinterpret_cast<const S4*>(m.ut) + e.vbase;
  for (int i = threadIdx.x; i < e.nsolved; i += blockDim.x) {
    const S4 u0 = U[i], v0 = V[i], xi = x[e.vbase + i];
    const SReal dt = SReal(sc.dt), dt2 = SReal(sc.dt2);
    const SReal tx = u0.x + v0.x * dt + SReal(sc.g[0]) * dt2;
    const SReal ty = u0.y + v0.y * dt + SReal(sc.g[1]) * dt2;
    const SReal tz = u0.z + v0.z * dt + SReal(sc.g[2]) * dt2;
    const double dx = double(xi.x - tx), dy = double(xi.y - ty), dz = double(xi.z - tz);
    acc += 0.5 * double(UT[i].w) * sc.inv_dt2 * (dx * dx + dy * dy + dz * dz);
  }
  __shared__ double s_part[8];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += s_part[w];
    out[blockIdx.x] = v;
  }
}

struct PotentialLaunch {
  const DevMesh& m;
  const StepParams& p;
  const void* x;
  double* out;
  cudaStream_t s;
  template <typename Real, typename SReal, int TPV, int MAT, int FMT>
  cudaError_t run() {
    if (TPV != 4 || FMT != kFmtIdx32) return cudaSuccess;  // one instantiation per precision
    potential_kernel<Real, SReal, MAT><<<m.n_env, 256, 0, s>>>(
        m, p, static_cast<const real4<SReal>*>(x), out);
    return cudaGetLastError();
  }
};

inline int nblk(int n, int t) { return (n + t - 1) / t; }
}  // namespace

int env_kernel_max_smem() { return kMaxSmem; }

cudaError_t launch_potential(int prec, int material, const DevMesh& m, const StepParams& p,
                             const void* x, double* out, cudaStream_t s) {
  if (m.n_env <= 0) return cudaSuccess;
  PotentialLaunch f{m, p, x, out, s};
  return dispatch(prec, material, kFmtIdx32, 4, f);
}

cudaError_t launch_env_step(int prec, int material, int tpv, int threads, const DevMesh& m,
                            const StepParams& p, const double* tol_env, const int4* work,
                            int n_blocks, int cluster, size_t smem, cudaStream_t s) {
  if (threads < 32 || threads > 512 || threads % 32) return cudaErrorInvalidValue;
  if (cluster < 1 || cluster > kMaxGroup || n_blocks % cluster) return cudaErrorInvalidValue;
  EnvLaunch f{threads, m, p, tol_env, work, n_blocks, cluster, smem, s};
  return dispatch(prec, material, m.fmt, tpv, f);
}

cudaError_t env_occupancy(int prec, int material, int fmt, int tpv, int threads, size_t smem,
                          int cluster, int* out) {
  EnvOccupancy f{threads, smem, cluster, out};
  return dispatch(prec, material, fmt, tpv, f);
}

cudaError_t launch_color(int prec, int material, int tpv, int threads, const DevMesh& m,
                         int color, int n_chunks, const StepParams* p, LoopControl* ctl,
                         cudaStream_t s) {
  if (threads != 256) return cudaErrorInvalidValue;  // color_kernel reduces over 8 warps
  const int blocks = (n_chunks + 7) / 8;
  if (blocks == 0) return cudaSuccess;
  ColorLaunch f{blocks, threads, m, color, p, ctl, s};
  return dispatch(prec, material, m.fmt, tpv, f);
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
