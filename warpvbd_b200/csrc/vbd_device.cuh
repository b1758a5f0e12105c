// Device-side building blocks shared by the solver kernels (vbd_kernels.cu)
// and the allocation-free step (vbd_noalloc.cu): vector types, the per-slot
// elastic terms, the guarded 3x3 solve and the per-chunk vertex update.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "vbd_internal.h"

namespace vbd {

template <typename Real>
struct V4;
template <>
struct V4<float> {
  using type = float4;
};
template <>
struct V4<double> {
  using type = double4;
};
template <typename Real>
using real4 = typename V4<Real>::type;

__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned sm_id() {
  unsigned r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
}
__device__ __forceinline__ float4 ldcg4(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ double4 ldcg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldcg(q), b = __ldcg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ double4 ldg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ unsigned long long conv_bits(double c) {
  // c >= 0 or NaN; fabs clears the sign so NaN bits sort above +Inf
  return static_cast<unsigned long long>(__double_as_longlong(fabs(c)));
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
    v = o > v ? o : v;
  }
  return v;
}

// ---------------------------------------------------------------------------
// Elastic gradient / Hessian of one (vertex, tet) slot, accumulated into g, h
// (h = h00 h01 h02 h11 h12 h22).  d* = u_n - u_v of the tet's other three
// vertices, q* = (b_n, p): p0 = V*mu, p1 = V*lambda (material-adjusted).
// ---------------------------------------------------------------------------
template <typename Real, int MAT>
__device__ __forceinline__ void slot_accumulate(Real d0x, Real d0y, Real d0z, Real d1x, Real d1y,
                                                Real d1z, Real d2x, Real d2y, Real d2z,
                                                const real4<Real>& q0, const real4<Real>& q1,
                                                const real4<Real>& q2, Real* g, Real* h) {
  const Real G00 = d0x * q0.x + d1x * q1.x + d2x * q2.x;
  const Real G01 = d0x * q0.y + d1x * q1.y + d2x * q2.y;
  const Real G02 = d0x * q0.z + d1x * q1.z + d2x * q2.z;
  const Real G10 = d0y * q0.x + d1y * q1.x + d2y * q2.x;
  const Real G11 = d0y * q0.y + d1y * q1.y + d2y * q2.y;
  const Real G12 = d0y * q0.z + d1y * q1.z + d2y * q2.z;
  const Real G20 = d0z * q0.x + d1z * q1.x + d2z * q2.x;
  const Real G21 = d0z * q0.y + d1z * q1.y + d2z * q2.y;
  const Real G22 = d0z * q0.z + d1z * q1.z + d2z * q2.z;
  const Real bx = -(q0.x + q1.x + q2.x);
  const Real by = -(q0.y + q1.y + q2.y);
  const Real bz = -(q0.z + q1.z + q2.z);
  const Real p0 = q0.w, p1 = q1.w;
  const Real bb = bx * bx + by * by + bz * bz;
  if (MAT == kSNH && sizeof(Real) == 8) {
    // fp64: the reference's own form (vbd_solver.py:111-114, 118-123)
    //   P b = mu' (1 - 1/(Ic+1)) F b + lambda' (J - alpha) cof(F) b
    // with lambda' (J - alpha) = lambda' (J - 1) - 3/4 mu'.  The difference
    // J - 1 cancels at small strain, as the reference's J - alpha does; in
    // double precision that costs ~1e-16 / strain relative, far below the
    // solver's tolerance, and it needs fewer operations and live values than
    // the cancellation-free form the fp32 path uses below.
    const Real F00 = Real(1) + G00, F11 = Real(1) + G11, F22 = Real(1) + G22;
    const Real Fbx = F00 * bx + G01 * by + G02 * bz;
    const Real Fby = G10 * bx + F11 * by + G12 * bz;
    const Real Fbz = G20 * bx + G21 * by + F22 * bz;
    const Real Ic = F00 * F00 + G01 * G01 + G02 * G02 + G10 * G10 + F11 * F11 + G12 * G12 +
                    G20 * G20 + G21 * G21 + F22 * F22;
    // cof(F) row by row: J from row 0, cof(F) b from all three
    Real c0 = F11 * F22 - G12 * G21, c1 = G12 * G20 - G10 * F22, c2 = G10 * G21 - F11 * G20;
    const Real J = F00 * c0 + G01 * c1 + G02 * c2;
    const Real Cbx = c0 * bx + c1 * by + c2 * bz;
    c0 = G21 * G02 - F22 * G01;
    c1 = F22 * F00 - G20 * G02;
    c2 = G20 * G01 - G21 * F00;
    const Real Cby = c0 * bx + c1 * by + c2 * bz;
    c0 = G01 * G12 - G02 * F11;
    c1 = G02 * G10 - F00 * G12;
    c2 = F00 * F11 - G01 * G10;
    const Real Cbz = c0 * bx + c1 * by + c2 * bz;
    const Real p0 = q0.w, p1 = q1.w;
    const Real inv = Real(1) / (Ic + Real(1));
    const Real a = p0 * (Real(1) - inv);
    const Real kJ = p1 * (J - Real(1)) - Real(0.75) * p0;
    g[0] += a * Fbx + kJ * Cbx;
    g[1] += a * Fby + kJ * Cby;
    g[2] += a * Fbz + kJ * Cbz;
    const Real hF = Real(2) * p0 * inv * inv;
    const Real hI = a * bb;
    const Real Fx = hF * Fbx, Fy = hF * Fby, Fz = hF * Fbz;
    const Real Cx = p1 * Cbx, Cy = p1 * Cby, Cz = p1 * Cbz;
    h[0] += Fx * Fbx + Cx * Cbx + hI;
    h[1] += Fx * Fby + Cx * Cby;
    h[2] += Fx * Fbz + Cx * Cbz;
    h[3] += Fy * Fby + Cy * Cby + hI;
    h[4] += Fy * Fbz + Cy * Cbz;
    h[5] += Fz * Fbz + Cz * Cbz + hI;
    return;
  }
  const Real Gbx = G00 * bx + G01 * by + G02 * bz;
  const Real Gby = G10 * bx + G11 * by + G12 * bz;
  const Real Gbz = G20 * bx + G21 * by + G22 * bz;
  const Real Fbx = bx + Gbx, Fby = by + Gby, Fbz = bz + Gbz;
  const Real t = G00 + G11 + G22;
  if (MAT == kSNH) {
    const Real c00 = G11 * G22 - G12 * G21, c01 = G12 * G20 - G10 * G22,
               c02 = G10 * G21 - G11 * G20;
    const Real c10 = G21 * G02 - G22 * G01, c11 = G22 * G00 - G20 * G02,
               c12 = G20 * G01 - G21 * G00;
    const Real c20 = G01 * G12 - G02 * G11, c21 = G02 * G10 - G00 * G12,
               c22 = G00 * G11 - G01 * G10;
    const Real detG = G00 * c00 + G01 * c01 + G02 * c02;
    const Real trG2 =
        G00 * G00 + G11 * G11 + G22 * G22 + Real(2) * (G01 * G10 + G02 * G20 + G12 * G21);
    const Real nG2 = G00 * G00 + G01 * G01 + G02 * G02 + G10 * G10 + G11 * G11 + G12 * G12 +
                     G20 * G20 + G21 * G21 + G22 * G22;
    const Real Jm1 = t + Real(0.5) * (t * t - trG2) + detG;
    const Real Icm3 = Real(2) * t + nG2;
    const Real inv = Real(1) / (Icm3 + Real(4));
    const Real GTbx = G00 * bx + G10 * by + G20 * bz;
    const Real GTby = G01 * bx + G11 * by + G21 * bz;
    const Real GTbz = G02 * bx + G12 * by + G22 * bz;
    const Real cGbx = c00 * bx + c01 * by + c02 * bz;
    const Real cGby = c10 * bx + c11 * by + c12 * bz;
    const Real cGbz = c20 * bx + c21 * by + c22 * bz;
    const Real t1 = Real(1) + t;
    const Real Cbx = t1 * bx - GTbx + cGbx;
    const Real Cby = t1 * by - GTby + cGby;
    const Real Cbz = t1 * bz - GTbz + cGbz;
    const Real a = Real(0.25) * p0 * Icm3 * inv;
    const Real k3 = Real(0.75) * p0;
    const Real kJ = p1 * Jm1;
    g[0] += a * Fbx + k3 * (Gbx + GTbx - t * bx - cGbx) + kJ * Cbx;
    g[1] += a * Fby + k3 * (Gby + GTby - t * by - cGby) + kJ * Cby;
    g[2] += a * Fbz + k3 * (Gbz + GTbz - t * bz - cGbz) + kJ * Cbz;
    const Real hF = Real(2) * p0 * inv * inv;
    const Real hI = p0 * (Icm3 + Real(3)) * inv * bb;
    const Real Fx = hF * Fbx, Fy = hF * Fby, Fz = hF * Fbz;
    const Real Cx = p1 * Cbx, Cy = p1 * Cby, Cz = p1 * Cbz;
    h[0] += Fx * Fbx + Cx * Cbx + hI;
    h[1] += Fx * Fby + Cx * Cby;
    h[2] += Fx * Fbz + Cx * Cbz;
    h[3] += Fy * Fby + Cy * Cby + hI;
    h[4] += Fy * Fbz + Cy * Cbz;
    h[5] += Fz * Fbz + Cz * Cbz + hI;
  } else {
    // E = (G + G^T + G^T G) / 2
    const Real E00 = G00 + Real(0.5) * (G00 * G00 + G10 * G10 + G20 * G20);
    const Real E11 = G11 + Real(0.5) * (G01 * G01 + G11 * G11 + G21 * G21);
    const Real E22 = G22 + Real(0.5) * (G02 * G02 + G12 * G12 + G22 * G22);
    const Real E01 = Real(0.5) * (G01 + G10 + G00 * G01 + G10 * G11 + G20 * G21);
    const Real E02 = Real(0.5) * (G02 + G20 + G00 * G02 + G10 * G12 + G20 * G22);
    const Real E12 = Real(0.5) * (G12 + G21 + G01 * G02 + G11 * G12 + G21 * G22);
    const Real trE = E00 + E11 + E22;
    const Real Ebx = E00 * bx + E01 * by + E02 * bz;
    const Real Eby = E01 * bx + E11 * by + E12 * bz;
    const Real Ebz = E02 * bx + E12 * by + E22 * bz;
    const Real FEbx = Ebx + G00 * Ebx + G01 * Eby + G02 * Ebz;
    const Real FEby = Eby + G10 * Ebx + G11 * Eby + G12 * Ebz;
    const Real FEbz = Ebz + G20 * Ebx + G21 * Eby + G22 * Ebz;
    const Real k2 = Real(2) * p0, kt = p1 * trE;
    g[0] += k2 * FEbx + kt * Fbx;
    g[1] += k2 * FEby + kt * Fby;
    g[2] += k2 * FEbz + kt * Fbz;
    const Real bEb = bx * Ebx + by * Eby + bz * Ebz;
    // F F^T = I + G + G^T + G G^T
    const Real A00 = Real(1) + Real(2) * G00 + G00 * G00 + G01 * G01 + G02 * G02;
    const Real A11 = Real(1) + Real(2) * G11 + G10 * G10 + G11 * G11 + G12 * G12;
    const Real A22 = Real(1) + Real(2) * G22 + G20 * G20 + G21 * G21 + G22 * G22;
    const Real A01 = G01 + G10 + G00 * G10 + G01 * G11 + G02 * G12;
    const Real A02 = G02 + G20 + G00 * G20 + G01 * G21 + G02 * G22;
    const Real A12 = G12 + G21 + G10 * G20 + G11 * G21 + G12 * G22;
    const Real kff = p1 + p0;
    const Real kA = p0 * bb;
    const Real kI = kt * bb + k2 * bEb;
    h[0] += kff * Fbx * Fbx + kA * A00 + kI;
    h[1] += kff * Fbx * Fby + kA * A01;
    h[2] += kff * Fbx * Fbz + kA * A02;
    h[3] += kff * Fby * Fby + kA * A11 + kI;
    h[4] += kff * Fby * Fbz + kA * A12;
    h[5] += kff * Fbz * Fbz + kA * A22 + kI;
  }
}

// Guarded Newton step: solve H dx = -g by 3x3 Cholesky (the reference's
// tile_cholesky / tile_cholesky_solve, vbd_solver.py:267-268).  Returns false
// when a pivot is not positive (H not positive definite).
template <typename Real>
__device__ __forceinline__ bool chol_solve3(const Real* h, const Real* g, Real* x) {
  const Real L00 = sqrt(h[0]);
  const Real i0 = Real(1) / L00;
  const Real L10 = h[1] * i0, L20 = h[2] * i0;
  const Real d1 = h[3] - L10 * L10;
  const Real L11 = sqrt(d1);
  const Real i1 = Real(1) / L11;
  const Real L21 = (h[4] - L20 * L10) * i1;
  const Real d2 = h[5] - L20 * L20 - L21 * L21;
  const Real L22 = sqrt(d2);
  const Real i2 = Real(1) / L22;
  const Real y0 = -g[0] * i0;
  const Real y1 = (-g[1] - L10 * y0) * i1;
  const Real y2 = (-g[2] - L20 * y0 - L21 * y1) * i2;
  x[2] = y2 * i2;
  x[1] = (y1 - L21 * x[2]) * i1;
  x[0] = (y0 - L10 * x[1] - L20 * x[2]) * i0;
  return (h[0] > Real(0)) && (d1 > Real(0)) && (d2 > Real(0));
}

struct StepConst {
  double inv_dt2, kd_dt, dt, dt2;
  double g[3];
  bool damp, strict;
};

__device__ __forceinline__ StepConst make_const(const StepParams& p) {
  StepConst c;
  c.dt = p.dt;
  c.dt2 = p.dt * p.dt;
  c.inv_dt2 = 1.0 / c.dt2;
  c.kd_dt = p.kd / p.dt;
  c.damp = p.kd != 0.0;
  c.strict = p.strict_spd != 0;
  c.g[0] = p.g[0];
  c.g[1] = p.g[1];
  c.g[2] = p.g[2];
  return c;
}

// ---------------------------------------------------------------------------
// State accessors: environment-local vertex ids -> displacement.
// SmemState: packed xyz (3 values per vertex) in shared memory (block mode).
// GlobalState: Real4 per vertex in global memory (grid mode).
// ---------------------------------------------------------------------------
// Byte offset of an environment's staged record table in block-mode shared
// memory: after the packed xyz state of its nv vertices, 16-byte aligned.
template <typename SReal>
__host__ __device__ __forceinline__ size_t tab_smem_offset(int nv) {
  return ((size_t)nv * 3 * sizeof(SReal) + 15) / 16 * 16;
}

template <typename SReal>
struct SmemState {
  SReal* p;
  __device__ __forceinline__ real4<SReal> load(int i) const {
    real4<SReal> v;
    v.x = p[3 * i];
    v.y = p[3 * i + 1];
    v.z = p[3 * i + 2];
    v.w = SReal(0);
    return v;
  }
  __device__ __forceinline__ void store(int i, const real4<SReal>& v) const {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
  }
};

template <typename SReal>
struct GlobalState {
  real4<SReal>* p;
  // neighbours of other colours are not written during a colour's kernel, and
  // the vertex's own value was written by an earlier kernel: the read-only
  // path is safe
  __device__ __forceinline__ real4<SReal> load(int i) const { return ldg4(p + i); }
  __device__ __forceinline__ void store(int i, const real4<SReal>& v) const { p[i] = v; }
};

template <int FMT>
__device__ __forceinline__ int4 load_slot(const DevMesh& m, size_t i) {
  if (FMT == kFmtIdx16) {
    const ushort4 s = __ldg(m.rec_idx16 + i);
    return make_int4(s.x, s.y, s.z, s.w);
  }
  return __ldg(m.rec_idx + i);
}

// A slot as stored (kept packed in registers while prefetched).
template <int FMT>
struct RawSlot;
template <>
struct RawSlot<kFmtIdx16> {
  using type = ushort4;
  static __device__ __forceinline__ ushort4 load(const DevMesh& m, size_t i) {
    return __ldg(m.rec_idx16 + i);
  }
  static __device__ __forceinline__ int4 unpack(const ushort4& s) {
    return make_int4(s.x, s.y, s.z, s.w);
  }
};
template <>
struct RawSlot<kFmtIdx32> {
  using type = int4;
  static __device__ __forceinline__ int4 load(const DevMesh& m, size_t i) {
    return __ldg(m.rec_idx + i);
  }
  static __device__ __forceinline__ int4 unpack(const int4& s) { return s; }
};

// Bounds-checked build (make check -> libvbd_b200_check.so): every slot's
// neighbour and record ids, and the vertex's own id, are checked against its
// environment before use; an id out of range sets kStatBounds (the step then
// fails with VBD_ERR_BOUNDS) and the access is skipped.
#ifndef VBD_CHECK_BOUNDS
#define VBD_CHECK_BOUNDS 0
#endif

// Slot steps of a chunk whose indices are loaded up front: enough for the
// reference's 20 incident tets per vertex (MAX_ELEMENTS_PER_VERTEX); longer
// chunks stream the rest.
template <int TPV>
struct Prefetch {
  static constexpr int steps = (20 + TPV - 1) / TPV;
};

// The vertex's update from its summed elastic gradient g and Hessian h (the
// lane that holds them): inertia term, damping, guarded 3x3 Newton step,
// store, convergence measure.
template <typename Real, typename SReal, class State>
__device__ __forceinline__ void finish_vertex(const DevMesh& m, int gv, int lv,
                                              const real4<SReal>& uo, const real4<SReal>& tt,
                                              const Real (&g)[3], Real (&h)[6], const State& st,
                                              const StepConst& sc, unsigned long long& cmax,
                                              unsigned& stat, unsigned long long* dxrec) {
  using S4 = real4<SReal>;
  const Real mdt2 = Real(tt.w * SReal(sc.inv_dt2));
  Real G[3], H[6];
  G[0] = g[0] + mdt2 * Real(uo.x - tt.x);
  G[1] = g[1] + mdt2 * Real(uo.y - tt.y);
  G[2] = g[2] + mdt2 * Real(uo.z - tt.z);
  if (sc.damp) {
    // Rayleigh-like damping kd * H_el (x - x_prev) / dt (vbd_solver.py:222-223)
    const S4 u0 = ldcg4(reinterpret_cast<const S4*>(m.up) + gv);
    const Real kd = Real(sc.kd_dt);
    const Real ex = Real(uo.x - u0.x), ey = Real(uo.y - u0.y), ez = Real(uo.z - u0.z);
    G[0] += kd * (h[0] * ex + h[1] * ey + h[2] * ez);
    G[1] += kd * (h[1] * ex + h[3] * ey + h[4] * ez);
    G[2] += kd * (h[2] * ex + h[4] * ey + h[5] * ez);
#pragma unroll
    for (int i = 0; i < 6; ++i) h[i] *= (Real(1) + kd);
  }
  H[0] = h[0] + mdt2;
  H[1] = h[1];
  H[2] = h[2];
  H[3] = h[3] + mdt2;
  H[4] = h[4];
  H[5] = h[5] + mdt2;
  Real dx[3];
  if (!chol_solve3<Real>(H, G, dx)) {
    stat |= kStatGuard;
    if (!sc.strict) {
      // fallback: inertia-only Hessian (m/dt^2) I; a massless vertex stays
      const Real s = mdt2 > Real(0) ? Real(-1) / mdt2 : Real(0);
      dx[0] = G[0] * s;
      dx[1] = G[1] * s;
      dx[2] = G[2] * s;
    }
  }
  S4 un = uo;
  un.x += SReal(dx[0]);
  un.y += SReal(dx[1]);
  un.z += SReal(dx[2]);
  st.store(lv, un);
  const double c = fabs(double(dx[0] + dx[1] + dx[2]));
  if (!isfinite(c)) stat |= kStatNonFinite;
  const unsigned long long cb = conv_bits(c);
  cmax = cb > cmax ? cb : cmax;
  // the last sweep allowed: its largest |dx| component, for the
  // non-convergence report
  if (dxrec)
    atomicMax(dxrec, conv_bits(fmax(fabs(double(dx[0])),
                                    fmax(fabs(double(dx[1])), fabs(double(dx[2]))))));
}

// ---------------------------------------------------------------------------
// One warp processes one chunk (32/TPV vertices of one colour).  `st` reads
// and writes the environment's displacements by environment-local id.
// ---------------------------------------------------------------------------
template <typename Real, typename SReal, int TPV, int MAT, int FMT, class State>
__device__ __forceinline__ void process_chunk(const DevMesh& m, int vbase, const ColorInfo& ci,
                                              int q, int lane, const State& st,
                                              const StepConst& sc, unsigned long long& cmax,
                                              unsigned& stat, const real4<Real>* tab,
                                              unsigned long long* dxrec = nullptr) {
  using R4 = real4<Real>;
  using S4 = real4<SReal>;
  constexpr int CPW = 32 / TPV;
  const int vi = lane / TPV, sub = lane % TPV;
  const int gv = ci.vbegin + (q - ci.chunk_begin) * CPW + vi;
  const bool valid = gv < ci.vend;
  const int lv = gv - vbase;
  const ChunkInfo ch = m.chunk[q];
  // Every load that does not depend on another is issued here, before the
  // first use: the chunk's slot indices (all steps up to the prefetch
  // depth; the SELL blocks are padded, so every lane's load is in bounds),
  // the vertex's valence, position and inertia target.
  using RS = RawSlot<FMT>;
  constexpr int PF = Prefetch<TPV>::steps;
  const size_t base = (size_t)ch.block * 32 + lane;
  typename RS::type sl[PF];
#pragma unroll
  for (int s = 0; s < PF; ++s)
    if (s < ch.steps) sl[s] = RS::load(m, base + (size_t)s * 32);
#if VBD_CHECK_BOUNDS
  // the vertex itself: a lane with an id out of range does no work, but stays
  // in the warp for the shuffles below
  const EnvInfo eb = m.env[m.chunk_owner[q].y];
  const bool vbad = valid && (lv < 0 || lv >= eb.nsolved);
  if (vbad) stat |= kStatBounds;
#else
  constexpr bool vbad = false;
#endif
  int k = 0;
  S4 uo, tt;
  uo.x = uo.y = uo.z = uo.w = SReal(0);
  tt = uo;
  if (valid && !vbad) {
    k = __ldg(m.valence + gv);
    uo = st.load(lv);
    // ut / up are written in this launch by another block of a group: read
    // them through L2, past a possibly stale L1 line
    if (sub == 0) tt = ldcg4(reinterpret_cast<const S4*>(m.ut) + gv);
  }
  Real g[3] = {Real(0), Real(0), Real(0)};
  Real h[6] = {Real(0), Real(0), Real(0), Real(0), Real(0), Real(0)};
  // the environment's record table: shared memory (staged by the caller) or
  // global memory, read through the same generic pointer
  auto visit = [&](const int4& id) {
#if VBD_CHECK_BOUNDS
    if ((unsigned)id.x >= (unsigned)eb.nv || (unsigned)id.y >= (unsigned)eb.nv ||
        (unsigned)id.z >= (unsigned)eb.nv || (unsigned)id.w >= (unsigned)eb.nrec) {
      stat |= kStatBounds;
      return;
    }
#endif
    const R4* t = tab + 3 * (size_t)id.w;
    const R4 q0 = t[0];
    const R4 q1 = t[1];
    const R4 q2 = t[2];
    const S4 a = st.load(id.x);
    const S4 b = st.load(id.y);
    const S4 c = st.load(id.z);
    // neighbour offsets formed in the state precision, then rounded
    slot_accumulate<Real, MAT>(Real(a.x - uo.x), Real(a.y - uo.y), Real(a.z - uo.z),
                               Real(b.x - uo.x), Real(b.y - uo.y), Real(b.z - uo.z),
                               Real(c.x - uo.x), Real(c.y - uo.y), Real(c.z - uo.z), q0, q1, q2,
                               g, h);
  };
#pragma unroll
  for (int s = 0; s < PF; ++s)
    if (s < ch.steps && s * TPV + sub < k) visit(RS::unpack(sl[s]));
  for (int s = PF; s < ch.steps; ++s)
    if (s * TPV + sub < k) visit(load_slot<FMT>(m, base + (size_t)s * 32));
#pragma unroll
  for (int off = TPV / 2; off > 0; off >>= 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] += __shfl_xor_sync(0xffffffffu, g[i], off);
#pragma unroll
    for (int i = 0; i < 6; ++i) h[i] += __shfl_xor_sync(0xffffffffu, h[i], off);
  }
  if (valid && !vbad && sub == 0)
    finish_vertex<Real, SReal>(m, gv, lv, uo, tt, g, h, st, sc, cmax, stat, dxrec);
}

// ---------------------------------------------------------------------------
// Split chunks (block mode).  A colour with fewer chunks than a block has
// warps (kSplitWarps) leaves most warps idle while each busy lane walks all
// of its vertex's slot steps in sequence -- at 2 lanes per vertex up to 10
// dependent FP64 slot evaluations, ~6 us for a 3-vertex colour.  Such a
// colour instead gives each chunk W = split_ways(chunks) warps: part p of W
// takes the slot steps s = p, p + W, ...; each part's per-vertex sums (after
// the lanes-per-vertex shuffle) go to shared memory, and after a barrier one
// warp per chunk adds the W parts in part order and updates the vertices.
// W depends only on the colour's chunk count, so the arithmetic is the same
// whatever the block size or the number of blocks sharing the environment.
// ---------------------------------------------------------------------------
constexpr int kSplitWarps = 16;  // chunks x parts per colour at most

template <int TPV>
__device__ __forceinline__ int split_ways(int chunks) {
  if (chunks <= 0 || chunks * 2 > kSplitWarps) return 1;
  const int w = kSplitWarps / chunks;
  return w < Prefetch<TPV>::steps ? w : Prefetch<TPV>::steps;
}

// Floats (Real) of the per-part sums of one part: 9 per vertex of a chunk.
template <int TPV>
struct SplitBuf {
  static constexpr int per_part = 9 * (32 / TPV);
};

// Part `part` of `W` of chunk q: the slot steps s = part, part + W, ...
// summed per vertex and written to buf[9 * vertex-in-chunk + i] (g then h).
template <typename Real, typename SReal, int TPV, int MAT, int FMT, class State>
__device__ __forceinline__ void process_chunk_part(const DevMesh& m, int vbase,
                                                   const ColorInfo& ci, int q, int lane,
                                                   const State& st, unsigned& stat,
                                                   const real4<Real>* tab, int part, int W,
                                                   Real* buf) {
  using R4 = real4<Real>;
  using S4 = real4<SReal>;
  constexpr int CPW = 32 / TPV;
  const int vi = lane / TPV, sub = lane % TPV;
  const int gv = ci.vbegin + (q - ci.chunk_begin) * CPW + vi;
  const bool valid = gv < ci.vend;
  const int lv = gv - vbase;
  const ChunkInfo ch = m.chunk[q];
  const size_t base = (size_t)ch.block * 32 + lane;
#if VBD_CHECK_BOUNDS
  const EnvInfo eb = m.env[m.chunk_owner[q].y];
  const bool vbad = valid && (lv < 0 || lv >= eb.nsolved);
  if (vbad) stat |= kStatBounds;
#else
  constexpr bool vbad = false;
#endif
  int k = 0;
  S4 uo;
  uo.x = uo.y = uo.z = uo.w = SReal(0);
  if (valid && !vbad) {
    k = __ldg(m.valence + gv);
    uo = st.load(lv);
  }
  Real g[3] = {Real(0), Real(0), Real(0)};
  Real h[6] = {Real(0), Real(0), Real(0), Real(0), Real(0), Real(0)};
  for (int s = part; s < ch.steps; s += W) {
    if (s * TPV + sub >= k) continue;
    const int4 id = load_slot<FMT>(m, base + (size_t)s * 32);
#if VBD_CHECK_BOUNDS
    if ((unsigned)id.x >= (unsigned)eb.nv || (unsigned)id.y >= (unsigned)eb.nv ||
        (unsigned)id.z >= (unsigned)eb.nv || (unsigned)id.w >= (unsigned)eb.nrec) {
      stat |= kStatBounds;
      continue;
    }
#endif
    const R4* t = tab + 3 * (size_t)id.w;
    const R4 q0 = t[0];
    const R4 q1 = t[1];
    const R4 q2 = t[2];
    const S4 a = st.load(id.x);
    const S4 b = st.load(id.y);
    const S4 c = st.load(id.z);
    slot_accumulate<Real, MAT>(Real(a.x - uo.x), Real(a.y - uo.y), Real(a.z - uo.z),
                               Real(b.x - uo.x), Real(b.y - uo.y), Real(b.z - uo.z),
                               Real(c.x - uo.x), Real(c.y - uo.y), Real(c.z - uo.z), q0, q1, q2,
                               g, h);
  }
#pragma unroll
  for (int off = TPV / 2; off > 0; off >>= 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] += __shfl_xor_sync(0xffffffffu, g[i], off);
#pragma unroll
    for (int i = 0; i < 6; ++i) h[i] += __shfl_xor_sync(0xffffffffu, h[i], off);
  }
  if (sub == 0) {
#pragma unroll
    for (int i = 0; i < 3; ++i) buf[9 * vi + i] = g[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) buf[9 * vi + 3 + i] = h[i];
  }
}

// Chunk q after its W parts are in parts[w * SplitBuf<TPV>::per_part + ...]:
// the sums in part order, then the vertex updates.
template <typename Real, typename SReal, int TPV, class State>
__device__ __forceinline__ void finish_split_chunk(const DevMesh& m, int vbase,
                                                   const ColorInfo& ci, int q, int lane,
                                                   const State& st, const StepConst& sc,
                                                   unsigned long long& cmax, unsigned& stat,
                                                   unsigned long long* dxrec, const Real* parts,
                                                   int W) {
  using S4 = real4<SReal>;
  constexpr int CPW = 32 / TPV;
  if (lane >= CPW) return;  // one lane per vertex
  const int vi = lane;
  const int gv = ci.vbegin + (q - ci.chunk_begin) * CPW + vi;
  if (gv >= ci.vend) return;
  const int lv = gv - vbase;
#if VBD_CHECK_BOUNDS
  const EnvInfo eb = m.env[m.chunk_owner[q].y];
  if (lv < 0 || lv >= eb.nsolved) return;  // reported by the parts
#endif
  Real g[3], h[6];
#pragma unroll
  for (int i = 0; i < 3; ++i) g[i] = parts[9 * vi + i];
#pragma unroll
  for (int i = 0; i < 6; ++i) h[i] = parts[9 * vi + 3 + i];
  for (int w = 1; w < W; ++w) {
    const Real* p = parts + w * SplitBuf<TPV>::per_part + 9 * vi;
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] += p[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) h[i] += p[3 + i];
  }
  const S4 uo = st.load(lv);
  const S4 tt = ldcg4(reinterpret_cast<const S4*>(m.ut) + gv);
  finish_vertex<Real, SReal>(m, gv, lv, uo, tt, g, h, st, sc, cmax, stat, dxrec);
}

// ---------------------------------------------------------------------------
// Incremental potential.  Strain energy V psi(F) of one tet from one of its
// slots (any vertex of the tet gives the same F), with the same G as
// slot_accumulate:
//   SNH   psi = mu'/2 (Ic-3) - mu'/2 ln((Ic+1)/4) + lambda'/2 (J-alpha)^2
//   StVK  psi = mu E:E + lambda/2 tr(E)^2
// (the SNH form differs from mu'/2 (Ic-3) - mu'/2 ln(Ic+1) + ... by a
// constant, and its F-derivative is the P of slot_accumulate).  Used only to
// compare two configurations, so constants cancel.
// ---------------------------------------------------------------------------
template <typename Real, int MAT>
__device__ __forceinline__ Real slot_psi(Real d0x, Real d0y, Real d0z, Real d1x, Real d1y,
                                         Real d1z, Real d2x, Real d2y, Real d2z,
                                         const real4<Real>& q0, const real4<Real>& q1,
                                         const real4<Real>& q2) {
  const Real G00 = d0x * q0.x + d1x * q1.x + d2x * q2.x;
  const Real G01 = d0x * q0.y + d1x * q1.y + d2x * q2.y;
  const Real G02 = d0x * q0.z + d1x * q1.z + d2x * q2.z;
  const Real G10 = d0y * q0.x + d1y * q1.x + d2y * q2.x;
  const Real G11 = d0y * q0.y + d1y * q1.y + d2y * q2.y;
  const Real G12 = d0y * q0.z + d1y * q1.z + d2y * q2.z;
  const Real G20 = d0z * q0.x + d1z * q1.x + d2z * q2.x;
  const Real G21 = d0z * q0.y + d1z * q1.y + d2z * q2.y;
  const Real G22 = d0z * q0.z + d1z * q1.z + d2z * q2.z;
  const Real p0 = q0.w, p1 = q1.w;
  const Real t = G00 + G11 + G22;
  Real psi;
  if (MAT == kSNH) {
    const Real c00 = G11 * G22 - G12 * G21, c01 = G12 * G20 - G10 * G22,
               c02 = G10 * G21 - G11 * G20;
    const Real detG = G00 * c00 + G01 * c01 + G02 * c02;
    const Real trG2 =
        G00 * G00 + G11 * G11 + G22 * G22 + Real(2) * (G01 * G10 + G02 * G20 + G12 * G21);
    const Real nG2 = G00 * G00 + G01 * G01 + G02 * G02 + G10 * G10 + G11 * G11 + G12 * G12 +
                     G20 * G20 + G21 * G21 + G22 * G22;
    const Real Jm1 = t + Real(0.5) * (t * t - trG2) + detG;
    const Real Icm3 = Real(2) * t + nG2;
    const Real am1 = Real(0.75) * p0 / p1;  // alpha - 1 = 3/4 mu' / lambda'
    const Real r = Jm1 - am1;
    psi = Real(0.5) * p0 * (Icm3 - log1p(Real(0.25) * Icm3)) + Real(0.5) * p1 * r * r;
  } else {
    const Real E00 = G00 + Real(0.5) * (G00 * G00 + G10 * G10 + G20 * G20);
    const Real E11 = G11 + Real(0.5) * (G01 * G01 + G11 * G11 + G21 * G21);
    const Real E22 = G22 + Real(0.5) * (G02 * G02 + G12 * G12 + G22 * G22);
    const Real E01 = Real(0.5) * (G01 + G10 + G00 * G01 + G10 * G11 + G20 * G21);
    const Real E02 = Real(0.5) * (G02 + G20 + G00 * G02 + G10 * G12 + G20 * G22);
    const Real E12 = Real(0.5) * (G12 + G21 + G01 * G02 + G11 * G12 + G21 * G22);
    const Real trE = E00 + E11 + E22;
    const Real EE = E00 * E00 + E11 * E11 + E22 * E22 +
                    Real(2) * (E01 * E01 + E02 * E02 + E12 * E12);
    psi = p0 * EE + Real(0.5) * p1 * trE * trE;
  }
  return psi;
}

// Strain energies of the environment's tets (its tet list: one owner slot per
// tet with a solved vertex, the slot's G taken relative to the owner, the
// energy counted once at full weight), for the entries first, first + stride,
// ...: x = at the state `st`, y (when `pair`) = at the state shifted by the
// predicted correction (DevMesh::ws_pred, where w > 0).  The shifted
// positions are formed exactly as the warm-start stage stores them (state +
// correction in the state precision).
template <typename Real, typename SReal, int MAT, class State>
__device__ __forceinline__ double2 tet_energy(const DevMesh& m, const EnvInfo& e,
                                              const State& st, const real4<Real>* tab,
                                              int first, int stride, bool pair) {
  using R4 = real4<Real>;
  using S4 = real4<SReal>;
  auto shifted = [&](S4 v, int local_id) {
    const float4 d = m.ws_pred[e.vbase + local_id];
    if (d.w > 0.f) {
      v.x += SReal(d.x);
      v.y += SReal(d.y);
      v.z += SReal(d.z);
    }
    return v;
  };
  double acc = 0.0, accb = 0.0;
  for (int i = first; i < e.ntets; i += stride) {
    const int4 id = __ldg(m.tet_slot + e.tbase + i);
    const int o = __ldg(m.tet_owner + e.tbase + i);
    const R4* t = tab + 3 * (size_t)id.w;
    const R4 q0 = t[0], q1 = t[1], q2 = t[2];
    const S4 uo = st.load(o);
    const S4 a = st.load(id.x);
    const S4 b = st.load(id.y);
    const S4 c = st.load(id.z);
    acc += double(slot_psi<Real, MAT>(Real(a.x - uo.x), Real(a.y - uo.y), Real(a.z - uo.z),
                                      Real(b.x - uo.x), Real(b.y - uo.y), Real(b.z - uo.z),
                                      Real(c.x - uo.x), Real(c.y - uo.y), Real(c.z - uo.z), q0,
                                      q1, q2));
    if (pair) {
      const S4 uob = shifted(uo, o);
      const S4 ab = shifted(a, id.x), bb = shifted(b, id.y), cb = shifted(c, id.z);
      accb += double(slot_psi<Real, MAT>(
          Real(ab.x - uob.x), Real(ab.y - uob.y), Real(ab.z - uob.z), Real(bb.x - uob.x),
          Real(bb.y - uob.y), Real(bb.z - uob.z), Real(cb.x - uob.x), Real(cb.y - uob.y),
          Real(cb.z - uob.z), q0, q1, q2));
    }
  }
  return make_double2(acc, accb);
}

// Inertia energies m/(2 dt^2) |x - ut|^2 of the environment's solved
// vertices first, first + stride, ...: x = the state `st`, or (shifted) the
// state plus the predicted correction.
template <typename SReal, class State>
__device__ __forceinline__ double inertia_energy(const DevMesh& m, const EnvInfo& e,
                                                 const State& st, const StepConst& sc,
                                                 int first, int stride, bool shifted) {
  using S4 = real4<SReal>;
  double acc = 0.0;
  for (int i = first; i < e.nsolved; i += stride) {
    S4 u = st.load(i);
    if (shifted) {
      const float4 d = m.ws_pred[e.vbase + i];
      if (d.w > 0.f) {
        u.x += SReal(d.x);
        u.y += SReal(d.y);
        u.z += SReal(d.z);
      }
    }
    // ut is written in this launch by another block of a group: through L2
    const S4 tt = ldcg4(reinterpret_cast<const S4*>(m.ut) + e.vbase + i);
    const double dx = double(u.x - tt.x), dy = double(u.y - tt.y), dz = double(u.z - tt.z);
    acc += 0.5 * double(tt.w) * sc.inv_dt2 * (dx * dx + dy * dy + dz * dz);
  }
  return acc;
}

// Inertia target and initial guess (position_initialization,
// vbd_solver.py:277-292): ut = u + dt v + dt^2 g (w keeps the lumped mass),
// up = u (written when write_back), and active vertices start from ut.
template <typename Real>
__device__ __forceinline__ real4<Real> begin_vertex(const DevMesh& m, int gv, bool active,
                                                    const StepConst& sc, bool write_back) {
  using R4 = real4<Real>;
  R4* U = reinterpret_cast<R4*>(m.u);
  R4* UT = reinterpret_cast<R4*>(m.ut);
  R4* UP = reinterpret_cast<R4*>(m.up);
  const R4* VEL = reinterpret_cast<const R4*>(m.vel);
  const R4 u0 = U[gv];
  const R4 v0 = VEL[gv];
  R4 tt = UT[gv];
  const Real dt = Real(sc.dt), dt2 = Real(sc.dt2);
  tt.x = u0.x + v0.x * dt + Real(sc.g[0]) * dt2;
  tt.y = u0.y + v0.y * dt + Real(sc.g[1]) * dt2;
  tt.z = u0.z + v0.z * dt + Real(sc.g[2]) * dt2;
  if (write_back) {
    UT[gv] = tt;
    UP[gv] = u0;
  }
  R4 un = u0;
  if (active) {
    un.x = tt.x;
    un.y = tt.y;
    un.z = tt.z;
  }
  return un;
}

// Velocity update (vbd_solver.py:609): v = (x_new - x_old) / dt.
template <typename Real>
__device__ __forceinline__ void end_vertex(const DevMesh& m, int gv, const real4<Real>& un,
                                           const StepConst& sc) {
  using R4 = real4<Real>;
  const R4 u0 = reinterpret_cast<const R4*>(m.up)[gv];
  R4 v;
  const Real idt = Real(1.0 / sc.dt);
  v.x = (un.x - u0.x) * idt;
  v.y = (un.y - u0.y) * idt;
  v.z = (un.z - u0.z) * idt;
  v.w = Real(0);
  reinterpret_cast<R4*>(m.vel)[gv] = v;
}

// ---------------------------------------------------------------------------
// Runtime (precision, material, record format, lanes per vertex) -> template
// instantiation: calls f.template run<Real, SReal, TPV, MAT, FMT>().
template <typename Real, typename SReal, int MAT, int FMT, class F>
cudaError_t dispatch_tpv(int tpv, F& f) {
  switch (tpv) {
    case 2: return f.template run<Real, SReal, 2, MAT, FMT>();
    case 4: return f.template run<Real, SReal, 4, MAT, FMT>();
    case 8: return f.template run<Real, SReal, 8, MAT, FMT>();
    case 16: return f.template run<Real, SReal, 16, MAT, FMT>();
    default: return cudaErrorInvalidValue;
  }
}

template <typename Real, typename SReal, int MAT, class F>
cudaError_t dispatch_fmt(int fmt, int tpv, F& f) {
  if (fmt == kFmtIdx16) return dispatch_tpv<Real, SReal, MAT, kFmtIdx16>(tpv, f);
  if (fmt == kFmtIdx32) return dispatch_tpv<Real, SReal, MAT, kFmtIdx32>(tpv, f);
  return cudaErrorInvalidValue;
}

template <typename Real, typename SReal, class F>
cudaError_t dispatch_mat(int material, int fmt, int tpv, F& f) {
  return material == kSNH ? dispatch_fmt<Real, SReal, kSNH>(fmt, tpv, f)
                          : dispatch_fmt<Real, SReal, kStVK>(fmt, tpv, f);
}

template <class F>
cudaError_t dispatch(int prec, int material, int fmt, int tpv, F& f) {
  switch (prec) {
    case 0: return dispatch_mat<float, float>(material, fmt, tpv, f);
    case 1: return dispatch_mat<float, double>(material, fmt, tpv, f);
    case 2: return dispatch_mat<double, double>(material, fmt, tpv, f);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace vbd
