// Host side of libvbd_b200.so: mesh setup, device layout, the conditional
// CUDA-graph sweep loop and the C ABI declared in include/vbd_b200.h.
//
// Setup restates VBDSolver.__init__ (mmichelis/WarpVBD src/vbd_solver.py:366-498)
// natively: Lame parameters (:345-362), Dm^-1 / volume / mass per tet
// (:295-343), the greedy colouring (src/coloring.py:24-72) and the
// vertex -> tet adjacency (:485-498).  Instead of the reference's padded
// [n_colors, max_group] colour table and [V, 20] adjacency it renumbers the
// vertices colour by colour and stores one record per incident (vertex, tet)
// pair in a SELL-32 layout (see vbd_internal.h).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/vbd_b200.h"
#include "vbd_internal.h"
#include "vbd_launch.h"
#include "vbd_persist.h"
#include "vbd_noalloc.h"
#include "vbd_setup.h"
#include "vbd_warmstart.h"

using namespace vbd;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CUDA_TRY(expr)                                                                  \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess)                                                              \
      return fail(VBD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));    \
  } while (0)

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t count) {
    n = count;
    return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1));
  }
  cudaError_t upload(const std::vector<T>& h, cudaStream_t s) {
    cudaError_t e = alloc(h.size());
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpyAsync(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// ---------------------------------------------------------------------------
// Greedy colouring (coloring.py:24-72): vertices in index order, each takes
// the smallest colour not used by an already-coloured vertex sharing a tet.
// Vertex count = max(tets)+1.  Returns the colour count or -1 (> 256 colours).
// ---------------------------------------------------------------------------
int greedy_coloring(const int32_t* tets, int T, int nv, int32_t* col) {
  std::vector<int> off(nv + 1, 0), inc(4 * (size_t)T);
  for (int i = 0; i < 4 * T; ++i) off[tets[i] + 1]++;
  for (int v = 0; v < nv; ++v) off[v + 1] += off[v];
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int t = 0; t < T; ++t)
    for (int q = 0; q < 4; ++q) inc[fill[tets[4 * t + q]]++] = t;
  std::fill(col, col + nv, -1);
  int ncol = 0;
  uint8_t used[257];
  for (int v = 0; v < nv; ++v) {
    std::memset(used, 0, sizeof used);
    for (int s = off[v]; s < off[v + 1]; ++s) {
      const int32_t* e = tets + 4 * (size_t)inc[s];
      for (int q = 0; q < 4; ++q) {
        const int n = e[q];
        if (n != v && col[n] >= 0) used[col[n]] = 1;
      }
    }
    int c = 0;
    while (c < 256 && used[c]) ++c;
    if (c == 256) return -1;
    col[v] = c;
    ncol = std::max(ncol, c + 1);
  }
  return ncol;
}

struct TetData {
  std::vector<double> b;  // [T][4][3] shape-function gradients
  std::vector<double> p;  // [T][3] (V*mu, V*lambda, alpha)
  std::vector<double> mass, vol;
  const double *E = nullptr, *nu = nullptr, *rho = nullptr;  // caller's per-tet arrays
};

int build_tet_data(const double* X, const int32_t* tets, int T, const double* rho,
                   const double* E, const double* nu, int material, TetData& td) {
  td.b.assign((size_t)T * 12, 0.0);
  td.p.assign((size_t)T * 3, 0.0);
  td.mass.assign(T, 0.0);
  td.vol.assign(T, 0.0);
  td.E = E;
  td.nu = nu;
  td.rho = rho;
  for (int t = 0; t < T; ++t) {
    const int32_t* e = tets + 4 * (size_t)t;
    double D[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) D[r * 3 + c] = X[3 * (size_t)e[c] + r] - X[3 * (size_t)e[3] + r];
    const double det = D[0] * (D[4] * D[8] - D[5] * D[7]) - D[1] * (D[3] * D[8] - D[5] * D[6]) +
                       D[2] * (D[3] * D[7] - D[4] * D[6]);
    if (!(det != 0.0) || !std::isfinite(det))
      return fail(VBD_ERR_SINGULAR_DM, "tet " + std::to_string(t) + " has zero rest volume");
    const double s = 1.0 / det;
    double I[9];
    I[0] = (D[4] * D[8] - D[5] * D[7]) * s;
    I[1] = (D[2] * D[7] - D[1] * D[8]) * s;
    I[2] = (D[1] * D[5] - D[2] * D[4]) * s;
    I[3] = (D[5] * D[6] - D[3] * D[8]) * s;
    I[4] = (D[0] * D[8] - D[2] * D[6]) * s;
    I[5] = (D[2] * D[3] - D[0] * D[5]) * s;
    I[6] = (D[3] * D[7] - D[4] * D[6]) * s;
    I[7] = (D[1] * D[6] - D[0] * D[7]) * s;
    I[8] = (D[0] * D[4] - D[1] * D[3]) * s;
    double* b = &td.b[(size_t)t * 12];
    for (int q = 0; q < 3; ++q)
      for (int c = 0; c < 3; ++c) b[q * 3 + c] = I[q * 3 + c];  // row q of Dm^-1
    for (int c = 0; c < 3; ++c) b[9 + c] = -(I[c] + I[3 + c] + I[6 + c]);
    const double vol = std::fabs(det) / 6.0;
    td.mass[t] = rho[t] * vol;
    td.vol[t] = vol;
    const double mu = E[t] / (2.0 * (1.0 + nu[t]));
    const double lam = (E[t] * nu[t]) / ((1.0 + nu[t]) * (1.0 - 2.0 * nu[t]));
    double* p = &td.p[(size_t)t * 3];
    if (material == kSNH) {
      const double mu2 = 4.0 * mu / 3.0, lam2 = lam + 5.0 * mu / 6.0;
      p[0] = vol * mu2;
      p[1] = vol * lam2;
      p[2] = 1.0 + 0.75 * mu2 / lam2;
    } else {
      p[0] = vol * mu;
      p[1] = vol * lam;
      p[2] = 0.0;
    }
  }
  return VBD_OK;
}

// Unique slot-record values (b_n0, p0, b_n1, p1, b_n2, p2).  Two slots share an
// entry when their values are bitwise equal after conversion to the solver's
// arithmetic precision, so sharing never changes a result.  Voxel meshes have
// a handful of tet shapes, so thousands of slots map to one entry.
struct RecordTable {
  bool fp64 = false;
  std::vector<double> vals;  // 12 per entry
  struct Key {
    uint64_t w[12];
    bool operator==(const Key& o) const { return std::memcmp(w, o.w, sizeof w) == 0; }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      uint64_t h = 1469598103934665603ull;
      for (uint64_t x : k.w) h = (h ^ x) * 1099511628211ull;
      return (size_t)(h ^ (h >> 29));
    }
  };
  std::unordered_map<Key, int, KeyHash> index;

  int insert(const double* v) {
    Key k;
    for (int i = 0; i < 12; ++i) {
      if (fp64) {
        std::memcpy(&k.w[i], &v[i], 8);
      } else {
        const float f = (float)v[i];
        uint32_t b;
        std::memcpy(&b, &f, 4);
        k.w[i] = b;
      }
    }
    auto it = index.find(k);
    if (it != index.end()) return it->second;
    const int id = (int)(vals.size() / 12);
    vals.insert(vals.end(), v, v + 12);
    index.emplace(k, id);
    return id;
  }
  int size() const { return (int)(vals.size() / 12); }
};

struct Layout {
  std::vector<EnvInfo> env;
  std::vector<ColorInfo> color;
  std::vector<ChunkInfo> chunk;
  std::vector<int4> rec_idx;  // (n0, n1, n2, record id)
  std::vector<int4> tet_slot;  // owner slot of every tet with a solved vertex
  std::vector<int> tet_owner;  // its owner's environment-local id
  RecordTable table;
  std::vector<int> valence;     // new id
  std::vector<double> mass;     // new id
  std::vector<float> wstat;     // new id, 4 per vertex: warm-start vertex constants
  std::vector<int2> chunk_owner;  // (colour index, environment) per chunk
  std::vector<int> new_of_old;
  std::vector<int32_t> table0;  // env 0 colour table (original ids)
  int table_colors = 0, table_max_group = 0;
  int max_valence = 0, max_colors = 0, max_env_vertices = 0, max_env_records = 0;
  long long n_slots = 0;
};

// `greedy`: the greedy colouring of the whole mesh, already computed (on the
// GPU); every environment's colours are its slice (environments share no tet,
// so a vertex's lower neighbours all lie in its environment).  Null: the
// colouring is computed here per environment.
int build_layout(const double* X, int V, const int32_t* tets, int T, const uint8_t* active,
                 const std::vector<int>& voff, const std::vector<int>& toff,
                 const int32_t* coloring, const TetData& td, int tpv, bool order_index,
                 Layout& L, const int32_t* greedy = nullptr) {
  const int n_env = (int)voff.size() - 1;
  const int cpw = 32 / tpv;
  L.new_of_old.assign(V, -1);
  L.valence.assign(V, 0);
  L.mass.assign(V, 0.0);
  L.wstat.assign(4 * (size_t)V, 0.0f);
  int block_count = 0;
  for (int e = 0; e < n_env; ++e) {
    const int vo = voff[e], vn = voff[e + 1] - voff[e];
    const int to = toff[e], tn = toff[e + 1] - toff[e];
    if (vn < 0 || tn < 0) return fail(VBD_ERR_INVALID_ARG, "environment offsets decrease");
    std::vector<int32_t> lt(4 * (size_t)tn);
    int nv_col = 0;
    for (size_t i = 0; i < lt.size(); ++i) {
      const int g = tets[4 * (size_t)to + i];
      if (g < vo || g >= vo + vn)
        return fail(VBD_ERR_INVALID_ARG, "tet " + std::to_string(to + i / 4) +
                                             " references a vertex outside its environment");
      lt[i] = g - vo;
      nv_col = std::max(nv_col, lt[i] + 1);
    }
    // colours of the local vertices (-1: not coloured)
    std::vector<int32_t> col(vn, -1);
    int ncol = 0;
    if (coloring && n_env == 1) {
      for (int v = 0; v < nv_col; ++v) {
        col[v] = coloring[v];
        if (col[v] < 0 || col[v] >= 256) return fail(VBD_ERR_INVALID_ARG, "bad colour value");
        ncol = std::max(ncol, col[v] + 1);
      }
      // vertices of one colour must not share a tet, or their updates race
      for (int t = 0; t < tn; ++t)
        for (int a = 0; a < 4; ++a)
          for (int b = a + 1; b < 4; ++b)
            if (col[lt[4 * (size_t)t + a]] == col[lt[4 * (size_t)t + b]])
              return fail(VBD_ERR_INVALID_ARG,
                          "coloring gives two vertices of tet " + std::to_string(t) +
                              " the same colour");
    } else if (tn > 0 && greedy) {
      // as the per-environment pass colours them: ids 0 .. max local id
      for (int v = 0; v < nv_col; ++v) {
        col[v] = greedy[vo + v];
        ncol = std::max(ncol, col[v] + 1);
      }
    } else if (tn > 0) {
      ncol = greedy_coloring(lt.data(), tn, nv_col, col.data());
      if (ncol < 0) return fail(VBD_ERR_TOO_MANY_COLORS, "Exceeded maximum number of colors");
    }
    // incident tets, ascending tet id
    std::vector<int> off(vn + 1, 0), inc(4 * (size_t)tn), loc(4 * (size_t)tn);
    for (size_t i = 0; i < lt.size(); ++i) off[lt[i] + 1]++;
    for (int v = 0; v < vn; ++v) off[v + 1] += off[v];
    {
      std::vector<int> fill(off.begin(), off.end() - 1);
      for (int t = 0; t < tn; ++t)
        for (int q = 0; q < 4; ++q) {
          const int v = lt[4 * (size_t)t + q];
          inc[fill[v]] = t;
          loc[fill[v]] = q;
          fill[v]++;
        }
    }
    // colour table of environment 0 in the reference layout
    if (e == 0) {
      std::vector<std::vector<int>> groups(ncol);
      for (int v = 0; v < nv_col; ++v)
        if (col[v] >= 0) groups[col[v]].push_back(vo + v);
      int mg = 0;
      for (auto& g : groups) mg = std::max(mg, (int)g.size());
      L.table_colors = ncol;
      L.table_max_group = mg;
      L.table0.assign((size_t)ncol * mg, -1);
      for (int c = 0; c < ncol; ++c)
        for (size_t i = 0; i < groups[c].size(); ++i) L.table0[(size_t)c * mg + i] = groups[c][i];
    }
    // classify and order
    std::vector<std::vector<int>> solved(ncol);
    std::vector<int> freev, fixedv;
    for (int v = 0; v < vn; ++v) {
      const bool act = active ? active[vo + v] != 0 : true;
      const int k = off[v + 1] - off[v];
      if (!act)
        fixedv.push_back(v);
      else if (col[v] >= 0 && k > 0)
        solved[col[v]].push_back(v);
      else
        freev.push_back(v);
      L.max_valence = std::max(L.max_valence, k);
    }
    EnvInfo ei{};
    ei.vbase = vo;
    ei.nv = vn;
    ei.cbase = (int)L.color.size();
    int next = 0;
    std::vector<int> new_local(vn, -1);
    for (int c = 0; c < ncol; ++c) {
      auto& g = solved[c];
      if (g.empty()) continue;
      if (!order_index)
        std::stable_sort(g.begin(), g.end(), [&](int a, int b) {
          return (off[a + 1] - off[a]) > (off[b + 1] - off[b]);
        });
      ColorInfo ci{};
      ci.vbegin = vo + next;
      for (int v : g) new_local[v] = next++;
      ci.vend = vo + next;
      ci.chunk_begin = (int)L.chunk.size();
      const int ng = (int)g.size();
      for (int base = 0; base < ng; base += cpw) {
        int kmax = 0;
        for (int i = base; i < std::min(ng, base + cpw); ++i)
          kmax = std::max(kmax, off[g[i] + 1] - off[g[i]]);
        ChunkInfo ch{};
        ch.block = block_count;
        ch.steps = (kmax + tpv - 1) / tpv;
        block_count += ch.steps;
        L.chunk.push_back(ch);
      }
      ci.chunk_end = (int)L.chunk.size();
      L.color.push_back(ci);
    }
    ei.nsolved = next;
    for (int v : freev) new_local[v] = next++;
    ei.nact = next;
    for (int v : fixedv) new_local[v] = next++;
    ei.ncolors = (int)L.color.size() - ei.cbase;
    L.env.push_back(ei);
    L.max_colors = std::max(L.max_colors, ei.ncolors);
    L.max_env_vertices = std::max(L.max_env_vertices, vn);
    for (int v = 0; v < vn; ++v) {
      const int gnew = vo + new_local[v];
      L.new_of_old[vo + v] = gnew;
      const int k = off[v + 1] - off[v];
      L.valence[gnew] = k;
      double m = 0.0, hs = 0.0, logE = 0.0, rho = 0.0, nu = 0.0;
      for (int s = off[v]; s < off[v + 1]; ++s) {
        const int t = to + inc[s];
        m += td.mass[t] / 4.0;
        hs += std::cbrt(6.0 * td.vol[t]);
        logE += std::log10(td.E[t]);
        rho += td.rho[t];
        nu += td.nu[t];
      }
      L.mass[gnew] = m;
      // warm-start vertex constants: local length scale h (mean cube root of
      // 6 V over the incident tets), log10(E / (rho h^2)), nu, valence / 20
      float* w4 = &L.wstat[4 * (size_t)gnew];
      if (k > 0) {
        const double h = hs / k;
        w4[0] = (float)h;
        w4[1] = (float)(logE / k - std::log10(rho / k * h * h));
        w4[2] = (float)(nu / k);
        w4[3] = (float)(k / 20.0);
      } else {
        w4[0] = 1.0f;
        w4[1] = w4[2] = w4[3] = 0.0f;
      }
    }
    for (int c = ei.cbase; c < ei.cbase + ei.ncolors; ++c)
      for (int q = L.color[c].chunk_begin; q < L.color[c].chunk_end; ++q)
        L.chunk_owner.push_back(make_int2(c, e));
    // slot records: (n0, n1, n2, record id) per slot, the record values in a
    // table of this environment shared by every slot with the same values in
    // the solver precision (record ids are environment-local, so a block can
    // stage its environment's table in shared memory)
    L.rec_idx.resize((size_t)block_count * 32, make_int4(0, 0, 0, 0));
    RecordTable etab;
    etab.fp64 = L.table.fp64;
    std::vector<std::pair<int, int4>> tlist;  // (owner, owner slot) per tet
    std::vector<int> old_of_new_local(vn);
    for (int v = 0; v < vn; ++v) old_of_new_local[new_local[v]] = v;
    for (int ci_i = ei.cbase; ci_i < ei.cbase + ei.ncolors; ++ci_i) {
      const ColorInfo ci = L.color[ci_i];
      for (int q = ci.chunk_begin; q < ci.chunk_end; ++q) {
        const ChunkInfo ch = L.chunk[q];
        for (int lane = 0; lane < 32; ++lane) {
          const int vi = lane / tpv, sub = lane % tpv;
          const int gv = ci.vbegin + (q - ci.chunk_begin) * cpw + vi;
          if (gv >= ci.vend) continue;
          const int ov = old_of_new_local[gv - vo];
          const int k = off[ov + 1] - off[ov];
          for (int s = 0; s < ch.steps; ++s) {
            const int j = s * tpv + sub;
            if (j >= k) break;
            const int t = to + inc[off[ov] + j];
            const int a = loc[off[ov] + j];
            const size_t blk = (size_t)ch.block + s;
            int ids[3];
            double val[12];
            const double* bt = &td.b[(size_t)t * 12];
            const double* pt = &td.p[(size_t)t * 3];
            int n = 0, solved_in_tet = 0, owner = vn;
            for (int qq = 0; qq < 4; ++qq) {
              const int nl = new_local[tets[4 * (size_t)t + qq] - vo];
              if (nl < ei.nsolved) {
                ++solved_in_tet;
                owner = std::min(owner, nl);
              }
              if (qq == a) continue;
              ids[n] = new_local[tets[4 * (size_t)t + qq] - vo];
              val[4 * n + 0] = bt[qq * 3 + 0];
              val[4 * n + 1] = bt[qq * 3 + 1];
              val[4 * n + 2] = bt[qq * 3 + 2];
              val[4 * n + 3] = pt[n];
              ++n;
            }
            // 4th value of the last plane: this slot's share of the tet's
            // strain energy, so that summing over slots counts every tet with
            // a solved vertex once (incremental-potential evaluation)
            val[11] = 1.0 / solved_in_tet;
            const int rid = etab.insert(val);
            L.rec_idx[blk * 32 + lane] = make_int4(ids[0], ids[1], ids[2], rid);
            if (owner == gv - vo) tlist.emplace_back(owner, make_int4(ids[0], ids[1], ids[2], rid));
            L.n_slots++;
          }
        }
      }
    }
    L.env.back().rbase = L.table.size();
    L.env.back().nrec = etab.size();
    // the tet list in owner order (neighbouring entries read nearby state)
    std::stable_sort(tlist.begin(), tlist.end(),
                     [](const std::pair<int, int4>& a, const std::pair<int, int4>& b) {
                       return a.first < b.first;
                     });
    L.env.back().tbase = (int)L.tet_slot.size();
    L.env.back().ntets = (int)tlist.size();
    for (const auto& x : tlist) {
      L.tet_owner.push_back(x.first);
      L.tet_slot.push_back(x.second);
    }
    L.table.vals.insert(L.table.vals.end(), etab.vals.begin(), etab.vals.end());
    L.max_env_records = std::max(L.max_env_records, etab.size());
  }
  return VBD_OK;
}

}  // namespace

struct vbd_solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool fp64 = false;     // arithmetic and slot records in double
  bool state64 = false;  // state vectors in double
  int prec = 0;          // 0 fp32, 1 mixed (fp64 state, fp32 arithmetic), 2 fp64
  int material = 0, mode = 0, tpv = 4, threads = 256, flags = 0;
  int V = 0, T = 0, n_env = 0;
  double kd = 0.0, g[3] = {0, 0, 0};
  size_t real4_bytes = 16;
  Layout L;
  size_t smem_bytes = 0;
  long long n_records = 0;
  long long device_bytes = 0;
  // device
  DevBuf<EnvInfo> d_env;
  DevBuf<ColorInfo> d_color;
  DevBuf<ChunkInfo> d_chunk;
  DevBuf<int4> d_rec_idx;
  DevBuf<ushort4> d_rec_idx16;
  DevBuf<int4> d_tet_slot;
  DevBuf<int> d_tet_owner;
  // vbd_step_batched_to: device-mapped pointer of the caller's page-locked
  // output array during the enqueue of that step, else null
  double* host_out = nullptr;
  // vbd_incremental_potential: candidate state (Real4) and per-env results
  DevBuf<unsigned char> d_xeval;
  DevBuf<double> d_pot;
  DevBuf<unsigned char> d_rec_tab;
  int fmt = kFmtIdx32;
  DevBuf<int> d_valence, d_map, d_iters;
  DevBuf<unsigned> d_status;
  // per env: largest |dx| component of the last allowed sweep (DevMesh::dxmax)
  DevBuf<unsigned long long> d_dxmax;
  unsigned long long* h_dxmax = nullptr;  // pinned
  std::vector<double> final_dx;           // per env, of the last step; NaN if it converged
  DevBuf<unsigned char> d_u, d_ut, d_up, d_vel;
  DevBuf<double> d_X, d_io, d_tol;
  DevBuf<StepParams> d_params;
  DevBuf<LoopControl> d_ctl;
  DevBuf<PersistCtl> d_pctl;  // persistent mode
  DevBuf<double> d_pparts;    // persistent mode: warm-start energy partial sums
  int persist_blocks = 0;
  // persistent mode: neighbour-scoped readiness between colours (PersistNbr)
  DevBuf<int> d_nbr_off, d_nbr_idx;
  DevBuf<unsigned long long> d_epoch;
  bool persist_scoped = false;
  PersistLimits wait_limits{1ll << 26, 2000000000ull};  // every grid-barrier wait
  // block-mode work map: (environment, rank, group size) per thread block
  int cluster = 1;           // blocks per cluster = group size of a split environment
  bool replan = false;       // re-plan from the measured sweep counts after each step
  int capacity_blocks = 0;   // resident blocks on the device for this launch shape
  // tiered mode: clusters of the split / wide size that can be resident at
  // once (a cluster needs its blocks in one GPC, so fewer than blocks / size)
  int max_clusters_split = 0, max_clusters_wide = 0;
  std::vector<double> env_work;  // incident slots per environment
  // sweeps per environment for the plan.  Plain VBD's counts change slowly
  // from step to step: env_sweeps_decay = max(last, 0.95 x previous).  The
  // learned warm start's vary (consecutive-step correlation about 0.7 on the
  // 256-environment batch): the maximum of the last kSweepWindow counts for
  // the length of its job (an environment whose count jumps must not run
  // alone on one block) and their running mean for the total block time;
  // env_sweep_ring holds the window
  static constexpr int kSweepWindow = 8;
  std::vector<double> env_sweeps, env_sweeps_mean, env_sweeps_decay;
  std::vector<int> env_sweep_ring;
  int ring_pos = 0;
  std::vector<int4> work;
  DevBuf<int4> d_work;
  // tiered block mode (VBD_TIERED): `work` lists the split environments
  // (heavy launch), `work2` the others, one block each (light launch)
  bool tiered = false;
  int heavy_threads = 512;
  size_t smem_per_vertex = 24;
  size_t rec_bytes = 48;      // one record: 3 Real4
  bool tab_in_smem = false;   // kernels stage the record table in shared memory
  size_t persist_smem = 0;    // persistent mode: bytes of the staged table
  size_t smem_heavy = 0, smem_light = 0;
  std::vector<int4> work2;
  DevBuf<int4> d_work2;
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // wide tier (VBD_TIERED_WIDE): `work3` lists the environments split over a
  // cluster of cluster_wide blocks (third launch, stream aux2)
  int cluster_wide = 0;
  size_t smem_wide = 0;
  std::vector<int4> work3;
  DevBuf<int4> d_work3;
  cudaStream_t aux2 = nullptr;
  cudaEvent_t ev_join2 = nullptr;
  // timing of the step kernels of every step (events around them on the
  // solver's stream) and the number of kernels the step launched
  cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr;
  int launches_pending = 0, launches_last = 0;
  float kernel_ms_last = 0.f;
  // block-mode timeline (vbd_set_trace): 4 words per block of the step's
  // launches: wide tier, split (or single) launch, then the light launch
  bool trace_on = false;
  DevBuf<unsigned long long> d_trace;
  int trace_pending = 0, trace_last = 0;
  // learned warm start
  DevBuf<float4> d_wstat;
  DevBuf<int2> d_chunk_owner;
  DevBuf<float> d_feat;           // [V][24], allocated on first use
  DevBuf<float> d_wpack;          // [V][6] packed fp32 displacement / velocity (features)
  DevBuf<float4> d_pred;          // [V]
  DevBuf<unsigned char> d_wbf;    // bf16 network parameters
  DevBuf<float> d_wparams;        // fp32 staging for the conversion
  DevBuf<float> d_wnorm;          // input / target normalisation (50 floats)
  DevBuf<unsigned> d_ws_err;      // set by the tensor-core inference when a wait ran out
  unsigned* h_ws_err = nullptr;   // pinned copy, read back with every warm step
  bool warm = false;
  bool ws_history = false;        // the previous step's inertia target is in ut
  // pinned host
  int* h_iters = nullptr;
  unsigned* h_status = nullptr;
  StepParams* h_params = nullptr;
  LoopControl* h_ctl = nullptr;
  StepParams cur_params{};
  bool params_valid = false;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int last_status = VBD_OK;
  bool pending = false;

  DevMesh mesh() const {
    DevMesh m{};
    m.env = d_env.p;
    m.color = d_color.p;
    m.chunk = d_chunk.p;
    m.rec_idx = d_rec_idx.p;
    m.rec_idx16 = d_rec_idx16.p;
    m.rec_tab = d_rec_tab.p;
    m.tet_slot = d_tet_slot.p;
    m.tet_owner = d_tet_owner.p;
    m.host_out = host_out;
    m.map = d_map.p;
    m.rest = d_X.p;
    m.fmt = fmt;
    m.wstat = d_wstat.p;
    m.chunk_owner = d_chunk_owner.p;
    m.ws_pred = warm ? d_pred.p : nullptr;
    m.valence = d_valence.p;
    m.u = d_u.p;
    m.ut = d_ut.p;
    m.up = d_up.p;
    m.vel = d_vel.p;
    m.iters = d_iters.p;
    m.status = d_status.p;
    m.dxmax = d_dxmax.p;
    m.n_env = n_env;
    m.n_vertices = V;
    return m;
  }
};

namespace {

void free_solver(vbd_solver* s) {
  if (!s) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->d_env.release();
  s->d_color.release();
  s->d_chunk.release();
  s->d_rec_idx.release();
  s->d_rec_idx16.release();
  s->d_tet_slot.release();
  s->d_tet_owner.release();
  s->d_xeval.release();
  s->d_pot.release();
  s->d_rec_tab.release();
  s->d_valence.release();
  s->d_map.release();
  s->d_iters.release();
  s->d_status.release();
  s->d_dxmax.release();
  s->d_u.release();
  s->d_ut.release();
  s->d_up.release();
  s->d_vel.release();
  s->d_X.release();
  s->d_io.release();
  s->d_tol.release();
  s->d_work.release();
  s->d_work2.release();
  s->d_work3.release();
  s->d_trace.release();
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_k0) cudaEventDestroy(s->ev_k0);
  if (s->ev_k1) cudaEventDestroy(s->ev_k1);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->aux) {
    cudaStreamSynchronize(s->aux);
    cudaStreamDestroy(s->aux);
  }
  if (s->ev_join2) cudaEventDestroy(s->ev_join2);
  if (s->aux2) {
    cudaStreamSynchronize(s->aux2);
    cudaStreamDestroy(s->aux2);
  }
  s->d_wstat.release();
  s->d_chunk_owner.release();
  s->d_feat.release();
  s->d_wpack.release();
  s->d_pred.release();
  s->d_wbf.release();
  s->d_wparams.release();
  s->d_wnorm.release();
  s->d_ws_err.release();
  s->d_params.release();
  s->d_ctl.release();
  s->d_pctl.release();
  s->d_pparts.release();
  s->d_nbr_off.release();
  s->d_nbr_idx.release();
  s->d_epoch.release();
  if (s->h_iters) cudaFreeHost(s->h_iters);
  if (s->h_status) cudaFreeHost(s->h_status);
  if (s->h_dxmax) cudaFreeHost(s->h_dxmax);
  if (s->h_params) cudaFreeHost(s->h_params);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_ws_err) cudaFreeHost(s->h_ws_err);
  if (s->stream) cudaStreamDestroy(s->stream);
  cudaSetDevice(prev);
  delete s;
}

// NVTX range over a host-side scope (header-only NVTX v3: a no-op unless a
// profiler is attached).  Names: "vbd_step" (enqueue, and the wait when the
// call blocks), "vbd_warm_start" (feature and inference launches),
// "vbd_step_kernels" (the step launches), "vbd_sync".
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Dynamic shared memory of a block-mode block running environment `ei`: its
// packed xyz state, then (with_tab) its record table, 16-byte aligned.
size_t env_smem(const vbd_solver* s, const EnvInfo& ei, bool with_tab) {
  const size_t state = ((size_t)ei.nv * s->smem_per_vertex + 15) / 16 * 16;
  return with_tab ? state + (size_t)ei.nrec * s->rec_bytes : state;
}

// Block-mode work map.  Each environment's duration is predicted from its
// slot count and its sweep count (1 before the first step) with a per-sweep
// cost model measured on B200 at 512 threads, in units of one slot visit of
// a single block:
//   one block              sweeps * (slots + A1)
//   split over C blocks    sweeps * (slots / C + I_C)
//                          (I_C interpolated between C = 2, 4, 8, 16)
// fitted to single environments of 7K, 27K and 68K slots on 1-16 blocks:
//   mixed precision, 4 lanes per vertex: A1 = 8300, I_C = 10300 / 11200 /
//     12200 / 16500 (1.72 ns per slot visit; the 68K-slot environment 129 /
//     78 / 49 / 35 / 36 us per sweep on 1 / 2 / 4 / 8 / 16 blocks)
//   fp64, 2 lanes per vertex: A1 = 10200, I_C = 12900 / 13500 / 13900 / 18000
//     (2.34 ns per slot visit; 183 / 112 / 67 / 54 / 55 us)
// (the fixed part is the per-colour barrier and dependency chain; at 16
// blocks every store also goes to 15 replicas, which I_16 absorbs).  With cluster > 1 the longest environments may each take a whole
// cluster (group = cluster); the split set is the one with the smallest
// predicted step time, the largest of (longest split environment, longest
// single-block environment, all block time / resident blocks).  With the
// learned warm start, job lengths use the high sweep estimate (the maximum
// of the last eight steps) and the total block time the mean, both plus the
// cost of its energy checks (0.7 sweeps): its counts vary from step to step,
// and an environment whose count jumps while it runs alone on one block sets
// the step time.  Blocks are listed longest first, which the block scheduler
// then starts first.
// I_C of the duration model: measured at C = 2, 4, 8, 16, linear in C between
// those points (C = 3, 5-7, 9-15).
double split_overhead(int C, bool fp64) {
  static const double c[4] = {2.0, 4.0, 8.0, 16.0};
  static const double vm[4] = {10300.0, 11200.0, 12200.0, 16500.0};
  static const double vd[4] = {12900.0, 13500.0, 13900.0, 18000.0};
  const double* v = fp64 ? vd : vm;
  if (C <= 2) return v[0];
  for (int i = 1; i < 4; ++i)
    if (C <= c[i]) return v[i - 1] + (v[i] - v[i - 1]) * (C - c[i - 1]) / (c[i] - c[i - 1]);
  return v[3];
}

// With the wide tier (VBD_TIERED_WIDE, tiered mode) the longest split
// environments may instead take a cluster of Cw = cluster_wide blocks, in a
// third launch: the planner tries every split of the environments, longest
// first, into h1 wide, h - h1 split over C and n - h single-block ones, and
// keeps the one with the smallest predicted step time (the largest of the
// longest job of each kind, the total block time / resident blocks, and each
// split tier's total / its resident clusters -- a cluster needs its blocks in
// one GPC, so fewer clusters than blocks / size fit; with more jobs than
// that, they run in waves).  At most as many wide jobs as wide clusters fit.
void make_plan(const vbd_solver* s, const int* iters, std::vector<int4>& work,
               std::vector<int4>& work2, std::vector<int4>& work3) {
  const int n = s->n_env, C = s->cluster;
  const int Cw = s->tiered ? s->cluster_wide : 0;
  work2.clear();
  work3.clear();
  const bool f64 = s->prec == 2;
  const double a1 = f64 ? 10200.0 : 8300.0;
  const double aC = split_overhead(C, f64);
  const double aW = Cw > 1 ? split_overhead(Cw, f64) : 0.0;
  // high and mean estimates on one block, on C blocks and on Cw blocks
  std::vector<double> d1(n), dC(n), dW(n), m1(n), mC(n), mW(n);
  const bool hist = s->env_sweeps.size() == (size_t)n && s->env_sweeps_mean.size() == (size_t)n &&
                    s->env_sweeps_decay.size() == (size_t)n;
  // the learned warm start's energy checks cost about 0.7 sweeps (measured)
  const double kw = s->warm ? 0.7 : 0.0;
  for (int e = 0; e < n; ++e) {
    const double last = iters ? (double)iters[e] : 1.0;
    double k = last, km = last;
    if (hist) {
      k = std::max(last, s->warm ? s->env_sweeps[e] : s->env_sweeps_decay[e]);
      km = s->warm ? s->env_sweeps_mean[e] : k;
    }
    k = std::max(1.0, k) + kw;
    km = std::max(1.0, km) + kw;
    const double slots = s->env_work[e];
    d1[e] = k * (slots + a1);
    dC[e] = C > 1 ? k * (slots / C + aC) : d1[e];
    dW[e] = Cw > 1 ? k * (slots / Cw + aW) : dC[e];
    m1[e] = km * (slots + a1);
    mC[e] = C > 1 ? km * (slots / C + aC) : m1[e];
    mW[e] = Cw > 1 ? km * (slots / Cw + aW) : mC[e];
  }
  std::vector<int> order(n);
  for (int e = 0; e < n; ++e) order[e] = e;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d1[a] > d1[b]; });
  work.clear();
  if (C <= 1) {
    for (int e : order) work.push_back(make_int4(e, 0, 1, 0));
    return;
  }
  if (n == 1) {
    for (int r = 0; r < C; ++r) work.push_back(make_int4(0, r, C, 0));
    return;
  }
  const double cap = std::max(1, s->capacity_blocks);
  double area0 = 0.0;
  for (double x : m1) area0 += x;
  int best_h1 = 0, best_h = 0;
  double best_t = 1e300;
  double t_wide = 0.0, sum_wide = 0.0;
  // clusters resident at once (tiered mode; 0 = not known): more split jobs
  // than that run in waves, which the per-tier sums over the resident
  // clusters bound from below
  const int max_w = s->max_clusters_wide, max_c = s->max_clusters_split;
  // h1: the longest environments on a wide cluster (none without the tier,
  // and never more than can be resident at once)
  for (int h1 = 0; h1 <= (Cw > 1 ? std::min(n, max_w) : 0); ++h1) {
    if (h1 > 0) {
      const int e = order[h1 - 1];
      area0 += Cw * mW[e] - m1[e];
      t_wide = std::max(t_wide, dW[e]);
      sum_wide += mW[e];
    }
    // clusters of C that still fit beside the wide ones
    const int c_free = max_c > 0 ? std::max(1, (max_c * C - h1 * Cw) / C) : 0;
    double area = area0, t_split = 0.0, sum_split = 0.0;
    for (int h = h1; h <= n; ++h) {
      // environments h1 .. h-1 are split over C blocks
      if (h > h1) {
        const int e = order[h - 1];
        area += C * mC[e] - m1[e];
        t_split = std::max(t_split, dC[e]);
        sum_split += mC[e];
      }
      const double t_single = h < n ? d1[order[h]] : 0.0;
      double t = std::max(std::max(std::max(t_wide, t_split), t_single), area / cap);
      if (max_w > 0) t = std::max(t, sum_wide / max_w);
      if (c_free > 0) t = std::max(t, sum_split / c_free);
      if (t < best_t * 0.999) {
        best_t = t;
        best_h1 = h1;
        best_h = h;
      }
      if (t_single <= std::max(t_split, t_wide)) break;  // splitting more cannot help
    }
    // a wider cluster for the next environment cannot beat this once the
    // wide jobs alone are the longest
    if (h1 < n && t_wide >= best_t) break;
  }
  std::stable_sort(order.begin(), order.begin() + best_h1,
                   [&](int a, int b) { return dW[a] > dW[b]; });
  std::stable_sort(order.begin() + best_h1, order.begin() + best_h,
                   [&](int a, int b) { return dC[a] > dC[b]; });
  for (int i = 0; i < best_h1; ++i)
    for (int r = 0; r < Cw; ++r) work3.push_back(make_int4(order[i], r, Cw, 2));
  for (int i = best_h1; i < best_h; ++i)
    for (int r = 0; r < C; ++r) work.push_back(make_int4(order[i], r, C, 0));
  if (s->tiered) {
    // the others run one block each in the light launch
    for (int i = best_h; i < n; ++i) work2.push_back(make_int4(order[i], 0, 1, 1));
    return;
  }
  int in_cluster = 0;
  for (int i = best_h; i < n; ++i) {
    work.push_back(make_int4(order[i], 0, 1, 0));
    in_cluster = (in_cluster + 1) % C;
  }
  while (in_cluster != 0) {
    work.push_back(make_int4(-1, 0, 0, 0));
    in_cluster = (in_cluster + 1) % C;
  }
}

size_t tier_smem(const vbd_solver* s, const std::vector<int4>& w) {
  size_t need = 0;
  for (const int4& x : w)
    if (x.x >= 0) need = std::max(need, env_smem(s, s->L.env[x.x], s->tab_in_smem));
  return need;
}

int upload_plan(vbd_solver* s, const int* iters) {
  std::vector<int4> w, w2, w3;
  make_plan(s, iters, w, w2, w3);
  auto same_as = [](const std::vector<int4>& a, const std::vector<int4>& b) {
    return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(int4)) == 0;
  };
  if (same_as(w, s->work) && same_as(w2, s->work2) && same_as(w3, s->work3)) return VBD_OK;
  if (w.size() > s->d_work.n || w2.size() > s->d_work2.n || w3.size() > s->d_work3.n)
    return fail(VBD_ERR_CUDA, "work map larger than its buffer");
  // the streams are idle here (create, or after a synchronising step)
  if (!w.empty())
    CUDA_TRY(cudaMemcpy(s->d_work.p, w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice));
  if (!w2.empty())
    CUDA_TRY(
        cudaMemcpy(s->d_work2.p, w2.data(), w2.size() * sizeof(int4), cudaMemcpyHostToDevice));
  if (!w3.empty())
    CUDA_TRY(
        cudaMemcpy(s->d_work3.p, w3.data(), w3.size() * sizeof(int4), cudaMemcpyHostToDevice));
  s->work.swap(w);
  s->work2.swap(w2);
  s->work3.swap(w3);
  if (s->tiered) {
    s->smem_heavy = tier_smem(s, s->work);
    s->smem_light = tier_smem(s, s->work2);
    s->smem_wide = tier_smem(s, s->work3);
  }
  return VBD_OK;
}

// Neighbour lists of the persistent kernel's readiness waits (PersistNbr):
// for every block b and colour c, the other blocks that own a solved vertex
// sharing a tet with one of b's colour-c vertices.  The owner of a vertex
// follows persist_kernel's assignment exactly: a large colour's chunk q goes
// to block ((q - chunk_begin) / warps per block) mod (every block), a small
// colour's to block (q - chunk_begin) mod nsb, nsb = the largest small
// colour's chunk count.
void build_persist_neighbours(const Layout& L, int tpv, int nwarps, int nb, std::vector<int>& off,
                              std::vector<int>& idx) {
  const EnvInfo& e = L.env[0];
  const int C = e.ncolors, cpw = 32 / tpv;
  auto is_small = [&](int nch) { return nb > 1 && nch <= kPersistSmallBlocks * nwarps; };
  int nsb = 1;
  for (int c = 0; c < C; ++c) {
    const ColorInfo& ci = L.color[e.cbase + c];
    const int nch = ci.chunk_end - ci.chunk_begin;
    if (is_small(nch)) nsb = std::max(nsb, nch);
  }
  nsb = std::min(nsb, nb);
  std::vector<int> owner(e.nsolved, -1);
  auto for_each_vertex = [&](auto&& f) {
    for (int c = 0; c < C; ++c) {
      const ColorInfo& ci = L.color[e.cbase + c];
      const bool small = is_small(ci.chunk_end - ci.chunk_begin);
      for (int q = ci.chunk_begin; q < ci.chunk_end; ++q) {
        // a small colour: chunk k on block k mod nsb (its warps split it);
        // a large one: chunks in groups of nwarps, group g on block g mod nb
        const int b = small ? (q - ci.chunk_begin) % nsb : ((q - ci.chunk_begin) / nwarps) % nb;
        for (int vi = 0; vi < cpw; ++vi) {
          const int gv = ci.vbegin + (q - ci.chunk_begin) * cpw + vi;
          if (gv < ci.vend) f(c, q, vi, gv - e.vbase, b);
        }
      }
    }
  };
  for_each_vertex([&](int, int, int, int lv, int b) { owner[lv] = b; });
  std::vector<std::vector<int>> lists((size_t)nb * C);
  for_each_vertex([&](int c, int q, int vi, int lv, int b) {
    const ChunkInfo& ch = L.chunk[q];
    const int k = L.valence[e.vbase + lv];
    for (int st = 0; st < ch.steps; ++st)
      for (int sub = 0; sub < tpv; ++sub) {
        if (st * tpv + sub >= k) continue;
        const int4& sl = L.rec_idx[((size_t)ch.block + st) * 32 + vi * tpv + sub];
        for (int n : {sl.x, sl.y, sl.z})
          if (n >= 0 && n < e.nsolved && owner[n] >= 0 && owner[n] != b)
            lists[(size_t)b * C + c].push_back(owner[n]);
      }
  });
  off.assign(1, 0);
  idx.clear();
  for (auto& l : lists) {
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
    idx.insert(idx.end(), l.begin(), l.end());
    off.push_back((int)idx.size());
  }
}

int create_impl(const double* X, int V, const int32_t* tets, int T, const double* rho,
                const double* E, const double* nu, const uint8_t* active, double kd,
                const double* gravity, const int32_t* coloring, const std::vector<int>& voff,
                const std::vector<int>& toff, int flags, int tpv, int threads, int device,
                vbd_solver** out) {
  if (!out) return fail(VBD_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (V <= 0 || T < 0 || !X || (T > 0 && (!tets || !rho || !E || !nu)))
    return fail(VBD_ERR_INVALID_ARG, "empty mesh or NULL array");
  for (size_t i = 0; i < 4 * (size_t)T; ++i)
    if (tets[i] < 0 || tets[i] >= V)
      return fail(VBD_ERR_INVALID_ARG, "tet vertex id out of range");
  if (tpv != 0 && tpv != 2 && tpv != 4 && tpv != 8 && tpv != 16)
    return fail(VBD_ERR_INVALID_ARG, "tpv must be 2, 4, 8 or 16");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(VBD_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(VBD_ERR_INVALID_ARG, "bad device ordinal");
  DeviceGuard dg(device);

  vbd_solver* s = new vbd_solver();
  s->device = device;
  s->flags = flags;
  s->prec = (flags & VBD_PRECISION_FP64) ? 2 : ((flags & VBD_PRECISION_MIXED) ? 1 : 0);
  s->fp64 = s->prec == 2;
  s->state64 = s->prec >= 1;
  s->material = (flags & VBD_MATERIAL_STVK) ? kStVK : kSNH;
  s->V = V;
  s->T = T;
  s->n_env = (int)voff.size() - 1;
  s->kd = kd;
  for (int i = 0; i < 3; ++i) s->g[i] = gravity ? gravity[i] : (i == 2 ? -9.81 : 0.0);
  s->real4_bytes = s->state64 ? 32 : 16;

  TetData td;
  int rc = build_tet_data(X, tets, T, rho, E, nu, s->material, td);
  if (rc != VBD_OK) {
    delete s;
    return rc;
  }
  // VBD_GPU_SETUP: the greedy colouring of the whole mesh on the GPU (the
  // same colours as the per-environment host pass)
  std::vector<int32_t> gpu_colors;
  if ((flags & VBD_GPU_SETUP) && !coloring && T > 0) {
    gpu_colors.assign(V, -1);
    std::string why;
    const int nc = gpu_greedy_coloring(tets, T, V, gpu_colors.data(), nullptr, &why);
    if (nc == kSetupTooManyColors) {
      delete s;
      return fail(VBD_ERR_TOO_MANY_COLORS, "Exceeded maximum number of colors");
    }
    if (nc < 0) {
      delete s;
      return fail(VBD_ERR_CUDA, "GPU colouring: " + why);
    }
  }
  // mode / threads / tpv
  int mode = flags & VBD_MODE_MASK;
  // provisional environment size bound for the shared-memory check
  int max_env_v = 0;
  for (int e = 0; e < s->n_env; ++e) max_env_v = std::max(max_env_v, voff[e + 1] - voff[e]);
  // block mode keeps x, y, z of every vertex of the environment in shared memory
  const size_t smem_per_vertex = s->state64 ? 24 : 12;
  const size_t smem_need = (size_t)max_env_v * smem_per_vertex;
  const bool fits = smem_need <= (size_t)env_kernel_max_smem();
  if (mode == VBD_MODE_AUTO) {
    // measured on B200 (the autotuner's results for cantilever meshes):
    // one block, or one cluster, holding the mesh in shared memory wins up
    // to ~2k vertices; beyond that the persistent kernel over the whole GPU
    if (s->n_env > 1)
      mode = VBD_MODE_BLOCK;
    else
      mode = (fits && V <= 2048) ? VBD_MODE_BLOCK : VBD_MODE_PERSIST;
  }
  if (mode == VBD_MODE_BLOCK && !fits) {
    delete s;
    return fail(VBD_ERR_UNSUPPORTED, "an environment does not fit in shared memory for block mode");
  }
  if ((mode == VBD_MODE_GRAPH || mode == VBD_MODE_HOSTLOOP || mode == VBD_MODE_PERSIST) &&
      s->n_env != 1) {
    delete s;
    return fail(VBD_ERR_UNSUPPORTED, "graph / host-loop / persistent mode runs a single environment");
  }
  if (mode != VBD_MODE_BLOCK && mode != VBD_MODE_GRAPH && mode != VBD_MODE_HOSTLOOP &&
      mode != VBD_MODE_PERSIST) {
    delete s;
    return fail(VBD_ERR_INVALID_ARG, "unknown mode");
  }
  s->mode = mode;
  const bool block_mode = mode == VBD_MODE_BLOCK;
  const int cl = (flags >> VBD_CLUSTER_SHIFT) & 0x1F;
  // the cluster field is 5 bits wide and nothing lies above it: a set bit
  // there is a cluster size that did not fit (or a negative one)
  if (cl > 16 || (static_cast<unsigned>(flags) >> (VBD_CLUSTER_SHIFT + 5)) != 0u) {
    delete s;
    return fail(VBD_ERR_INVALID_ARG, "cluster size must be 0 (automatic) or 1 to 16");
  }
  s->cluster = !block_mode ? 1 : (cl ? cl : (s->n_env > 1 ? 4 : (V > 512 ? 8 : 1)));
  s->replan = block_mode && s->n_env > 1 && s->cluster > 1;
  s->tiered = s->replan && (flags & VBD_TIERED) != 0;
  // the wide tier: clusters twice the size of the split environments' (at
  // most 16 blocks)
  s->cluster_wide = s->tiered && (flags & VBD_TIERED_WIDE) && s->cluster < 16
                        ? std::min(16, 2 * s->cluster)
                        : 0;
  if (threads == 0)
    threads = block_mode ? (s->n_env > 1 ? 256 : 512) : (mode == VBD_MODE_PERSIST ? 128 : 256);
  if (mode == VBD_MODE_GRAPH || mode == VBD_MODE_HOSTLOOP) threads = 256;
  if (threads % 32 || threads < 32 || threads > 512) {
    delete s;
    return fail(VBD_ERR_INVALID_ARG, "block_threads must be a multiple of 32 in [32, 512]");
  }
  s->threads = threads;
  if (tpv == 0) {
    if (block_mode && s->n_env == 1) {
      // spread the largest colour over the block: lanes per vertex ~ threads / colour size
      std::vector<int32_t> col(V, -1);
      int nvc = 0;
      for (size_t i = 0; i < 4 * (size_t)T; ++i) nvc = std::max(nvc, tets[i] + 1);
      const int32_t* pre =
          coloring ? coloring : (gpu_colors.empty() ? nullptr : gpu_colors.data());
      int ncol = pre ? 0 : greedy_coloring(tets, T, nvc, col.data());
      if (pre) {
        for (int v = 0; v < nvc; ++v) col[v] = pre[v];
        for (int v = 0; v < nvc; ++v) ncol = std::max(ncol, col[v] + 1);
      }
      std::vector<int> cnt(std::max(ncol, 1), 0);
      for (int v = 0; v < nvc; ++v)
        if (col[v] >= 0) cnt[col[v]]++;
      const int mg = std::max(1, *std::max_element(cnt.begin(), cnt.end()));
      tpv = 2;
      while (tpv < 16 && mg * tpv * 2 <= threads) tpv *= 2;
    } else {
      tpv = 4;  // batched environments and the grid-mode colour kernels
    }
  }
  s->tpv = tpv;
  s->L.table.fp64 = s->fp64;
  rc = build_layout(X, V, tets, T, active, voff, toff, coloring, td, tpv,
                    (flags & VBD_ORDER_INDEX) != 0, s->L,
                    gpu_colors.empty() ? nullptr : gpu_colors.data());
  if (rc != VBD_OK) {
    delete s;
    return rc;
  }
  s->smem_per_vertex = smem_per_vertex;
  s->rec_bytes = 3 * (s->fp64 ? 32 : 16);
  // block mode stages each environment's record table after its state when
  // every environment's state + table fits in a block's shared memory
  {
    size_t need = 0;
    for (const EnvInfo& ei : s->L.env)
      need = std::max(need, env_smem(s, ei, true));
    s->tab_in_smem = block_mode && need <= (size_t)env_kernel_max_smem();
    s->smem_bytes = 0;
    for (const EnvInfo& ei : s->L.env)
      s->smem_bytes = std::max(s->smem_bytes, env_smem(s, ei, s->tab_in_smem));
    // the persistent kernel stages the mesh's table in every block if small
    s->persist_smem = (size_t)s->L.max_env_records * s->rec_bytes;
    if (mode == VBD_MODE_PERSIST) {
      if (s->persist_smem > (size_t)kPersistMaxTabSmem) s->persist_smem = 0;
      s->tab_in_smem = s->persist_smem > 0;
    }
  }
  s->n_records = (long long)s->L.rec_idx.size();
  // 16-bit slots when every environment-local id and record id fits
  s->fmt = (s->L.max_env_vertices <= 65536 && s->L.max_env_records <= 65536) ? kFmtIdx16
                                                                              : kFmtIdx32;

  // ---- device upload --------------------------------------------------------
  auto bad = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return false;
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return true;
  };
  int err = 0;
  if (bad(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream")) err = 1;
  if (!err && (bad(cudaEventCreate(&s->ev_k0), "event") || bad(cudaEventCreate(&s->ev_k1), "event")))
    err = 1;
  cudaStream_t st = s->stream;
  const Layout& L = s->L;
  if (!err && bad(s->d_env.upload(L.env, st), "env")) err = 1;
  if (!err && bad(s->d_color.upload(L.color, st), "color")) err = 1;
  if (!err && bad(s->d_chunk.upload(L.chunk, st), "chunk")) err = 1;
  if (!err) {
    if (s->fmt == kFmtIdx16) {
      std::vector<ushort4> r16(L.rec_idx.size());
      for (size_t i = 0; i < r16.size(); ++i) {
        const int4 r = L.rec_idx[i];
        r16[i] = make_ushort4((unsigned short)r.x, (unsigned short)r.y, (unsigned short)r.z,
                              (unsigned short)r.w);
      }
      if (bad(s->d_rec_idx16.upload(r16, st), "rec_idx16")) err = 1;
      if (!err) cudaStreamSynchronize(st);  // r16 goes out of scope
    } else if (bad(s->d_rec_idx.upload(L.rec_idx, st), "rec_idx")) {
      err = 1;
    }
  }
  if (!err) {
    // record table in the solver precision: 3 Real4 per entry
    const size_t nval = L.table.vals.size();
    if (s->fp64) {
      if (bad(s->d_rec_tab.alloc(nval * 8), "rec_tab")) err = 1;
      if (!err && nval &&
          bad(cudaMemcpyAsync(s->d_rec_tab.p, L.table.vals.data(), nval * 8,
                              cudaMemcpyHostToDevice, st),
              "rec_tab copy"))
        err = 1;
    } else {
      std::vector<float> f(nval);
      for (size_t i = 0; i < nval; ++i) f[i] = (float)L.table.vals[i];
      if (bad(s->d_rec_tab.alloc(nval * 4), "rec_tab")) err = 1;
      if (!err && nval &&
          bad(cudaMemcpyAsync(s->d_rec_tab.p, f.data(), nval * 4, cudaMemcpyHostToDevice, st),
              "rec_tab copy"))
        err = 1;
    }
    if (!err) cudaStreamSynchronize(st);  // staging vectors go out of scope
  }
  if (!err && bad(s->d_valence.upload(L.valence, st), "valence")) err = 1;
  if (!err && bad(s->d_tet_slot.upload(L.tet_slot, st), "tet list")) err = 1;
  if (!err && bad(s->d_tet_owner.upload(L.tet_owner, st), "tet owners")) err = 1;
  if (!err && bad(s->d_map.upload(L.new_of_old, st), "map")) err = 1;
  if (!err) {
    std::vector<float4> ws(V);
    for (int i = 0; i < V; ++i)
      ws[i] = make_float4(L.wstat[4 * (size_t)i], L.wstat[4 * (size_t)i + 1],
                          L.wstat[4 * (size_t)i + 2], L.wstat[4 * (size_t)i + 3]);
    if (bad(s->d_wstat.upload(ws, st), "wstat")) err = 1;
    if (!err && bad(s->d_chunk_owner.upload(L.chunk_owner, st), "chunk_owner")) err = 1;
    if (!err) cudaStreamSynchronize(st);  // ws goes out of scope
  }
  std::vector<double> Xv(X, X + 3 * (size_t)V);
  if (!err && bad(s->d_X.upload(Xv, st), "X")) err = 1;
  if (!err && bad(s->d_io.alloc(3 * (size_t)V), "io")) err = 1;
  if (!err && bad(s->d_tol.alloc(s->n_env), "tol")) err = 1;
  if (!err && bad(s->d_iters.alloc(s->n_env), "iters")) err = 1;
  if (!err && bad(s->d_status.alloc(s->n_env), "status")) err = 1;
  if (!err && bad(s->d_dxmax.alloc(s->n_env), "dxmax")) err = 1;
  if (!err && bad(s->d_params.alloc(1), "params")) err = 1;
  if (!err && bad(s->d_ctl.alloc(1), "ctl")) err = 1;
  if (!err && mode == VBD_MODE_PERSIST) {
    if (bad(s->d_pctl.alloc(1), "persist ctl")) err = 1;
    // resident blocks, but no more than the largest colour can keep busy
    // (one chunk per warp): fewer blocks make cheaper grid barriers
    int per_sm = 0, sms = 0;
    if (!err && bad(persist_occupancy(s->prec, s->material, s->fmt, s->tpv, s->threads,
                                      s->persist_smem, &per_sm),
                    "persist occupancy"))
      err = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int wpb = s->threads / 32;
    int need = 1;
    for (const ColorInfo& ci : s->L.color)
      need = std::max(need, (ci.chunk_end - ci.chunk_begin + wpb - 1) / wpb);
    s->persist_blocks = std::min(need, per_sm * sms);
    if (!err && s->persist_blocks > 0 &&
        bad(s->d_pparts.alloc(4 * (size_t)s->persist_blocks), "persist parts"))
      err = 1;
    if (!err && s->persist_blocks < 1) {
      g_last_error = "persistent mode: the kernel does not fit on the device";
      err = 1;
    }
    if (!err && s->persist_blocks > 1 && !(flags & VBD_PERSIST_GRID_BARRIERS)) {
      std::vector<int> off, idx;
      build_persist_neighbours(s->L, s->tpv, wpb, s->persist_blocks, off, idx);
      if (idx.empty()) idx.push_back(0);  // a device buffer needs one entry
      if (bad(s->d_nbr_off.upload(off, st), "persist neighbours") ||
          bad(s->d_nbr_idx.upload(idx, st), "persist neighbours") ||
          bad(s->d_epoch.alloc((size_t)s->persist_blocks * kEpochStride), "persist epochs"))
        err = 1;
      else
        s->persist_scoped = true;
      cudaStreamSynchronize(st);  // off / idx go out of scope
    }
  }
  const size_t sb = s->real4_bytes * (size_t)V;
  for (auto* b : {&s->d_u, &s->d_ut, &s->d_up, &s->d_vel})
    if (!err && bad(b->alloc(sb), "state")) err = 1;
  if (!err) {
    // state: u = up = vel = 0, ut.w = lumped mass
    cudaMemsetAsync(s->d_u.p, 0, sb, st);
    cudaMemsetAsync(s->d_up.p, 0, sb, st);
    cudaMemsetAsync(s->d_vel.p, 0, sb, st);
    if (s->state64) {
      std::vector<double> ut(4 * (size_t)V, 0.0);
      for (int i = 0; i < V; ++i) ut[4 * (size_t)i + 3] = L.mass[i];
      if (bad(cudaMemcpyAsync(s->d_ut.p, ut.data(), sb, cudaMemcpyHostToDevice, st), "ut"))
        err = 1;
      cudaStreamSynchronize(st);
    } else {
      std::vector<float> ut(4 * (size_t)V, 0.0f);
      for (int i = 0; i < V; ++i) ut[4 * (size_t)i + 3] = (float)L.mass[i];
      if (bad(cudaMemcpyAsync(s->d_ut.p, ut.data(), sb, cudaMemcpyHostToDevice, st), "ut"))
        err = 1;
      cudaStreamSynchronize(st);
    }
    cudaMemsetAsync(s->d_iters.p, 0, sizeof(int) * s->n_env, st);
    cudaMemsetAsync(s->d_status.p, 0, sizeof(unsigned) * s->n_env, st);
    cudaMemsetAsync(s->d_dxmax.p, 0, sizeof(unsigned long long) * s->n_env, st);
  }
  if (!err && bad(cudaMallocHost(reinterpret_cast<void**>(&s->h_iters), sizeof(int) * s->n_env),
                  "pinned"))
    err = 1;
  if (!err &&
      bad(cudaMallocHost(reinterpret_cast<void**>(&s->h_status), sizeof(unsigned) * s->n_env),
          "pinned"))
    err = 1;
  if (!err && bad(cudaMallocHost(reinterpret_cast<void**>(&s->h_dxmax),
                                 sizeof(unsigned long long) * s->n_env),
                  "pinned"))
    err = 1;
  s->final_dx.assign(s->n_env, std::nan(""));
  if (!err && bad(cudaMallocHost(reinterpret_cast<void**>(&s->h_params), sizeof(StepParams)),
                  "pinned"))
    err = 1;
  if (!err && bad(cudaMallocHost(reinterpret_cast<void**>(&s->h_ctl), sizeof(LoopControl)),
                  "pinned"))
    err = 1;
  if (!err && bad(cudaStreamSynchronize(st), "setup sync")) err = 1;
  if (!err && block_mode) {
    // work estimate per environment: its incident (vertex, tet) slots
    s->env_work.assign(s->n_env, 0.0);
    for (int e = 0; e < s->n_env; ++e) s->env_work[e] = 4.0 * (toff[e + 1] - toff[e]) + 1.0;
    int occ = 0;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (s->tiered) {
      // capacity of the light launch (one block per environment) at the
      // largest environment's shared memory: a lower bound
      if (bad(env_occupancy(s->prec, s->material, s->fmt, s->tpv, s->threads, s->smem_bytes, 1,
                            &occ),
              "occupancy"))
        err = 1;
      s->capacity_blocks = occ * sms;
      int occ_c = 0, occ_w = 0;
      if (!err && bad(env_occupancy(s->prec, s->material, s->fmt, s->tpv, s->heavy_threads,
                                    s->smem_bytes, s->cluster, &occ_c),
                      "occupancy"))
        err = 1;
      if (!err && s->cluster_wide > 0 &&
          bad(env_occupancy(s->prec, s->material, s->fmt, s->tpv, s->heavy_threads,
                            s->smem_bytes, s->cluster_wide, &occ_w),
              "occupancy"))
        err = 1;
      s->max_clusters_split = occ_c;
      s->max_clusters_wide = occ_w;
      if (!err && (bad(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking), "stream") ||
                   bad(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming), "event") ||
                   bad(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming), "event")))
        err = 1;
      if (!err && bad(s->d_work2.alloc((size_t)s->n_env), "work")) err = 1;
      if (!err && s->cluster_wide > 0 &&
          (bad(cudaStreamCreateWithFlags(&s->aux2, cudaStreamNonBlocking), "stream") ||
           bad(cudaEventCreateWithFlags(&s->ev_join2, cudaEventDisableTiming), "event") ||
           bad(s->d_work3.alloc((size_t)s->n_env * s->cluster_wide), "work")))
        err = 1;
    } else {
      if (bad(env_occupancy(s->prec, s->material, s->fmt, s->tpv, s->threads, s->smem_bytes,
                            s->cluster, &occ),
              "occupancy"))
        err = 1;
      s->capacity_blocks = s->cluster > 1 ? occ * s->cluster : occ * sms;
    }
    if (!err && s->capacity_blocks < 1) {
      g_last_error = "block mode: this launch shape does not fit on the device";
      err = 1;
    }
    if (!err && bad(s->d_work.alloc((size_t)s->n_env * s->cluster + s->cluster), "work"))
      err = 1;
    if (!err && upload_plan(s, nullptr) != VBD_OK) err = 1;
  }
  if (err) {
    free_solver(s);
    return VBD_ERR_CUDA;
  }
  s->device_bytes = 0;
  s->device_bytes += (long long)(s->d_rec_idx.n * sizeof(int4) +
                                 s->d_rec_idx16.n * sizeof(ushort4) + s->d_rec_tab.n);
  s->device_bytes += (long long)(4 * sb + s->d_X.n * 8 + s->d_io.n * 8);
  s->device_bytes += (long long)(s->d_valence.n * 4 + s->d_map.n * 4);
  s->device_bytes += (long long)(s->d_tet_slot.n * sizeof(int4) + s->d_tet_owner.n * 4);
  *out = s;
  return VBD_OK;
}

int status_from_bits(const vbd_solver* s, const unsigned* st) {
  int rc = VBD_OK;
  for (int e = 0; e < s->n_env; ++e) {
    const unsigned b = st[e];
    if (b & kStatNonFinite) return fail(VBD_ERR_NONFINITE, "non-finite value in the iterate");
    if ((b & kStatGuard) && (s->flags & VBD_STRICT_SPD))
      return fail(VBD_ERR_NONFINITE, "3x3 vertex block not positive definite");
    if (b & kStatTimeout) return fail(VBD_ERR_TIMEOUT, "device-side wait timed out");
    if (b & kStatBounds) return fail(VBD_ERR_BOUNDS, "slot index out of range (checked build)");
    if (b & kStatIterCap) rc = VBD_NOT_CONVERGED;
  }
  return rc;
}

int set_params(vbd_solver* s, double dt, double tol, int max_iter) {
  StepParams p{};
  p.dt = dt;
  p.tol = tol;
  p.kd = s->kd;
  p.g[0] = s->g[0];
  p.g[1] = s->g[1];
  p.g[2] = s->g[2];
  p.max_iter = max_iter;
  p.strict_spd = (s->flags & VBD_STRICT_SPD) ? 1 : 0;
  p.warm = s->warm ? 1 : 0;
  p.tab_in_smem = s->tab_in_smem ? 1 : 0;
  p.trace = (s->trace_on && s->mode == VBD_MODE_BLOCK) ? s->d_trace.p : nullptr;
  if (s->params_valid && std::memcmp(&p, &s->cur_params, sizeof p) == 0) return VBD_OK;
  // the pinned staging struct may still be read by an earlier copy
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  *s->h_params = p;
  CUDA_TRY(cudaMemcpyAsync(s->d_params.p, s->h_params, sizeof p, cudaMemcpyHostToDevice,
                           s->stream));
  s->cur_params = p;
  s->params_valid = true;
  return VBD_OK;
}

int build_graph(vbd_solver* s) {
  if (s->graph_exec) return VBD_OK;
  cudaStream_t st = s->stream;
  const DevMesh m = s->mesh();
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaGraphCreate(&g, 0));
  s->graph = g;
  CUDA_TRY(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  cudaError_t le = launch_begin(s->state64, m, s->d_params.p, s->d_ctl.p, st);
  cudaGraph_t gout = nullptr;
  CUDA_TRY(cudaStreamEndCapture(st, &gout));
  CUDA_TRY(le);
  size_t n = 0;
  CUDA_TRY(cudaGraphGetNodes(g, nullptr, &n));
  if (n != 1) return fail(VBD_ERR_CUDA, "unexpected node count in the step graph");
  cudaGraphNode_t begin_node;
  CUDA_TRY(cudaGraphGetNodes(g, &begin_node, &n));
  cudaGraphConditionalHandle handle;
  CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, g, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond_node;
  CUDA_TRY(cudaGraphAddNode(&cond_node, g, &begin_node, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CUDA_TRY(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  le = cudaSuccess;
  const EnvInfo& e = s->L.env[0];
  for (int c = e.cbase; c < e.cbase + e.ncolors && le == cudaSuccess; ++c) {
    const ColorInfo& ci = s->L.color[c];
    le = launch_color(s->prec, s->material, s->tpv, s->threads, m, c,
                      ci.chunk_end - ci.chunk_begin, s->d_params.p, s->d_ctl.p, st);
  }
  if (le == cudaSuccess)
    le = launch_check(s->d_ctl.p, s->d_params.p, (unsigned long long)handle, 1, st);
  CUDA_TRY(cudaStreamEndCapture(st, &gout));
  CUDA_TRY(le);
  CUDA_TRY(cudaStreamBeginCaptureToGraph(st, g, &cond_node, nullptr, 1,
                                         cudaStreamCaptureModeThreadLocal));
  le = launch_end(s->state64, m, s->d_params.p, s->d_ctl.p, st);
  CUDA_TRY(cudaStreamEndCapture(st, &gout));
  CUDA_TRY(le);
  CUDA_TRY(cudaGraphInstantiate(&s->graph_exec, g, 0));
  return VBD_OK;
}

int enqueue_step(vbd_solver* s, double dt, double tol, const double* tol_env, int max_iter) {
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(VBD_ERR_INVALID_ARG, "dt must be > 0");
  if (max_iter < 1) return fail(VBD_ERR_INVALID_ARG, "max_iter must be >= 1");
  int rc = set_params(s, dt, tol, max_iter);
  if (rc != VBD_OK) return rc;
  const DevMesh m = s->mesh();
  cudaStream_t st = s->stream;
  int launches = 0;
  if (s->mode == VBD_MODE_BLOCK) {
    const double* dtol = nullptr;
    if (tol_env) {
      CUDA_TRY(cudaStreamSynchronize(st));
      CUDA_TRY(cudaMemcpy(s->d_tol.p, tol_env, sizeof(double) * s->n_env,
                          cudaMemcpyHostToDevice));
      dtol = s->d_tol.p;
    }
    if (s->cur_params.trace)
      CUDA_TRY(cudaMemsetAsync(s->d_trace.p, 0, sizeof(unsigned long long) * s->d_trace.n, st));
    if (s->warm) {
      NvtxRange nw("vbd_warm_start");
      // features of the coming step, then the network's predicted corrections
      CUDA_TRY(launch_ws_features(s->prec, s->tpv, m, (int)s->L.chunk.size(), dt, s->g,
                                  s->ws_history ? 1 : 0, s->d_wpack.p, s->d_feat.p, st));
      CUDA_TRY(launch_ws_infer(s->d_feat.p, s->V, s->d_wbf.p, s->d_wnorm.p, s->d_wstat.p,
                               s->d_pred.p, s->d_ws_err.p, st));
      launches += 3;  // pack, features, inference
    }
    CUDA_TRY(cudaEventRecord(s->ev_k0, st));
    NvtxRange nk("vbd_step_kernels");
    if (!s->tiered) {
      ++launches;
      CUDA_TRY(launch_env_step(s->prec, s->material, s->tpv, s->threads, m, s->cur_params, dtol,
                               s->d_work.p, (int)s->work.size(), s->cluster, s->smem_bytes, st));
    } else {
      // the launches with the widest clusters first (they need whole groups
      // of free SMs): wide tier, split environments, then the single-block
      // ones; the first non-empty one on the solver's stream, the others on
      // their own streams beside it, joined before the end.  Trace records
      // follow the same order.
      struct Tier {
        const std::vector<int4>* w;
        const int4* dw;
        int cluster, threads;
        size_t smem;
      };
      const Tier tiers[3] = {
          {&s->work3, s->d_work3.p, s->cluster_wide, s->heavy_threads, s->smem_wide},
          {&s->work, s->d_work.p, s->cluster, s->heavy_threads, s->smem_heavy},
          {&s->work2, s->d_work2.p, 1, s->threads, s->smem_light}};
      // second and third launch: streams aux and aux2 (aux2 exists with the
      // wide tier, the only way to have three)
      const cudaStream_t side[2] = {s->aux, s->aux2};
      const cudaEvent_t side_join[2] = {s->ev_join, s->ev_join2};
      int nonempty = 0;
      for (const Tier& t : tiers) nonempty += t.w->empty() ? 0 : 1;
      launches += nonempty;
      if (nonempty > 1) CUDA_TRY(cudaEventRecord(s->ev_fork, st));
      int k = -1;  // launches so far, minus one
      size_t trace_off = 0;
      for (const Tier& t : tiers) {
        if (t.w->empty()) continue;
        cudaStream_t ts = k < 0 ? st : side[k];
        if (k >= 0) CUDA_TRY(cudaStreamWaitEvent(ts, s->ev_fork, 0));
        StepParams lp = s->cur_params;
        if (lp.trace) lp.trace += 4 * trace_off;
        CUDA_TRY(launch_env_step(s->prec, s->material, s->tpv, t.threads, m, lp, dtol, t.dw,
                                 (int)t.w->size(), t.cluster, t.smem, ts));
        if (k >= 0) CUDA_TRY(cudaEventRecord(side_join[k], ts));
        ++k;
        trace_off += t.w->size();
      }
      for (int j = 0; j < k; ++j) CUDA_TRY(cudaStreamWaitEvent(st, side_join[j], 0));
    }
  } else if (s->mode == VBD_MODE_PERSIST) {
    if (s->warm) {
      NvtxRange nw("vbd_warm_start");
      CUDA_TRY(launch_ws_features(s->prec, s->tpv, m, (int)s->L.chunk.size(), dt, s->g,
                                  s->ws_history ? 1 : 0, s->d_wpack.p, s->d_feat.p, st));
      CUDA_TRY(launch_ws_infer(s->d_feat.p, s->V, s->d_wbf.p, s->d_wnorm.p, s->d_wstat.p,
                               s->d_pred.p, s->d_ws_err.p, st));
      launches += 3;
    }
    CUDA_TRY(cudaEventRecord(s->ev_k0, st));
    NvtxRange nk("vbd_step_kernels");
    ++launches;
    PersistNbr nbr{};
    if (s->persist_scoped) nbr = PersistNbr{s->d_nbr_off.p, s->d_nbr_idx.p, s->d_epoch.p};
    CUDA_TRY(launch_persist(s->prec, s->material, s->tpv, s->threads, m, s->d_params.p,
                            s->d_pctl.p, s->persist_blocks, s->wait_limits, s->d_pparts.p,
                            s->persist_smem, nbr, st));
  } else if (s->mode == VBD_MODE_GRAPH) {
    rc = build_graph(s);
    if (rc != VBD_OK) return rc;
    CUDA_TRY(cudaEventRecord(s->ev_k0, st));
    CUDA_TRY(cudaGraphLaunch(s->graph_exec, st));
    launches = -1;  // begin + sweeps x (colours + check) + end: counted in finish
  } else {
    CUDA_TRY(cudaEventRecord(s->ev_k0, st));
    launches = -1;
    // host-driven loop: one device->host read of the loop state per sweep
    CUDA_TRY(launch_begin(s->state64, m, s->d_params.p, s->d_ctl.p, st));
    const EnvInfo& e = s->L.env[0];
    for (int it = 0; it < max_iter; ++it) {
      for (int c = e.cbase; c < e.cbase + e.ncolors; ++c) {
        const ColorInfo& ci = s->L.color[c];
        CUDA_TRY(launch_color(s->prec, s->material, s->tpv, s->threads, m, c,
                              ci.chunk_end - ci.chunk_begin, s->d_params.p, s->d_ctl.p, st));
      }
      CUDA_TRY(launch_check(s->d_ctl.p, s->d_params.p, 0ull, 0, st));
      CUDA_TRY(cudaMemcpyAsync(s->h_ctl, s->d_ctl.p, sizeof(LoopControl), cudaMemcpyDeviceToHost,
                               st));
      CUDA_TRY(cudaStreamSynchronize(st));
      if (s->h_ctl->status & 0x80000000u) break;
    }
    CUDA_TRY(launch_end(s->state64, m, s->d_params.p, s->d_ctl.p, st));
  }
  CUDA_TRY(cudaEventRecord(s->ev_k1, st));
  s->launches_pending = launches;
  s->trace_pending = s->cur_params.trace && s->mode == VBD_MODE_BLOCK
                         ? (int)(s->work.size() + s->work2.size() + s->work3.size())
                         : 0;
  s->pending = true;
  s->ws_history = true;  // ut now holds this step's inertia target
  return VBD_OK;
}

// The tensor-core inference records a wait that ran out in d_ws_err; the
// rows it did not finish kept no prediction, so the step itself fell back to
// the inertia guess, but the caller is told.
// (*h_ws_err holds the device word once the stream has been synchronised.)
int ws_error_status(vbd_solver* s) {
  if (!s->warm || !s->h_ws_err || *s->h_ws_err == 0) return VBD_OK;
  *s->h_ws_err = 0;
  CUDA_TRY(cudaMemset(s->d_ws_err.p, 0, sizeof(unsigned)));
  return fail(VBD_ERR_TIMEOUT, "warm-start inference: a tensor-core wait timed out");
}

// warm_step: the step ran the learned warm start (its inference may have
// recorded a timeout in d_ws_err)
int finish(vbd_solver* s, int* iters_out, bool warm_step) {
  cudaStream_t st = s->stream;
  CUDA_TRY(cudaMemcpyAsync(s->h_iters, s->d_iters.p, sizeof(int) * s->n_env,
                           cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(s->h_status, s->d_status.p, sizeof(unsigned) * s->n_env,
                           cudaMemcpyDeviceToHost, st));
  if (warm_step && s->h_ws_err)
    CUDA_TRY(cudaMemcpyAsync(s->h_ws_err, s->d_ws_err.p, sizeof(unsigned),
                             cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  s->pending = false;
  if (cudaEventElapsedTime(&s->kernel_ms_last, s->ev_k0, s->ev_k1) != cudaSuccess) {
    s->kernel_ms_last = -1.f;
    cudaGetLastError();  // not a step failure: keep it out of the next launch check
  }
  s->trace_last = s->trace_pending;
  s->launches_last = s->launches_pending >= 0
                         ? s->launches_pending
                         : 2 + s->h_iters[0] * ((int)s->L.color.size() + 1);
  if (iters_out) std::memcpy(iters_out, s->h_iters, sizeof(int) * s->n_env);
  // environments that used every allowed sweep recorded the largest |dx|
  // component of the last one: read it, then clear the words for the next
  // step that reaches its cap (the stream is idle here)
  bool capped = false;
  for (int e = 0; e < s->n_env; ++e) capped |= (s->h_status[e] & kStatIterCap) != 0;
  std::fill(s->final_dx.begin(), s->final_dx.end(), std::nan(""));
  if (capped) {
    CUDA_TRY(cudaMemcpy(s->h_dxmax, s->d_dxmax.p, sizeof(unsigned long long) * s->n_env,
                        cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemset(s->d_dxmax.p, 0, sizeof(unsigned long long) * s->n_env));
    for (int e = 0; e < s->n_env; ++e)
      if (s->h_status[e] & kStatIterCap) {
        double v;
        std::memcpy(&v, &s->h_dxmax[e], sizeof v);
        s->final_dx[e] = v;
      }
  }
  s->last_status = status_from_bits(s, s->h_status);
  if (s->last_status >= 0 && warm_step) {
    const int ws = ws_error_status(s);
    if (ws != VBD_OK) s->last_status = ws;
  }
  if (s->replan) {
    // re-balance the next step from this step's sweep counts (stream is idle)
    const int W = vbd_solver::kSweepWindow;
    const bool first = s->env_sweeps.empty();
    s->env_sweeps.resize(s->n_env, 1.0);
    s->env_sweeps_mean.resize(s->n_env, 1.0);
    s->env_sweeps_decay.resize(s->n_env, 1.0);
    s->env_sweep_ring.resize((size_t)s->n_env * W, 0);
    for (int e = 0; e < s->n_env; ++e) {
      const double k = s->h_iters[e];
      int* ring = &s->env_sweep_ring[(size_t)e * W];
      ring[s->ring_pos] = s->h_iters[e];
      s->env_sweeps[e] = *std::max_element(ring, ring + W);
      s->env_sweeps_mean[e] = first ? k : 0.9 * s->env_sweeps_mean[e] + 0.1 * k;
      s->env_sweeps_decay[e] = std::max(k, 0.95 * s->env_sweeps_decay[e]);
    }
    s->ring_pos = (s->ring_pos + 1) % W;
    const int rc = upload_plan(s, s->h_iters);
    if (rc != VBD_OK) return rc;
  }
  return s->last_status;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int vbd_version(void) { return 1; }

const char* vbd_status_string(int status) {
  switch (status) {
    case VBD_OK: return "ok";
    case VBD_NOT_CONVERGED: return "not converged within max_iter";
    case VBD_ERR_INVALID_ARG: return "invalid argument";
    case VBD_ERR_CUDA: return "CUDA error";
    case VBD_ERR_SINGULAR_DM: return "singular rest shape (zero-volume tet)";
    case VBD_ERR_TOO_MANY_COLORS: return "colouring needs more than 256 colours";
    case VBD_ERR_NONFINITE: return "non-finite value";
    case VBD_ERR_TIMEOUT: return "device-side wait timed out";
    case VBD_ERR_NO_DEVICE: return "no CUDA device";
    case VBD_ERR_UNSUPPORTED: return "unsupported configuration";
    default: return "unknown status";
  }
}

const char* vbd_last_error_message(void) { return g_last_error.c_str(); }

int vbd_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int vbd_graph_coloring(const int32_t* tets, int n_tets, int32_t* coloring_out,
                       int* n_vertices_out, int* n_colors_out) {
  if (n_tets < 0 || (n_tets > 0 && (!tets || !coloring_out)))
    return fail(VBD_ERR_INVALID_ARG, "bad arguments");
  int nv = 0;
  for (size_t i = 0; i < 4 * (size_t)n_tets; ++i) {
    if (tets[i] < 0) return fail(VBD_ERR_INVALID_ARG, "negative vertex id");
    nv = std::max(nv, tets[i] + 1);
  }
  int nc = nv ? greedy_coloring(tets, n_tets, nv, coloring_out) : 0;
  if (n_vertices_out) *n_vertices_out = nv;
  if (nc < 0) return fail(VBD_ERR_TOO_MANY_COLORS, "Exceeded maximum number of colors");
  if (n_colors_out) *n_colors_out = nc;
  return VBD_OK;
}

int vbd_graph_coloring_gpu(const int32_t* tets, int n_tets, int32_t* coloring_out,
                           int* n_vertices_out, int* n_colors_out, int device) {
  if (n_tets < 0 || (n_tets > 0 && (!tets || !coloring_out)))
    return fail(VBD_ERR_INVALID_ARG, "bad arguments");
  int nv = 0;
  for (size_t i = 0; i < 4 * (size_t)n_tets; ++i) {
    if (tets[i] < 0) return fail(VBD_ERR_INVALID_ARG, "negative vertex id");
    nv = std::max(nv, tets[i] + 1);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(VBD_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(VBD_ERR_INVALID_ARG, "bad device ordinal");
  DeviceGuard dg(device);
  std::string why;
  const int nc = nv ? gpu_greedy_coloring(tets, n_tets, nv, coloring_out, nullptr, &why) : 0;
  if (n_vertices_out) *n_vertices_out = nv;
  if (nc == kSetupTooManyColors)
    return fail(VBD_ERR_TOO_MANY_COLORS, "Exceeded maximum number of colors");
  if (nc < 0) return fail(VBD_ERR_CUDA, "GPU colouring: " + why);
  if (n_colors_out) *n_colors_out = nc;
  return VBD_OK;
}

int vbd_create(const double* rest_positions, int n_vertices, const int32_t* tets, int n_tets,
               const double* densities, const double* youngs_modulus,
               const double* poissons_ratio, const uint8_t* active_mask,
               double damping_coefficient, const double* gravity, const int32_t* coloring,
               int flags, int tpv, int block_threads, int device, vbd_solver** out) {
  std::vector<int> voff{0, n_vertices}, toff{0, n_tets};
  return create_impl(rest_positions, n_vertices, tets, n_tets, densities, youngs_modulus,
                     poissons_ratio, active_mask, damping_coefficient, gravity, coloring, voff,
                     toff, flags, tpv, block_threads, device, out);
}

int vbd_create_batched(const double* rest_positions, int n_vertices, const int32_t* tets,
                       int n_tets, const double* densities, const double* youngs_modulus,
                       const double* poissons_ratio, const uint8_t* active_mask,
                       double damping_coefficient, const double* gravity,
                       const int32_t* env_vertex_offset, const int32_t* env_tet_offset,
                       int n_env, int flags, int tpv, int block_threads, int device,
                       vbd_solver** out) {
  if (n_env < 1 || !env_vertex_offset || !env_tet_offset)
    return fail(VBD_ERR_INVALID_ARG, "n_env < 1 or NULL offsets");
  if (env_vertex_offset[0] != 0 || env_tet_offset[0] != 0 ||
      env_vertex_offset[n_env] != n_vertices || env_tet_offset[n_env] != n_tets)
    return fail(VBD_ERR_INVALID_ARG, "environment offsets must span [0, n) exactly");
  std::vector<int> voff(env_vertex_offset, env_vertex_offset + n_env + 1);
  std::vector<int> toff(env_tet_offset, env_tet_offset + n_env + 1);
  for (int e = 0; e < n_env; ++e)
    if (voff[e + 1] <= voff[e] || toff[e + 1] < toff[e])
      return fail(VBD_ERR_INVALID_ARG, "every environment needs >= 1 vertex");
  return create_impl(rest_positions, n_vertices, tets, n_tets, densities, youngs_modulus,
                     poissons_ratio, active_mask, damping_coefficient, gravity, nullptr, voff,
                     toff, flags, tpv, block_threads, device, out);
}

void vbd_destroy(vbd_solver* s) { free_solver(s); }

int vbd_set_wait_limits(vbd_solver* s, long long max_polls, unsigned long long max_wait_ns) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  if (max_polls < 0) return fail(VBD_ERR_INVALID_ARG, "max_polls must be >= 0");
  s->wait_limits.max_polls = max_polls;
  s->wait_limits.max_wait_ns = max_wait_ns;
  return VBD_OK;
}

int vbd_set_trace(vbd_solver* s, int enable) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  DeviceGuard dg(s->device);
  if (enable && !s->d_trace.p) {
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    CUDA_TRY(s->d_trace.alloc(4 * (s->d_work.n + s->d_work2.n + s->d_work3.n)));
    CUDA_TRY(cudaMemset(s->d_trace.p, 0, sizeof(unsigned long long) * s->d_trace.n));
  }
  s->trace_on = enable != 0;
  return VBD_OK;
}

int vbd_get_trace(vbd_solver* s, unsigned long long* records, int cap, int* count) {
  if (!s || !count) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(s->device);
  if (s->pending) {
    const int rc = finish(s, nullptr, s->warm);
    if (rc < 0) return rc;
  }
  if (!records) {
    *count = s->trace_last;
    return VBD_OK;
  }
  const int n = std::min(std::max(cap, 0), s->trace_last);
  if (n > 0)
    CUDA_TRY(cudaMemcpy(records, s->d_trace.p, sizeof(unsigned long long) * 4 * (size_t)n,
                        cudaMemcpyDeviceToHost));
  *count = n;
  return VBD_OK;
}

int vbd_reset(vbd_solver* s) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  DeviceGuard dg(s->device);
  const size_t sb = s->real4_bytes * (size_t)s->V;
  CUDA_TRY(cudaMemsetAsync(s->d_u.p, 0, sb, s->stream));
  CUDA_TRY(cudaMemsetAsync(s->d_vel.p, 0, sb, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->ws_history = false;
  return VBD_OK;
}

int vbd_step(vbd_solver* s, double dt, double tol, int max_iter, int* iterations_out) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  NvtxRange nr("vbd_step");
  DeviceGuard dg(s->device);
  int rc = enqueue_step(s, dt, tol, nullptr, max_iter);
  if (rc != VBD_OK) return rc;
  if (!iterations_out) return VBD_OK;
  return finish(s, iterations_out, s->warm);
}

int vbd_step_batched(vbd_solver* s, double dt, double tol, const double* tol_per_env,
                     int max_iter, int* iterations_out) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  NvtxRange nr("vbd_step");
  DeviceGuard dg(s->device);
  if (tol_per_env && s->mode != VBD_MODE_BLOCK)
    return fail(VBD_ERR_UNSUPPORTED, "per-environment tolerances need block mode");
  int rc = enqueue_step(s, dt, tol, tol_per_env, max_iter);
  if (rc != VBD_OK) return rc;
  if (!iterations_out) return VBD_OK;
  return finish(s, iterations_out, s->warm);
}

static int exchange(vbd_solver* s, const double* in, double* out, bool positions);

int vbd_step_batched_to(vbd_solver* s, double dt, double tol, const double* tol_per_env,
                        int max_iter, int* iterations_out, double* positions_out) {
  if (!s || !iterations_out || !positions_out) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  NvtxRange nr("vbd_step");
  DeviceGuard dg(s->device);
  if (tol_per_env && s->mode != VBD_MODE_BLOCK)
    return fail(VBD_ERR_UNSUPPORTED, "per-environment tolerances need block mode");
  double* dptr = nullptr;
  if (s->mode == VBD_MODE_BLOCK &&
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&dptr), positions_out, 0) != cudaSuccess) {
    cudaGetLastError();  // not page-locked and mapped: copy after the step instead
    dptr = nullptr;
  }
  s->host_out = dptr;
  int rc = enqueue_step(s, dt, tol, tol_per_env, max_iter);
  s->host_out = nullptr;
  if (rc != VBD_OK) return rc;
  rc = finish(s, iterations_out, s->warm);
  if (rc < 0 || dptr) return rc;
  const int rc2 = exchange(s, nullptr, positions_out, true);
  return rc2 != VBD_OK ? rc2 : rc;
}

int vbd_sync(vbd_solver* s) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  NvtxRange nr("vbd_sync");
  DeviceGuard dg(s->device);
  if (!s->pending) {
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return s->last_status;
  }
  return finish(s, nullptr, s->warm);
}

int vbd_get_iterations(vbd_solver* s, int* iterations_out) {
  if (!s || !iterations_out) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(s->device);
  if (s->pending) {
    int rc = finish(s, iterations_out, s->warm);
    return rc < 0 ? rc : VBD_OK;
  }
  std::memcpy(iterations_out, s->h_iters, sizeof(int) * s->n_env);
  return VBD_OK;
}

int vbd_get_final_dx(vbd_solver* s, double* final_dx_out) {
  if (!s || !final_dx_out) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(s->device);
  if (s->pending) {
    const int rc = finish(s, nullptr, s->warm);
    if (rc < 0) return rc;
  }
  std::memcpy(final_dx_out, s->final_dx.data(), sizeof(double) * s->n_env);
  return VBD_OK;
}

static int exchange(vbd_solver* s, const double* in, double* out, bool positions) {
  if (!s || (!in && !out)) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(s->device);
  cudaStream_t st = s->stream;
  const size_t bytes = sizeof(double) * 3 * (size_t)s->V;
  void* state = positions ? (void*)s->d_u.p : (void*)s->d_vel.p;
  const double* off = positions ? s->d_X.p : nullptr;
  // The warm start's history feature (u minus the previous step's inertia
  // target) is kept: a caller handing back the positions a step produced
  // (the usual loop) keeps it valid, and after an unrelated state it only
  // makes the prediction worse, which the potential check then rejects.
  // vbd_reset clears it.
  if (out) {
    CUDA_TRY(launch_gather(s->state64, off, s->d_map.p, state, s->d_io.p, s->V, st));
    CUDA_TRY(cudaMemcpyAsync(out, s->d_io.p, bytes, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
  } else {
    CUDA_TRY(cudaStreamSynchronize(st));  // d_io may be in use by a pending gather
    CUDA_TRY(cudaMemcpyAsync(s->d_io.p, in, bytes, cudaMemcpyHostToDevice, st));
    CUDA_TRY(launch_scatter(s->state64, off, s->d_map.p, s->d_io.p, state, s->V, st));
    CUDA_TRY(cudaStreamSynchronize(st));
  }
  return VBD_OK;
}

int vbd_get_positions(vbd_solver* s, double* x) { return exchange(s, nullptr, x, true); }
int vbd_set_positions(vbd_solver* s, const double* x) { return exchange(s, x, nullptr, true); }
int vbd_get_velocities(vbd_solver* s, double* v) { return exchange(s, nullptr, v, false); }
int vbd_set_velocities(vbd_solver* s, const double* v) { return exchange(s, v, nullptr, false); }

int vbd_get_color_groups(vbd_solver* s, int32_t* table, int* n_colors, int* max_group) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  if (n_colors) *n_colors = s->L.table_colors;
  if (max_group) *max_group = s->L.table_max_group;
  if (table && !s->L.table0.empty())
    std::memcpy(table, s->L.table0.data(), sizeof(int32_t) * s->L.table0.size());
  return VBD_OK;
}

int vbd_get_info(vbd_solver* s, vbd_info_t* info) {
  if (!s || !info) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  info->n_vertices = s->V;
  info->n_tets = s->T;
  info->n_env = s->n_env;
  info->n_colors = s->L.max_colors;
  info->max_valence = s->L.max_valence;
  info->mode = s->mode;
  info->tpv = s->tpv;
  info->block_threads = s->threads;
  info->precision = s->prec;
  info->material = s->material;
  info->n_slots = s->L.n_slots;
  info->n_slot_records = s->n_records;
  info->device_bytes = s->device_bytes;
  info->n_unique_records = s->L.table.size();
  info->record_format = s->fmt == kFmtIdx16 ? 8 : 16;
  info->cluster = s->cluster;
  info->last_step_launches = s->launches_last;
  info->last_step_kernel_ms = s->kernel_ms_last;
  info->n_blocks = s->mode == VBD_MODE_PERSIST ? s->persist_blocks
                                                : (int)(s->work.size() + s->work2.size() + s->work3.size());
  return VBD_OK;
}

void* vbd_get_stream(vbd_solver* s) { return s ? (void*)s->stream : nullptr; }

// ---- learned warm start ----------------------------------------------------
int vbd_ws_param_count(void) { return kWsParams; }
int vbd_ws_feature_width(void) { return kWsRow; }

static int ensure_ws_buffers(vbd_solver* s) {
  if (!s->d_feat.p) {
    CUDA_TRY(s->d_feat.alloc((size_t)s->V * kWsRow));
    // rows of vertices that are never solved keep flag 0
    CUDA_TRY(cudaMemsetAsync(s->d_feat.p, 0, sizeof(float) * (size_t)s->V * kWsRow, s->stream));
  }
  if (!s->d_pred.p) CUDA_TRY(s->d_pred.alloc((size_t)s->V));
  if (!s->d_wpack.p) CUDA_TRY(s->d_wpack.alloc(6 * (size_t)s->V));
  return VBD_OK;
}

int vbd_set_warmstart(vbd_solver* s, const float* params, const float* norm) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  DeviceGuard dg(s->device);
  if (!params) {
    s->warm = false;
    return VBD_OK;
  }
  if (s->mode != VBD_MODE_BLOCK && s->mode != VBD_MODE_PERSIST)
    return fail(VBD_ERR_UNSUPPORTED, "the learned warm start runs in block or persistent mode");
  for (int i = 0; i < kWsParams; ++i)
    if (!std::isfinite(params[i])) return fail(VBD_ERR_INVALID_ARG, "non-finite parameter");
  std::vector<float> nrm(kWsNorm);
  for (int i = 0; i < kWsNorm; ++i) {
    // identity normalisation: mean 0, 1/std 1, std 1, mean 0
    const bool scale = (i >= kWsIn && i < 2 * kWsIn) || (i >= 2 * kWsIn && i < 2 * kWsIn + kWsOut);
    nrm[i] = norm ? norm[i] : (scale ? 1.0f : 0.0f);
    if (!std::isfinite(nrm[i])) return fail(VBD_ERR_INVALID_ARG, "non-finite normalisation");
  }
  int rc = ensure_ws_buffers(s);
  if (rc != VBD_OK) return rc;
  if (!s->d_wparams.p) CUDA_TRY(s->d_wparams.alloc(kWsParams));
  if (!s->d_wbf.p) CUDA_TRY(s->d_wbf.alloc(2 * (size_t)kWsParams));
  if (!s->d_wnorm.p) CUDA_TRY(s->d_wnorm.alloc(kWsNorm));
  if (!s->d_ws_err.p) CUDA_TRY(s->d_ws_err.alloc(1));
  if (!s->h_ws_err) CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&s->h_ws_err), sizeof(unsigned)));
  *s->h_ws_err = 0;
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  CUDA_TRY(cudaMemset(s->d_ws_err.p, 0, sizeof(unsigned)));
  CUDA_TRY(cudaMemcpy(s->d_wnorm.p, nrm.data(), sizeof(float) * kWsNorm, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(s->d_wparams.p, params, sizeof(float) * kWsParams, cudaMemcpyHostToDevice));
  CUDA_TRY(launch_to_bf16(s->d_wparams.p, s->d_wbf.p, kWsParams, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->warm = true;
  return VBD_OK;
}

int vbd_ws_features(vbd_solver* s, double dt, float* features) {
  if (!s || !features) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  if (!(dt > 0.0)) return fail(VBD_ERR_INVALID_ARG, "dt must be > 0");
  DeviceGuard dg(s->device);
  int rc = ensure_ws_buffers(s);
  if (rc != VBD_OK) return rc;
  CUDA_TRY(cudaMemsetAsync(features, 0, sizeof(float) * (size_t)s->V * kWsRow, s->stream));
  CUDA_TRY(launch_ws_features(s->prec, s->tpv, s->mesh(), (int)s->L.chunk.size(), dt, s->g,
                              s->ws_history ? 1 : 0, s->d_wpack.p, features, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return VBD_OK;
}

int vbd_incremental_potential(vbd_solver* s, double dt, const double* positions,
                              double* potential_out) {
  if (!s || !positions || !potential_out) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(VBD_ERR_INVALID_ARG, "dt must be > 0");
  DeviceGuard dg(s->device);
  cudaStream_t st = s->stream;
  if (s->pending) {
    const int rc = finish(s, nullptr, s->warm);
    if (rc < 0) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  if (!s->d_xeval.p) {
    CUDA_TRY(s->d_xeval.alloc(s->real4_bytes * (size_t)s->V));
    CUDA_TRY(cudaMemset(s->d_xeval.p, 0, s->real4_bytes * (size_t)s->V));
  }
  if (!s->d_pot.p) CUDA_TRY(s->d_pot.alloc((size_t)s->n_env));
  StepParams p{};
  p.dt = dt;
  p.kd = s->kd;
  for (int i = 0; i < 3; ++i) p.g[i] = s->g[i];
  CUDA_TRY(cudaMemcpyAsync(s->d_io.p, positions, sizeof(double) * 3 * (size_t)s->V,
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(launch_scatter(s->state64, s->d_X.p, s->d_map.p, s->d_io.p, s->d_xeval.p, s->V, st));
  CUDA_TRY(launch_potential(s->prec, s->material, s->mesh(), p, s->d_xeval.p, s->d_pot.p, st));
  CUDA_TRY(cudaMemcpyAsync(potential_out, s->d_pot.p, sizeof(double) * s->n_env,
                           cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return VBD_OK;
}

int vbd_ws_vertex_rows(vbd_solver* s, int32_t* rows) {
  if (!s || !rows) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  std::memcpy(rows, s->L.new_of_old.data(), sizeof(int32_t) * (size_t)s->V);
  return VBD_OK;
}

int vbd_ws_predict(vbd_solver* s, const float* features, float* predictions) {
  if (!s || !features || !predictions) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  if (!s->d_wbf.p || !s->d_wnorm.p)
    return fail(VBD_ERR_INVALID_ARG, "no warm-start model set (vbd_set_warmstart)");
  DeviceGuard dg(s->device);
  CUDA_TRY(launch_ws_infer(features, s->V, s->d_wbf.p, s->d_wnorm.p, s->d_wstat.p,
                           reinterpret_cast<float4*>(predictions), s->d_ws_err.p, s->stream));
  CUDA_TRY(cudaMemcpyAsync(s->h_ws_err, s->d_ws_err.p, sizeof(unsigned), cudaMemcpyDeviceToHost,
                           s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return ws_error_status(s);
}

int vbd_get_env_status(vbd_solver* s, uint32_t* status_out) {
  if (!s || !status_out) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(s->device);
  if (s->pending) {
    const int rc = finish(s, nullptr, s->warm);
    if (rc < 0) return rc;
  }
  std::memcpy(status_out, s->h_status, sizeof(uint32_t) * s->n_env);
  return VBD_OK;
}

int vbd_ws_targets(vbd_solver* s, const float* features, float* targets) {
  if (!s || !features || !targets) return fail(VBD_ERR_INVALID_ARG, "NULL argument");
  DeviceGuard dg(s->device);
  CUDA_TRY(launch_ws_targets(s->state64, s->mesh(), features, targets, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return VBD_OK;
}

int vbd_mlp_train_batch(const float* X, const float* Y, const int32_t* idx, int batch,
                        const float* params, float* grad, float* scratch, double* loss,
                        void* stream) {
  if (!X || !Y || !params || !grad || !scratch || batch <= 0)
    return fail(VBD_ERR_INVALID_ARG, "bad arguments");
  CUDA_TRY(launch_mlp_train_batch(X, Y, idx, batch, params, grad, scratch, loss,
                                  static_cast<cudaStream_t>(stream)));
  return VBD_OK;
}

size_t vbd_mlp_train_scratch_floats(int batch) {
  return batch > 0 ? mlp_train_scratch_floats(batch) : 0;
}

int vbd_mlp_forward(const float* X, int n, const float* params, float* out, float* scratch,
                    void* stream) {
  (void)scratch;
  if (!X || !params || !out || n < 0) return fail(VBD_ERR_INVALID_ARG, "bad arguments");
  if (n == 0) return VBD_OK;
  CUDA_TRY(launch_mlp_forward(X, n, params, out, static_cast<cudaStream_t>(stream)));
  return VBD_OK;
}

int vbd_mlp_adam(float* params, const float* grad, float* m, float* v, int n, float lr,
                 float beta1, float beta2, float eps, int t, void* stream) {
  if (!params || !grad || !m || !v || n <= 0 || t < 1)
    return fail(VBD_ERR_INVALID_ARG, "bad arguments");
  CUDA_TRY(launch_adam(params, grad, m, v, n, lr, beta1, beta2, eps, t,
                       static_cast<cudaStream_t>(stream)));
  return VBD_OK;
}

// Allocation-free step (see vbd_noalloc.cu for who needs it and the limits of
// its static scratch).  Runs the grid-mode colour sweep one sweep at a time
// from the host; every buffer it touches either belongs to the solver (made
// by vbd_create) or is the static scratch.  It always takes a plain step: on
// a solver with the learned warm start enabled the prediction is not used
// (its feature and inference buffers are allocated on first use).  The step's
// kernel time and launch count are recorded for vbd_get_info like vbd_step's.
int vbd_step_noalloc(vbd_solver* s, double dt, double tol, int max_iter, int* iterations_out) {
  if (!s) return fail(VBD_ERR_INVALID_ARG, "NULL solver");
  if (s->n_env != 1)
    return fail(VBD_ERR_UNSUPPORTED, "vbd_step_noalloc steps single-environment solvers");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(VBD_ERR_INVALID_ARG, "dt must be > 0");
  if (max_iter < 1) return fail(VBD_ERR_INVALID_ARG, "max_iter must be >= 1");
  DeviceGuard dg(s->device);
  if (s->pending) {  // an enqueued step: collect its results first
    const int rc = finish(s, nullptr, s->warm);
    if (rc < 0) return rc;
  }
  const EnvInfo& e = s->L.env[0];
  int total = 0;  // convergence partials one sweep writes (one per thread block)
  for (int c = e.cbase; c < e.cbase + e.ncolors; ++c) {
    const ColorInfo& ci = s->L.color[c];
    total += (ci.chunk_end - ci.chunk_begin + 7) / 8;
  }
  if (total > noalloc_max_partials())
    return fail(VBD_ERR_UNSUPPORTED,
                "vbd_step_noalloc: this mesh needs " + std::to_string(total) +
                    " convergence partials per sweep; its static scratch holds " +
                    std::to_string(noalloc_max_partials()));
  unsigned long long* scratch = nullptr;
  CUDA_TRY(noalloc_scratch_address(&scratch));
  LoopControl* ctl = reinterpret_cast<LoopControl*>(scratch + kNoAllocCtlOffset);
  StepParams* dp = reinterpret_cast<StepParams*>(scratch + kNoAllocParamOffset);
  unsigned long long* partial = scratch + kNoAllocPartialOffset;
  StepParams p{};
  p.dt = dt;
  p.tol = tol;
  p.kd = s->kd;
  p.g[0] = s->g[0];
  p.g[1] = s->g[1];
  p.g[2] = s->g[2];
  p.max_iter = max_iter;
  p.strict_spd = (s->flags & VBD_STRICT_SPD) ? 1 : 0;
  cudaStream_t st = s->stream;
  const DevMesh m = s->mesh();
  // from pageable memory: the copy has read `p` when the call returns
  CUDA_TRY(cudaMemcpyAsync(dp, &p, sizeof p, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaEventRecord(s->ev_k0, st));
  CUDA_TRY(launch_begin(s->state64, m, dp, ctl, st));  // also zeroes the loop control
  int launches = 2;  // begin, end
  LoopControl hc{};
  for (int it = 0; it < max_iter; ++it) {
    int off = 0;
    for (int c = e.cbase; c < e.cbase + e.ncolors; ++c) {
      const ColorInfo& ci = s->L.color[c];
      const int blocks = (ci.chunk_end - ci.chunk_begin + 7) / 8;
      CUDA_TRY(launch_noalloc_color(s->prec, s->material, s->tpv, m, c, blocks, dp, ctl,
                                    partial + off, st));
      off += blocks;
      launches += blocks > 0 ? 1 : 0;
    }
    CUDA_TRY(launch_noalloc_reduce(partial, off, ctl, st));
    CUDA_TRY(launch_check(ctl, dp, 0ull, 0, st));
    launches += 2;
    CUDA_TRY(cudaMemcpyAsync(&hc, ctl, sizeof hc, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (hc.status & 0x80000000u) break;
  }
  CUDA_TRY(launch_end(s->state64, m, dp, ctl, st));
  CUDA_TRY(cudaEventRecord(s->ev_k1, st));
  s->launches_pending = launches;
  s->trace_pending = 0;
  s->pending = true;
  return finish(s, iterations_out, false);
}

}  // extern "C"
