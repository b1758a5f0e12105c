// Internal layout shared by the host setup (vbd_host.cu) and the kernels
// (vbd_kernels.cu, vbd_persist.cu, vbd_noalloc.cu, vbd_warmstart.cu).
//
// Device data of one solver ("mesh" = one or more independent environments):
//
//   vertices   renumbered so that, inside each environment, the solved
//              vertices of colour 0, 1, ... are contiguous (sorted by valence
//              inside a colour), followed by the "free" active vertices (not
//              coloured or without incident tets: they follow the inertia
//              guess) and then the fixed vertices.
//   u, ut, up, vel   Real4 per vertex: displacement from the rest position,
//              inertia target (w = lumped mass), displacement at step start,
//              velocity.
//   slots      one per incident (vertex, tet) pair, SELL-32 layout: a
//              "chunk" is 32 lanes = 32/TPV vertices x TPV lanes; chunk q has
//              `steps` blocks of 32 slots, block s holds, for lane l, incident
//              tet j = s*TPV + (l % TPV) of vertex l / TPV.  A slot is
//              (n0, n1, n2, rid): the environment-local ids of the tet's
//              other three vertices and the environment-local id of its
//              record (ushort4 or int4, RecordFormat below); padding slots
//              are zero.
//   records    per environment, the distinct (b_n0, p0) (b_n1, p1) (b_n2, w)
//              Real4 triples of its slots (EnvInfo::rbase, nrec):
//              b_n = gradient of the tet's linear shape function of vertex n
//              (a row of Dm^-1, or minus their sum), p0 = V*mu, p1 = V*lambda
//              (material-adjusted), w = the slot's share of the tet's strain
//              energy (1 / solved vertices of the tet).
#pragma once
#include <cstdint>

namespace vbd {

enum Material : int { kSNH = 0, kStVK = 1 };

// status bits written by the kernels (per environment)
enum StatusBits : unsigned {
  kStatNonFinite = 1u,
  kStatGuard = 2u,      // a 3x3 block was not positive definite
  kStatIterCap = 4u,    // max_iter reached without convergence
  kStatTimeout = 8u,
  kStatWarmUsed = 16u,  // the step started from the learned prediction
  kStatBounds = 32u,    // bounds-checked build: a slot index out of range (access skipped)
};

struct EnvInfo {
  int vbase;    // first (global, renumbered) vertex id
  int nv;       // vertices
  int nact;     // active vertices (solved + free) = local ids [0, nact)
  int nsolved;  // solved vertices = local ids [0, nsolved)
  int cbase;    // first colour record in the colour table
  int ncolors;
  int rbase;    // first record of the environment's record table (3 Real4 each)
  int nrec;     // records of the environment (slot record ids are environment-local)
  int tbase;    // first entry of the environment's tet list (DevMesh::tet_slot)
  int ntets;    // tets with a solved vertex
};

struct ColorInfo {
  int vbegin, vend;       // global vertex ids
  int chunk_begin, chunk_end;
};

struct ChunkInfo {
  int block;  // first 32-record block
  int steps;  // number of blocks
};

struct StepParams {
  double dt, tol, kd;
  double g[3];
  int max_iter;
  int strict_spd;
  int warm;  // start from the learned prediction (DevMesh::ws_pred) when it lowers the energy
  int tab_in_smem;  // block mode: the launch's shared memory holds each environment's records
  unsigned long long* trace;  // block mode: 4 words per block of the launch, or null
};

// Grid-mode loop control (one per solver).
struct LoopControl {
  unsigned long long conv_bits;  // max |dx_x+dx_y+dx_z| of the current sweep, as
                                 // the bits of a non-negative double (ordered
                                 // like the values; NaN above +Inf)
  int iter;                      // sweeps done in this step
  unsigned status;
};

// Slot formats (both index the environment's table of distinct records, 3
// Real4 each, so slots that share a tet shape, material and energy weight
// share one entry):
//   kFmtIdx32  int4    (n0, n1, n2, record id)                     16 B/slot
//   kFmtIdx16  ushort4 (n0, n1, n2, record id), all values < 65536  8 B/slot
enum RecordFormat : int { kFmtIdx32 = 1, kFmtIdx16 = 2 };

struct DevMesh {
  const EnvInfo* env;
  const ColorInfo* color;
  const ChunkInfo* chunk;
  const int4* rec_idx;       // kFmtIdx32 slots
  const ushort4* rec_idx16;  // kFmtIdx16 slots
  const void* rec_tab;       // Real4 [n_unique][3]
  // per tet with a solved vertex, for the incremental potential: the slot of
  // its owner (its solved vertex of lowest local id) and the owner's local id
  const int4* tet_slot;
  const int* tet_owner;
  const int* valence;   // per global vertex
  void* u;              // Real4
  void* ut;
  void* up;
  void* vel;
  int* iters;           // per env
  unsigned* status;     // per env
  // per env: the largest |dx| component of the sweep numbered max_iter (the
  // last one allowed), as the bits of a non-negative double; written only on
  // that sweep, read when the step hit max_iter (the reference prints it in
  // its non-convergence warning, vbd_solver.py:581-582)
  unsigned long long* dxmax;
  int n_env;
  int n_vertices;
  int fmt;  // RecordFormat
  // learned warm start
  const float4* wstat;      // per vertex: h, log10(E / (rho h^2)), nu, valence / 20
  const int2* chunk_owner;  // per chunk: (colour index, environment)
  const float4* ws_pred;    // per vertex: predicted correction (xyz), w = 1 if predicted
  // block mode, vbd_step_batched_to: the step's final positions in the
  // caller's order (rest + displacement, float64 [n_vertices][3]) written
  // by each environment's block(s) straight into page-locked host memory
  // (device-mapped pointer), or null
  double* host_out;
  const int* map;      // caller vertex id -> renumbered id
  const double* rest;  // rest positions, caller order, [n_vertices][3]
};

}  // namespace vbd
