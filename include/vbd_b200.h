/*
 * vbd_b200.h -- C ABI of the B200 Vertex Block Descent solver (libvbd_b200.so).
 *
 * Plain C types only: pointers to host arrays plus sizes, an opaque handle and
 * integer status codes.  Every array argument is a HOST array; the library
 * copies it to the GPU and keeps the solver state resident in device memory.
 * Positions are exchanged in the caller's original vertex order as float64
 * [n_vertices][3], like the reference's wp.vec3d arrays.
 *
 * The entry points replace the reference solver's Python interface
 * (mmichelis/WarpVBD, src/vbd_solver.py):
 *
 *   vbd_create          VBDSolver.__init__            vbd_solver.py:366-498
 *   vbd_step            VBDSolver.step                vbd_solver.py:509-612
 *   vbd_reset           VBDSolver.reset               vbd_solver.py:501-506
 *   vbd_get_positions   new_positions.numpy()         vbd_solver.py:612 (returned array)
 *   vbd_set_positions   step(positions, ...) argument vbd_solver.py:535
 *   vbd_get_color_groups  VBDSolver.color_groups      vbd_solver.py:476-483
 *   vbd_graph_coloring  compute_adjacency_dict + graph_coloring  coloring.py:24-72
 *   vbd_create_batched / vbd_step_batched
 *                       the reference batches by concatenating meshes into one
 *                       solver (examples/run_mass_spring_parallel.py:40-58,
 *                       one global convergence test); here each environment
 *                       keeps its own convergence test and iteration count.
 *
 * Threading: one CUDA stream per handle; a handle is not thread-safe.
 */
#ifndef VBD_B200_H
#define VBD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vbd_solver vbd_solver;

/* ---- status codes ------------------------------------------------------ */
#define VBD_OK 0
/* the sweep loop reached max_iter without meeting the tolerance (the
 * reference prints a warning, vbd_solver.py:581-582); results are valid */
#define VBD_NOT_CONVERGED 1
#define VBD_ERR_INVALID_ARG (-1)
#define VBD_ERR_CUDA (-2)
#define VBD_ERR_SINGULAR_DM (-3)     /* a tet with zero rest volume */
#define VBD_ERR_TOO_MANY_COLORS (-4) /* greedy colouring needs > 256 colours (coloring.py:50) */
#define VBD_ERR_NONFINITE (-5)       /* NaN / Inf appeared in the iterate */
#define VBD_ERR_TIMEOUT (-6)         /* a bounded device-side wait gave up */
#define VBD_ERR_NO_DEVICE (-7)
#define VBD_ERR_UNSUPPORTED (-8)     /* e.g. an environment too large for block mode */
#define VBD_ERR_BOUNDS (-9)          /* bounds-checked build (libvbd_b200_check.so): a slot
                                        index out of range; the access was skipped */

/* ---- flags --------------------------------------------------------------- */
#define VBD_MATERIAL_SNH 0x0  /* Stable Neo-Hookean, vbd_solver.py:107-124 */
#define VBD_MATERIAL_STVK 0x1 /* St. Venant-Kirchhoff, vbd_solver.py:127-144 */
#define VBD_PRECISION_FP32 0x00  /* fp32 state and arithmetic */
#define VBD_PRECISION_FP64 0x10  /* fp64 state and arithmetic */
/* fp64 positions / velocities, fp32 per-tet arithmetic on fp64-formed
 * neighbour offsets: resolves position updates far below a 1e-7 m tolerance
 * at metre-scale displacements, which an fp32 state cannot */
#define VBD_PRECISION_MIXED 0x20
/* colour the mesh on the GPU at creation (vbd_graph_coloring_gpu; the same
 * colours as the host pass) */
#define VBD_GPU_SETUP 0x40
#define VBD_MODE_AUTO 0x000
#define VBD_MODE_BLOCK 0x100    /* one thread block per environment runs the whole step */
#define VBD_MODE_GRAPH 0x200    /* per-colour kernels looped by a CUDA-graph conditional node */
#define VBD_MODE_HOSTLOOP 0x300 /* per-colour kernels, the host reads the convergence test each sweep */
/* one cooperative launch per step: resident blocks run every colour of every
 * sweep, separated by bounded grid barriers (one environment) */
#define VBD_MODE_PERSIST 0x400
#define VBD_MODE_MASK 0xF00
#define VBD_ORDER_INDEX 0x1000  /* keep ascending vertex index inside a colour (default: by valence) */
/* fail a step instead of taking the guarded fallback when a 3x3 block is not
 * positive definite (the reference would produce NaN there) */
#define VBD_STRICT_SPD 0x2000
/* batched block mode: the environments the planner splits over a cluster run
 * in one launch (512 threads per block, shared memory for the largest of
 * them) and all others, one block each, in a second launch on a second stream
 * at the same time (block_threads threads, shared memory for the largest of
 * them, so several blocks share an SM) */
#define VBD_TIERED 0x4000
/* with VBD_TIERED: a third launch, beside the other two, with clusters twice
 * the size (at most 16 blocks) for the environments the planner predicts
 * would otherwise set the step time; the planner uses it only when its
 * duration model says it shortens the step */
#define VBD_TIERED_WIDE 0x80
/* persistent mode: separate the colours of a sweep with grid barriers instead
 * of the default neighbour-scoped readiness (each block waits only for the
 * blocks owning vertices that share a tet with its own) */
#define VBD_PERSIST_GRID_BARRIERS 0x8000
/* block mode: thread blocks per cluster (1 to 16; 0 = automatic).  An
 * environment much heavier than the others is split over all blocks of one
 * cluster, which share its state through distributed shared memory. */
#define VBD_CLUSTER_SHIFT 16
#define VBD_CLUSTER(n) ((n) << VBD_CLUSTER_SHIFT)

/* ---- library / device --------------------------------------------------- */
int vbd_version(void);
const char* vbd_status_string(int status);
/* Text of the last error raised on the calling thread. */
const char* vbd_last_error_message(void);
int vbd_device_count(void);

/* Greedy vertex colouring of the tet 1-ring in vertex index order
 * (coloring.py:24-72).  coloring_out must hold max(tets)+1 entries; that
 * count is written to *n_vertices_out and the colour count to *n_colors_out. */
int vbd_graph_coloring(const int32_t* tets, int n_tets, int32_t* coloring_out,
                       int* n_vertices_out, int* n_colors_out);
/* The same colouring computed on GPU `device` (coloring.py:40-72 replaced by
 * Jones-Plassmann rounds with the vertex index as priority: a vertex takes
 * the smallest colour its lower-indexed neighbours leave free once they all
 * have one, which is exactly what the sequential pass gives it).  Host
 * arrays in and out, as vbd_graph_coloring. */
int vbd_graph_coloring_gpu(const int32_t* tets, int n_tets, int32_t* coloring_out,
                           int* n_vertices_out, int* n_colors_out, int device);

/* ---- solver ------------------------------------------------------------ */
/* VBDSolver.__init__ (vbd_solver.py:367-498).
 *   rest_positions  float64 [n_vertices][3]   initial_positions
 *   tets            int32   [n_tets][4]       elements
 *   densities, youngs_modulus, poissons_ratio float64 [n_tets]
 *   active_mask     uint8   [n_vertices], NULL = all active
 *   damping_coefficient, gravity[3]
 *   coloring        int32   [max(tets)+1] colour per vertex, NULL = computed
 *   flags           VBD_MATERIAL_* | VBD_PRECISION_* | VBD_MODE_* | ...
 *   tpv             lanes per vertex (2, 4, 8, 16), 0 = pick automatically
 *   block_threads   threads per block, 0 = pick automatically
 *   device          CUDA device ordinal */
int vbd_create(const double* rest_positions, int n_vertices, const int32_t* tets, int n_tets,
               const double* densities, const double* youngs_modulus,
               const double* poissons_ratio, const uint8_t* active_mask,
               double damping_coefficient, const double* gravity, const int32_t* coloring,
               int flags, int tpv, int block_threads, int device, vbd_solver** out);

/* n_env independent environments concatenated: environment e owns vertices
 * [env_vertex_offset[e], env_vertex_offset[e+1]) and tets
 * [env_tet_offset[e], env_tet_offset[e+1]) (both arrays hold n_env+1
 * entries); tets use concatenated vertex ids and must stay inside their
 * environment.  Each environment is coloured on its own, which gives the same
 * colours as colouring the concatenation (the environments are disjoint). */
int vbd_create_batched(const double* rest_positions, int n_vertices, const int32_t* tets,
                       int n_tets, const double* densities, const double* youngs_modulus,
                       const double* poissons_ratio, const uint8_t* active_mask,
                       double damping_coefficient, const double* gravity,
                       const int32_t* env_vertex_offset, const int32_t* env_tet_offset,
                       int n_env, int flags, int tpv, int block_threads, int device,
                       vbd_solver** out);

void vbd_destroy(vbd_solver* s);

/* No counterpart in the reference.  Bounds every device-side wait of the
 * persistent mode (VBD_MODE_PERSIST grid barriers): a wait gives up after
 * max_polls polls or max_wait_ns nanoseconds, whichever comes first, and the
 * step then fails with VBD_ERR_TIMEOUT (positions undefined until
 * vbd_reset / vbd_set_positions).  Defaults: 2^26 polls, 2 s. */
int vbd_set_wait_limits(vbd_solver* s, long long max_polls, unsigned long long max_wait_ns);

/* No counterpart in the reference.  Step timeline of the block mode: after
 * vbd_set_trace(s, 1) every step records, per thread block of its
 * environment launches, four words:
 *   [0] global timer at the block's start (ns)   [1] at its end (ns)
 *   [2] (environment << 32) | (rank in its cluster << 16) | SM id
 *   [3] (sweeps << 8) | launch (0: the single or heavy launch, 1: light)
 * (blocks without an environment, padding a cluster, leave zeros).
 * vbd_get_trace copies the last finished step's records, at most `cap`, and
 * writes their number to *count (records = NULL: only the number); the other
 * modes record nothing (count 0). */
int vbd_set_trace(vbd_solver* s, int enable);
int vbd_get_trace(vbd_solver* s, unsigned long long* records, int cap, int* count);

/* VBDSolver.reset (vbd_solver.py:501-506): positions back to rest, velocity 0 */
int vbd_reset(vbd_solver* s);

/* One implicit-Euler step of every environment (vbd_solver.py:509-612):
 * inertia guess, sweeps over the colours until max |dx_x+dx_y+dx_z| < tol or
 * max_iter sweeps, then v = (x_new - x_old)/dt.  With iterations_out != NULL
 * the call blocks and writes the sweep count (per environment for the batched
 * form); with NULL it only enqueues the work on the solver's stream.
 * tol_per_env (batched only) may be NULL to use tol everywhere. */
int vbd_step(vbd_solver* s, double dt, double tol, int max_iter, int* iterations_out);
int vbd_step_batched(vbd_solver* s, double dt, double tol, const double* tol_per_env,
                     int max_iter, int* iterations_out);
/* vbd_step_batched followed by vbd_get_positions, in one blocking call (the
 * reference drivers read every step's positions: run_mass_spring_parallel.py
 * and run_cantilever.py:156).  When positions_out is page-locked, device-mapped
 * host memory (cudaHostAlloc / cudaMallocHost, or torch pin_memory) and the
 * solver runs in block mode, each environment's block writes its final
 * positions there directly as it finishes, overlapping the transfer with the
 * environments still running; otherwise the positions are copied after the
 * step.  The values are the same either way. */
int vbd_step_batched_to(vbd_solver* s, double dt, double tol, const double* tol_per_env,
                        int max_iter, int* iterations_out, double* positions_out);

/* Wait for the enqueued work; returns the status of the last step. */
int vbd_sync(vbd_solver* s);
/* Sweep counts of the last step, n_env entries. */
int vbd_get_iterations(vbd_solver* s, int* iterations_out);
/* Per environment (n_env entries): the largest |dx| component of the last
 * step's final sweep when that step used all max_iter sweeps, else NaN.
 * Replaces the value the reference prints in its non-convergence warning,
 * abs(dxs.numpy()).max() (src/vbd_solver.py:581-582). */
int vbd_get_final_dx(vbd_solver* s, double* final_dx_out);

/* State in the caller's vertex order, float64 [n_vertices][3].  A host
 * pointer to page-locked memory is copied directly (fastest).  Setting the
 * positions keeps the learned warm start's history (valid when the caller
 * hands back what a step produced); vbd_reset clears it. */
int vbd_get_positions(vbd_solver* s, double* positions_out);
int vbd_set_positions(vbd_solver* s, const double* positions);
int vbd_get_velocities(vbd_solver* s, double* velocities_out);
int vbd_set_velocities(vbd_solver* s, const double* velocities);

/* Reference-layout colour table: int32 [n_colors][max_group] of original
 * vertex ids, -1 padded (vbd_solver.py:476-483).  Pass table = NULL to query
 * the sizes first.  Batched solvers report the first environment. */
int vbd_get_color_groups(vbd_solver* s, int32_t* table, int* n_colors, int* max_group);

/* Sizes and the configuration the solver runs with. */
typedef struct vbd_info_t {
  int n_vertices, n_tets, n_env, n_colors, max_valence;
  int mode, tpv, block_threads, precision, material;
  long long n_slots, n_slot_records; /* incident (vertex, tet) pairs; padded records */
  long long device_bytes;
  int n_unique_records; /* entries of the shared slot-record table */
  int record_format;    /* bytes per slot: 8 (16-bit ids) or 16 (32-bit ids) */
  int cluster;          /* block mode: thread blocks per cluster */
  int n_blocks;         /* block mode: blocks of the current work map (> n_env: some
                           environments are split over a cluster) */
  int last_step_launches;     /* kernels the last finished step launched */
  float last_step_kernel_ms;  /* CUDA-event time of its step kernels (the sweeps: block,
                                 persistent or graph launch, both tiers), without the
                                 warm-start feature and inference kernels */
} vbd_info_t;
int vbd_get_info(vbd_solver* s, vbd_info_t* info);

/* The CUDA stream (cudaStream_t) all of the solver's work is enqueued on. */
void* vbd_get_stream(vbd_solver* s);

/* ---- learned warm start (not in the reference) ------------------------------
 * A per-vertex MLP (22 inputs -> 64 SiLU -> 64 SiLU -> 3) predicts each
 * step's converged-minus-inertia correction (scale-free: relative to the
 * vertex's motion scale); the step starts from the
 * prediction when it lowers the incremental potential and from the inertia
 * guess otherwise, then iterates to the same tolerance.  Parameters are fp32
 * in the order W1[64][22] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]; inference
 * runs with bf16 weights.  Feature rows hold vbd_ws_feature_width() floats in
 * the solver's internal vertex order (element 23 = 1 for solved vertices).
 * Pointers named "device" below are CUDA device pointers. */
int vbd_ws_param_count(void);
int vbd_ws_feature_width(void);
/* params: host fp32 [vbd_ws_param_count()] to enable, NULL to disable
 * (block mode only).  The network acts on normalised features and predicts
 * normalised targets; norm (host fp32 [50], NULL = identity) holds the
 * inputs' mean[22] and 1/std[22], then the targets' std[3] and mean[3]. */
int vbd_set_warmstart(vbd_solver* s, const float* params, const float* norm);
/* Features of the coming step of length dt at the current state, into device
 * [n_vertices][feature_width]. */
int vbd_ws_features(vbd_solver* s, double dt, float* features);
/* Row of every caller vertex in the feature, target and prediction arrays:
 * host int32 [n_vertices]. */
int vbd_ws_vertex_rows(vbd_solver* s, int32_t* rows);
/* After a step: the correction it converged to, (x_new - inertia guess) / h,
 * into device [n_vertices][3] (zero rows where features flag 0). */
int vbd_ws_targets(vbd_solver* s, const float* features, float* targets);
/* The model's predicted corrections for given features (the inference the
 * step runs), into device [n_vertices][4] (xyz in metres, w = 1 where
 * predicted). */
int vbd_ws_predict(vbd_solver* s, const float* features, float* predictions);
/* The incremental potential the warm start's check evaluates, per
 * environment, at `positions` (host float64 [n_vertices][3], caller order) for
 * a step of length dt from the current state: the strain energy of every tet
 * with a solved vertex plus, over the solved vertices,
 * m/(2 dt^2) |x - (x0 + dt v + dt^2 g)|^2 (vbd_solver.py:15-146 descend its
 * gradient; the SNH energy differs from the reference's by a constant per
 * tet).  potential_out: host float64 [n_env].  Allocates a scratch state on
 * first use. */
int vbd_incremental_potential(vbd_solver* s, double dt, const double* positions,
                              double* potential_out);
/* Per-environment status bits of the last step: 1 non-finite, 2 guarded
 * step taken, 4 max_iter reached, 16 started from the learned prediction. */
int vbd_get_env_status(vbd_solver* s, uint32_t* status_out);
/* One minibatch of training on device data: rows idx[0..batch) (NULL = the
 * first batch rows) of X [N][feature_width] and Y [N][3]; writes the loss
 * gradient with respect to params into grad and adds sum of squared errors to
 * *loss (device double, may be NULL).  scratch: device floats, at least
 * vbd_mlp_train_scratch_floats(batch) of them (one partial gradient per
 * 32-sample tile; the tiles' partials are added in tile order, so the
 * gradient is the same on every run).  Enqueued on `stream`. */
int vbd_mlp_train_batch(const float* X, const float* Y, const int32_t* idx, int batch,
                        const float* params, float* grad, float* scratch, double* loss,
                        void* stream);
/* Scratch floats vbd_mlp_train_batch needs for a minibatch of `batch` rows:
 * ceil(batch / 32) * (parameter count + 1). */
size_t vbd_mlp_train_scratch_floats(int batch);
/* fp32 forward pass: out [n][3] (device); scratch: not used, may be NULL. */
int vbd_mlp_forward(const float* X, int n, const float* params, float* out, float* scratch,
                    void* stream);
/* Adam update of n parameters, step t >= 1 (device arrays). */
int vbd_mlp_adam(float* params, const float* grad, float* m, float* v, int n, float lr,
                 float beta1, float beta2, float eps, int t, void* stream);

/* vbd_step for callers that may not allocate GPU memory while they step: an
 * application that commits its whole device-memory budget at start-up, or a
 * real-time loop whose per-step code may not call an allocator.  Create the
 * solver once at start-up with vbd_create; this call then allocates nothing
 * (no cudaMalloc / cudaFree, no graph instantiation) and blocks until the step
 * is done.  It has no counterpart in the reference.
 * The sweep's scratch (step parameters, loop control, one convergence partial
 * per thread block) lives in one static device array of 131,200 bytes that
 * every GPU loading the library holds until exit: a mesh whose sweep needs
 * more than 16,384 thread blocks, summed over all its colours (each block
 * takes 8 chunks of 32 / tpv vertices: about one million solved vertices in
 * the whole mesh at 4 lanes per vertex), is rejected with
 * VBD_ERR_UNSUPPORTED, as is a batched solver.  All calls share the array:
 * calls whose GPU work overlaps (other streams, other host threads) race and
 * must be serialised.  The first call on a device resolves the array's device
 * address, so make it before any stream capture on that device.  The step is
 * always a plain one: with the learned warm start enabled the prediction is
 * not used.  vbd_get_info reports its kernel time and launch count. */
int vbd_step_noalloc(vbd_solver* s, double dt, double tol, int max_iter, int* iterations_out);

#ifdef __cplusplus
}
#endif
#endif /* VBD_B200_H */
