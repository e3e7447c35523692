/*
 * C ABI of the B200 FDTD engine (librfn_fdtd.so).
 *
 * Replaces the reference's engine entry points for the 3D FDTD time loop:
 *   cuda_func.solver_run_cu  rfnetwork/core/src/cuda_binding.cpp:20-68
 *   core_func.solver_run     rfnetwork/core/src/core_binding.cpp:350-394
 * both called from FDTD_Solver.solve() at rfnetwork/solver.py:1636-1641, and the
 * engine behind them, SolverFDTD (rfnetwork/core/inc/solver.h:116-176).
 *
 * The reference takes one Python call with a dict of 30 coefficient arrays, a
 * probe list and a monitor list. Here the same data goes through plain
 * pointers and sizes on a handle; rfnetwork_b200/cuda_func.py rebuilds the
 * reference call (same signature, in-place results) on top of these.
 *
 * Conventions
 *  - Every function returns 0 on success and a nonzero FDTD_ERR_* code on
 *    failure; the message is in fdtd_last_error(). Nothing throws across the ABI.
 *  - Coefficient arrays are float32, C order [x][y][z] (z fastest), shape
 *    (nx, ny, nz): the "GPU shapes" the reference packs with gpu=True
 *    (rfnetwork/solver.py:1460-1518).
 *  - Field codes: 0 ex, 1 ey, 2 ez, 3 hx, 4 hy, 5 hz (rfnetwork/solver.py:1560).
 *  - Probe indices are full-grid component indices (the "idx" entry of a
 *    probe dict, rfnetwork/solver.py:1557-1575); the engine applies the Yee
 *    shift of solver_init_probes (rfnetwork/core/src/solver.cpp:503-525).
 *  - A handle is not thread-safe; distinct handles may be used concurrently.
 */
#ifndef RFN_FDTD_H
#define RFN_FDTD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_OK 0
#define FDTD_ERR_ARG 1        /* invalid argument, shape or index */
#define FDTD_ERR_CUDA 2       /* CUDA runtime error */
#define FDTD_ERR_STATE 3      /* call out of order (e.g. run before coefficients) */
#define FDTD_ERR_LIMIT 4      /* a size limit was exceeded */
#define FDTD_ERR_DEVICE 5     /* the kernel reported an error status (a bounded wait expired) */
#define FDTD_ERR_NONFINITE 6  /* the run diverged: a recorded probe value or a final field is NaN or infinite */

typedef struct fdtd_sim fdtd_sim;
typedef struct fdtd_batch fdtd_batch;

/* Statistics of the last prepared / run simulation. */
typedef struct fdtd_stats {
  int nx, ny, nz, nt;
  int n_rows;            /* distinct coefficient rows in the material table */
  int id_bytes;          /* bytes per cell of the material index (1 or 2) */
  int64_t e_split_cells; /* cells whose E components are stored as split fields */
  int64_t h_split_cells; /* cells whose H components are stored as split fields */
  int n_tiles;           /* thread blocks per time step */
  int64_t step_launches; /* time-step kernel launches issued by the last run */
  int64_t dft_launches;  /* DFT kernel launches issued by the last run */
  double last_run_ms;    /* device time of the last run (CUDA events) */
  double compile_ms;     /* host time spent building the material table */
  int variant;           /* step kernel: 0 plain loads, 1 TMA streaming */
  int tile_y;            /* tile height (rows) of the step kernel */
  int stages;            /* shared-memory pipeline stages (TMA kernel) */
  int zchunk;            /* z planes per tile */
  int grid;              /* blocks launched per step */
  int64_t h2d_bytes;     /* host-to-device bytes copied for this simulation so far */
  int64_t d2h_bytes;     /* device-to-host bytes read back from it so far */
  int64_t adjoint_launches; /* reverse-step kernel launches of the last fdtd_adjoint */
  double adjoint_ms;     /* device time of the last fdtd_adjoint (CUDA events) */
  int split_slab[6];     /* PML slab thickness holding split pairs: x-lo, x-hi, y-lo, y-hi, z-lo, z-hi */
  int64_t slab_cells;    /* cells inside those slabs */
  int64_t sparse_split_cells; /* split cells outside them (soft-source cells) */
  int64_t split_bytes;   /* device bytes of the split-pair storage (both time buffers) */
  double tune_ms;        /* host time the step-kernel autotuner spent timing candidate shapes when this
                          * engine was last tiled (0 when the choice came from its process-wide cache) */
  int tune_trials;       /* candidate shapes it timed */
} fdtd_stats;

/* --------------------------------------------------------------- one grid */

/* New simulation of nx x ny x nz cells (SolverFDTD::solver_init_fields,
 * rfnetwork/core/src/solver.cpp:239-349). Device memory is taken on first run. */
int fdtd_create(int nx, int ny, int nz, fdtd_sim** out);

/* Set one of the 30 coefficient arrays by its reference name ("Ca_ex_y",
 * "Db_hz_y2", ...; rfnetwork/solver.py:1473-1518). The data is copied. The
 * last x plane of the Cy, Cz and Dx groups is treated as zero, as
 * solver_init_fields does (rfnetwork/core/src/solver.cpp:294-328). */
int fdtd_set_coefficient(fdtd_sim* s, const char* name, const float* data, int nx, int ny, int nz);

/* As fdtd_set_coefficient, but the array is borrowed, not copied, as the
 * reference's solver_init_fields borrows the numpy arrays it is given
 * (rfnetwork/core/src/solver.cpp:80-117): `data` must stay valid and
 * unchanged until the simulation is destroyed or the coefficient is set
 * again. fdtd_set_box_coefficients copies a borrowed array before writing. */
int fdtd_set_coefficient_view(fdtd_sim* s, const char* name, const float* data, int nx, int ny, int nz);

/* Add a probe (solver_init_probes, rfnetwork/core/src/solver.cpp:465-532).
 * values: n_values >= nt floats, the soft-source amplitude per time step when
 * is_source is nonzero (copied). The recorded field series is read back with
 * fdtd_get_probe_values. Returns the probe's index through *index (may be NULL). */
int fdtd_add_probe(fdtd_sim* s, int field, int i, int j, int k, int is_source, const float* values,
                   int n_values, int* index);

/* Plane field monitor (solver_init_monitors, rfnetwork/core/src/solver.cpp:351-463,
 * GPU layout): axis 0/1/2, position = plane index as in the monitor dict,
 * samples every n_step steps. n_freq == 0: time samples, output float32
 * [nt/n_step+1][N1][N2]. n_freq > 0: phasors, output complex64 [n_freq][N1][N2]
 * accumulated with phase[m][f] (complex64 [nt/n_step+1][n_freq], interleaved re/im). */
int fdtd_add_monitor(fdtd_sim* s, int field, int axis, int position, int n_step, int n_freq,
                     const float* phase, int n_phase_rows, int* index);

/* Running DFT in FP64 of n_series probe combinations at n_freq angular
 * frequencies (radians per time step): X[s][f] = sum_n (sum_t w_t probe_t[n]) e^{-j omega_f n}.
 * Terms t = 0..n_terms-1 give (series, probe, weight). This is the DTFT of
 * rfnetwork/utils.py:14-71 applied to the port voltage / current series of
 * rfnetwork/solver.py:2482-2504, accumulated on the device during the run. */
int fdtd_set_dft(fdtd_sim* s, int n_series, int n_terms, const int* term_series, const int* term_probe,
                 const double* term_weight, int n_freq, const double* omega);

/* Build the material table on the host now (the first run does it otherwise).
 * Needs no GPU. Any output pointer may be NULL. */
int fdtd_compile(fdtd_sim* s, int* n_rows, int64_t* e_split_cells, int64_t* h_split_cells);

/* Copy the compiled material table: ids in the reference order [x][y][z]
 * (nx*ny*nz uint16 row indices) and rows (n_rows x 32 uint32 words: 30
 * coefficients as float bits in the kernel's slot order, flags, probe-list
 * offset). Either output may be NULL. */
int fdtd_get_material_table(fdtd_sim* s, uint16_t* ids, int64_t n_ids, uint32_t* rows, int n_rows);

/* Run nt time steps from zero fields (SolverFDTD::solver_run_cu,
 * rfnetwork/core/src/solver.cu:546-1143). Synchronous. */
int fdtd_run(fdtd_sim* s, int nt);

/* Asynchronous run on the handle's stream; fdtd_synchronize waits for it. */
int fdtd_run_async(fdtd_sim* s, int nt);
int fdtd_synchronize(fdtd_sim* s);

/* Step-kernel selection: variant 0 = plain loads (1 cell per thread, 31 x 7
 * tiles), 1 = TMA streaming, one thread per cell (31 x tile_y tiles, tile_y in
 * {4, 6, 8, 12}; stages = shared-memory plane slots, 3..8). zchunk = z planes
 * per tile (0: derived from the grid). tile_y = 0 with variant 1 autotunes:
 * the first run times a few candidate (tile_y, stages, zchunk, one or two
 * tile lists) shapes on the simulation itself for a few steps and keeps the
 * fastest, remembered per set of grid sizes for the life of the process. The
 * default comes from RFN_FDTD_KERNEL (plain / stream) / RFN_FDTD_TY /
 * RFN_FDTD_STAGES / RFN_FDTD_ZCHUNK or is (1, 0, 6, 0): autotuned streaming.
 * RFN_FDTD_ONE_LIST=1 sends the plain tiles of an explicit streaming shape
 * through the general kernel (one launch per step instead of two).
 * All variants give bit-identical results. The reference has one fixed 8x8x8
 * launch shape (solver.cu:549-557). */
int fdtd_set_kernel(fdtd_sim* s, int variant, int tile_y, int stages, int zchunk);

/* Launch on a caller stream (cudaStream_t passed as void*); NULL = own stream. */
int fdtd_set_stream(fdtd_sim* s, void* stream);

/* Whether runs replay the time loop as one captured CUDA graph (enabled = 1,
 * the default) or issue every launch from the host step by step (0), as the
 * reference's solver_run_cu does (rfnetwork/core/src/solver.cu:1005-1120). */
int fdtd_set_graph(fdtd_sim* s, int enabled);

/* Failure-path testing of the TMA streaming step kernel (variant 1), not for
 * production runs. wait_limit: sleeping polls (each at most ~2 us) after
 * which a shared-memory pipeline wait gives up (0 restores the default of
 * 2^20, about 2 s); withhold_plane >= 0: every block's producer skips the
 * loads of its plane number withhold_plane, so the waits for that plane
 * expire and the run returns FDTD_ERR_DEVICE; -1 issues every plane. The
 * next run captures its time loop again with these values. No counterpart
 * in the reference, whose kernels have no bounded waits. */
int fdtd_set_debug(fdtd_sim* s, unsigned wait_limit, int withhold_plane);

/* Results of the last run. out: n_probes x nt floats, probe-major. */
int fdtd_get_probe_values(fdtd_sim* s, float* out, int n_probes, int nt);
/* out: n_series x n_freq x 2 doubles (re, im). */
int fdtd_get_dft(fdtd_sim* s, double* out, int n_series, int n_freq);
/* Monitor m's output buffer (see fdtd_add_monitor for the layout); n_bytes checked. */
int fdtd_get_monitor(fdtd_sim* s, int m, void* out, int64_t n_bytes);

int fdtd_get_stats(const fdtd_sim* s, fdtd_stats* out);
const char* fdtd_last_error(const fdtd_sim* s);
void fdtd_destroy(fdtd_sim* s);

/* -------------------------------------------------------------- gradients */

/* Like fdtd_run, and keeps a snapshot of the whole field state every `every`
 * steps (ceil(nt/every) snapshots of 6 N floats, plus 12 N when split fields
 * exist) for fdtd_adjoint, which then recomputes each segment from its
 * snapshot. The reference has no gradient path; the functions of this section
 * have no counterpart there. Any later fdtd_run drops the snapshots. */
int fdtd_run_checkpointed(fdtd_sim* s, int nt, int every);

/* Like fdtd_run, and records for fdtd_adjoint the forward history of one
 * gradient box at every step: E and the six H differences of its cells,
 * 9 x box cells x nt floats (a 49 x 49 x 5 box over 4000 steps: 1.7 GB). The
 * adjoint then needs no recomputation. box as for fdtd_adjoint. Any later
 * fdtd_run drops the history. */
int fdtd_run_recorded(fdtd_sim* s, int nt, const int* box);

/* Sets the E-update coefficients of the cells of a box: coefs = 3 x 3 x box
 * cells floats, [ex ey ez][Ca, Cb1, Cb2][x][y][z] (the layout of fdtd_adjoint's
 * gradient); both Ca arrays of a component (Ca_ex_y and Ca_ex_z, ...) take the
 * same value, Cb1 / Cb2 are the first / second Cb array of the component in
 * the coefficient dict's order. The same as fdtd_set_coefficient on those 12
 * arrays, but once the simulation has been compiled it patches the material
 * table in place (one row per box cell) instead of compiling the grid again,
 * so design loops pay no per-iteration compile and keep their captured
 * graphs. The box cells must not be split (no PML, no source). Not while a
 * run of this simulation is in flight. No reference counterpart. */
int fdtd_set_box_coefficients(fdtd_sim* s, const int* box, const float* coefs);

/* Gradient of a real objective J of the last checkpointed or recorded run's
 * device DFT (fdtd_set_dft) with respect to the E-update coefficients of the
 * cells of a box: box = {x0, x1, y0, y1, z0, z1} in cell indices (the
 * coefficient arrays' indices), cells that are not split (no PML, no source);
 * after fdtd_run_recorded, the recorded box.
 *   dJ_dX  n_series x n_freq x 2 doubles: dJ/dRe X + i dJ/dIm X (the gradient
 *          torch hands a complex output)
 *   grad   3 x 3 x box cells doubles, [component ex ey ez][Ca, Cb1, Cb2][x][y][z]:
 *          dJ/d(Ca_e*), dJ/d(first Cb_e*), dJ/d(second Cb_e*) in the coefficient
 *          dict's order (Ca_ex_y with Ca_ex_z held equal, Cb_ex_y, Cb_ex_z, ...)
 * The discrete adjoint runs backwards from the last step, one kernel launch
 * per step, with the transposed update in FP32 and the products accumulated in
 * FP64. Its work buffers (about 36 floats per cell) stay allocated on the
 * simulation for the next call until fdtd_destroy. */
int fdtd_adjoint(fdtd_sim* s, const double* dJ_dX, int n_series, int n_freq, const int* box, double* grad);

/* ---------------------------------------------------------------- batches */

/* Many independent simulations of uneven sizes stepped together: one kernel
 * launch per time step covers the tile work lists of all members, and the time
 * loop is captured as a CUDA graph. The reference has no batched engine; its
 * counterpart is one solver_run_cu call per simulation
 * (rfnetwork/core/src/cuda_binding.cpp:20-68). Members keep their own
 * coefficients, probes and DFT; results are read per member after the run. */
int fdtd_batch_create(fdtd_sim* const* sims, int n_sims, fdtd_batch** out);
int fdtd_batch_run(fdtd_batch* b, int nt);
int fdtd_batch_set_kernel(fdtd_batch* b, int variant, int tile_y, int stages, int zchunk);
int fdtd_batch_set_stream(fdtd_batch* b, void* stream);
int fdtd_batch_get_stats(const fdtd_batch* b, fdtd_stats* out);

/* Gradients of a batch (no reference counterpart): fdtd_batch_run_recorded is
 * fdtd_run_recorded for every member, boxes = n_sims x 6 ints;
 * fdtd_batch_run_checkpointed is fdtd_run_checkpointed for every member (state
 * snapshots every `every` steps), with the boxes fixed at the run. Then
 * fdtd_batch_adjoint runs the adjoints of all members together, one launch per
 * reverse step over all their tiles; after a checkpointed run it replays each
 * segment of all members with one step launch per time step. dJ_dX[i] and
 * grad[i] are member i's arrays, sized as for fdtd_adjoint by its own DFT and
 * box. */
int fdtd_batch_run_recorded(fdtd_batch* b, int nt, const int* boxes);
int fdtd_batch_run_checkpointed(fdtd_batch* b, int nt, int every, const int* boxes);
int fdtd_batch_adjoint(fdtd_batch* b, const double* const* dJ_dX, double* const* grad);
const char* fdtd_batch_last_error(const fdtd_batch* b);
void fdtd_batch_destroy(fdtd_batch* b);

/* ------------------------------------------------------------- far field */

/* One face of the near-to-far-field integration surface: cells of n0 x n1
 * on the plane normal to `axis` at `pos` (meters), indexed along the two other
 * axes in x, y, z order; r0 / r1 their center coordinates along those axes
 * (meters), ds their areas (m^2); J and M the equivalent electric (n x H) and
 * magnetic (-n x E) surface currents, complex64 as interleaved (re, im)
 * floats, [component x y z][frequency][n0][n1]. */
typedef struct fdtd_nf2ff_face {
  int axis;
  int n0, n1;
  float pos;
  const float* r0;
  const float* r1;
  const float* ds;
  const float* J;
  const float* M;
} fdtd_nf2ff_face;

/* Far-field E of the surface currents, normalised by exp(-j beta r) / r
 * (rfnetwork/core/src/postprocess.cpp:130-505, postprocess_nf2ff, bound as
 * core_func.nf2ff at rfnetwork/solver.py:3014): beta [n_freq] wave numbers
 * (1/m), theta [n_theta] and phi [n_phi] in radians; out = 2 x n_freq x
 * n_theta x n_phi complex64 (interleaved floats), polarisations theta, phi.
 * Runs on the current device; errors read with fdtd_global_error. */
int fdtd_nf2ff(const fdtd_nf2ff_face* faces, int n_faces, int n_freq, const float* beta, int n_theta,
               const float* theta, int n_phi, const float* phi, float* out);

/* The engine keeps the device memory of destroyed simulations in a pool of
 * its own per device, so the next solve of a similar size maps nothing new.
 * This returns the pool's unused memory on the current device to the driver,
 * down to keep_bytes of unused reserve, and reports the pool's reserved and
 * in-use bytes afterwards (either pointer may be null). Synchronises the
 * device first. No reference counterpart: the reference allocates and frees
 * per solve (rfnetwork/core/src/solver.cu:560-760, 1100-1140). */
int fdtd_trim_memory(int64_t keep_bytes, int64_t* reserved, int64_t* used);

/* Last error of calls that have no handle (fdtd_create, fdtd_batch_create,
 * fdtd_step_noalloc, fdtd_nf2ff, fdtd_trim_memory), kept per calling thread. */
const char* fdtd_global_error(void);

/* ------------------------------------------------ caller-owned buffers */

/* Device buffers of one grid in the engine's own layout, all allocated and
 * owned by the caller. N = nz * ny * pitch, pitch >= nx.
 *   fields       2 x 6 x N floats: [time buffer][ex ey ez hx hy hz][z][y][pitch];
 *                zero before step 0. Step n reads buffer n & 1 and writes the other.
 *   splits       2 x 12 x N floats: [time buffer][(ex_y ex_z) (ey_z ey_x) (ez_x ez_y)
 *                (hx_y hx_z) (hy_z hy_x) (hz_x hz_y)][z][y][pitch][2], each
 *                component's two splits interleaved per cell; zero before step 0,
 *                8-byte aligned. Touched only for the components that a row's
 *                flags (bits 8..13 of word 30) mark as split, but required.
 *   mat          N uint16 row indices, [z][y][pitch]; columns x >= nx hold 0.
 *                The rows and the per-cell indices (C order [x][y][z]) are what
 *                fdtd_get_material_table returns for a compiled simulation.
 *   rows         n_rows x 32 words, as fdtd_get_material_table returns them.
 *   cell_probes  (probe, field) int32 pairs, one per probe, sorted by the probe's
 *                cell (x * ny + y) * nz + z after the Yee shift of
 *                fdtd_add_probe, ties in probe order; a row's word 31 is the
 *                index of its cell's first pair, bits 16..31 of word 30 the count.
 *   src, rec     n_probes x nt floats: source amplitudes in, recorded values out.
 *   is_src       n_probes int32 flags.
 *   n_rows       rows in `rows` (1 .. 65536); every index in `mat` must be below it.
 *   n_probes     probes (>= 0); every probe range a row names (word 31, count in
 *                bits 16..31 of word 30) must lie in [0, n_probes) of cell_probes.
 * The entry point checks the sizes and pointers it is given but cannot read
 * the caller's buffers: an index or probe range outside these bounds makes
 * the kernel read outside them. */
typedef struct fdtd_device_grid {
  int nx, ny, nz, pitch;
  int nt;
  float* fields;
  float* splits;
  const uint16_t* mat;
  const uint32_t* rows;
  const int32_t* cell_probes;
  const float* src;
  float* rec;
  const int32_t* is_src;
  int n_rows;
  int n_probes;
} fdtd_device_grid;

/* Advance steps n0 .. n0+n_steps-1 of a grid held in caller-owned buffers,
 * enqueued on `stream` (cudaStream_t as void*, NULL = default stream), with
 * the plain step kernel: the same bits as fdtd_run.
 *
 * It allocates nothing. It exists for callers that must not let a library take
 * device memory on its own. Examples are a host framework whose caching
 * allocator owns the GPU's memory and accounts for every byte, and a
 * memory-budgeted service. A cudaMalloc there bypasses the budget, and
 * cudaFree waits for the whole device. The kernel's only data besides the
 * caller's buffers are its grid descriptor and tile list. They live in a fixed
 * static device array of 1 MiB + 1 KiB, which every GPU that loads the library
 * keeps until the process exits.
 * Limits and rules:
 *  - At most 65536 tiles of 31 x 7 cells per z chunk, that is
 *    ceil(nx/31) * ceil(ny/7) <= 65536. Larger grids get FDTD_ERR_LIMIT.
 *  - The first call on a device looks up the array's device address. Make that
 *    first call before any stream capture on the device.
 *  - All calls share the array. Each call rewrites the descriptor and tile list
 *    it uses (a small set-up kernel on `stream`, before the steps), so nothing
 *    in it needs to start at zero. Calls whose work overlaps on the GPU, for
 *    example on two streams, race on it.
 *  - Everything the GPU reads comes from the caller's device buffers and from
 *    launch parameters; no host memory is read after the call returns.
 * Errors are reported through fdtd_global_error(). No counterpart exists in the
 * reference, which allocates its device buffers itself in every
 * solver_run_cu call. */
int fdtd_step_noalloc(const fdtd_device_grid* g, int n0, int n_steps, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RFN_FDTD_H */
