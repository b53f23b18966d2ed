/* grlbm.h -- C-ABI of the B200 implementation of the general-relativistic
 * lattice-Boltzmann radiation step of Tom-Olsen/2dRadiation.
 *
 * One context (grlbm_ctx) holds one Radiation problem resident on one GPU:
 * grid, metric arrays, stencil tables, fluid fields, geodesic tables and the
 * intensity double buffer.  Every entry point replaces one piece of the
 * reference's Radiation/Grid/Metric/Stencil interface, cited below as
 * path:line inside the reference project.
 *
 * Conventions
 *  - Every function returns GRLBM_OK (0) or a GRLBM_ERR_* code; none exits the
 *    process.  grlbm_last_error(ctx) describes the last failure (ctx may be
 *    NULL for failures of grlbm_create).
 *  - Host arrays are plain C arrays in the reference's layouts: per-node
 *    arrays have nx*ny entries indexed ij = i + j*nx with nx = nx_+2
 *    (src/Grid.cpp:14, 44-47); intensities are cell-major I[ij*nDir + d]
 *    (src/Radiation.cpp:89-92).  They are copied at call time; the caller
 *    keeps ownership.  Device layouts are private.
 *  - A context is used by one host thread at a time; all GPU work is ordered
 *    on the context's CUDA stream and every entry point returns after its
 *    work has completed (synchronous), except where stated.
 *  - Numbers: GRLBM_PLAIN_FP64 computes everything in IEEE FP64 without
 *    contracted multiply-adds.  Given the same Fourier coefficients
 *    (grlbm_set_fourier_coefficients) its steps reproduce the reference's
 *    IEEE build bit for bit; the coefficients it builds itself match the
 *    reference's to 1e-13 (the reference's pow(x, 0.25) step-size control is
 *    libm's, which is not correctly rounded, so the tables cannot be
 *    bitwise); whole runs match to relative L2 <= 1e-12 on E and F wherever
 *    the reference's own lambda-iteration exit test is not decided by
 *    rounding noise (scattering fluids at rest are: there the reference
 *    itself moves by ~1e-4 under a one-ulp change of its inputs).
 *    GRLBM_PRECISION_FP32 keeps intensities and the stream/collide arithmetic
 *    in FP32 (Kahan-compensated moment sums) on top of FP64 geodesic tables.
 *    GRLBM_FAST_FP64 (fixed streaming types only) computes in FP64 with
 *    contracted multiply-adds, a compact stored state and the lambda
 *    iteration run on the six moments: it matches the reference to relative
 *    L2 <= 1e-12 where the iteration's cycle count is not decided by rounding
 *    noise (always without scattering, kappa0 = kappa1 = 0: the first
 *    cycle's intensities are final there), and to the iteration's tolerance
 *    otherwise.  Batches and the adjoint take the other forms.
 */
#ifndef GRLBM_H
#define GRLBM_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRLBM_OK 0
#define GRLBM_ERR_ARGUMENT 1    /* bad argument or size */
#define GRLBM_ERR_CUDA 2        /* CUDA runtime error or no usable GPU */
#define GRLBM_ERR_STATE 3       /* call out of order (e.g. step before tables) */
#define GRLBM_ERR_UNSUPPORTED 4 /* valid in the reference, not in this build */
#define GRLBM_ERR_NONCONVERGED 5/* an RK45 backtrace hit its substep cap */
#define GRLBM_ERR_HOST 6        /* host-side failure (allocation, table build) */

/* Metric kinds: the reference's Metric subclasses (src/Spacetimes.h:7-45) */
#define GRLBM_MINKOWSKI 0
#define GRLBM_SCHWARZSCHILD 1
#define GRLBM_KERRSCHILD 2

/* StreamingType (src/Config.hh:5-12).  FlatFixed, CurvedFixed, FlatAdaptive
 * and CurvedAdaptive are built for both arithmetic forms; GeodesicFixed (a
 * performance test of the reference) is not built. */
#define GRLBM_FLAT_FIXED 0
#define GRLBM_FLAT_ADAPTIVE 1
#define GRLBM_CURVED_FIXED 2
#define GRLBM_CURVED_ADAPTIVE 3
#define GRLBM_GEODESIC_FIXED 4

/* InitialDataType (src/Config.hh:38-42) */
#define GRLBM_MOMENTS 0
#define GRLBM_INTENSITIES 1

/* Arithmetic forms */
#define GRLBM_PLAIN_FP64 0
#define GRLBM_PRECISION_FP32 1
#define GRLBM_FAST_FP64 2

typedef struct grlbm_ctx grlbm_ctx;

/* Grid(nx_, ny_, start, end, halo = 1) followed by Grid::SetCFL(cfl)
 * (src/Grid.cpp:4-37). */
typedef struct
{
    int64_t nx_, ny_;
    double startx, starty, endx, endy;
    double cfl;
} grlbm_grid_desc;

/* Minkowski / SchwarzSchild / KerrSchild(grid, m, a) (src/Spacetimes.cpp).
 * excision: InsideBH radius in units of m; <= 0 selects the reference's
 * hard-coded 2.1 (src/Spacetimes.cpp:42,81). */
typedef struct
{
    int32_t kind;
    double m, a;
    double excision;
} grlbm_metric_desc;

/* Stencil(n_dir, 0) and Stencil(n_fourier, 0, false) (src/Stencil.cpp:177)
 * plus the Config fields that shape the step (src/Config.hh:45-60). */
typedef struct
{
    int32_t n_dir;
    int32_t n_fourier;
    int32_t streaming_type;
    int32_t precision;
    int32_t keep_source_nodes_active;
    int32_t initial_data_type;
} grlbm_run_desc;

typedef struct
{
    int64_t steps;            /* steps taken since the last reset */
    int32_t max_iterations;   /* Radiation::maxItterationCount (src/Radiation.h:83) */
    double average_iterations;/* sum over steps and interior cells / (steps*(nx-2)*(ny-2)),
                                 as src/Radiation.cpp:856 */
    int64_t rk_substeps;      /* accepted + rejected RK45 trials of the table build */
    int32_t rk_nonconverged;  /* backtraces stopped by the substep cap */
    int32_t departures_off_grid; /* departure points outside the grid (whose
                                    corners are clamped onto it); the reference
                                    reads past its arrays there */
    double table_ms;          /* device time of the last table build */
    int64_t far_departures;   /* precision form: (cell, direction) pairs of the
                                 last table build whose gather leaves the
                                 staged patch (read from global memory) */
} grlbm_stats;

/* ---- context ------------------------------------------------------------
 * Replaces the constructor chain Grid -> Metric subclass -> Stencil x2 ->
 * Radiation(metric, stencil, streamingStencil, config)
 * (exe/main.cpp:540-569, src/Radiation.cpp:3-83): builds the metric arrays,
 * stencil tables and identity Fourier coefficients on the host and uploads
 * them.  device < 0 uses the current CUDA device. */
int grlbm_create(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric,
                 const grlbm_run_desc *run, int32_t device, grlbm_ctx **out);
void grlbm_destroy(grlbm_ctx *ctx);
const char *grlbm_last_error(const grlbm_ctx *ctx);
/* No counterpart in the reference.  Exercises the time limit of the
 * precision step's shared-memory staging wait on `device` (-1: the current
 * one): one block waits on an mbarrier phase that nothing completes
 * (arrive = 0) or that one of its threads completes (arrive = 1), for at most
 * limit_us microseconds (1 .. 1,000,000).  *completed receives 1 when the
 * phase completed and 0 when the wait ran out; *waited_us the wait's length
 * on the device clock.  The kernel returns either way; nothing faults. */
int grlbm_selftest_staging_wait(int32_t device, int32_t arrive, int32_t limit_us, int32_t *completed,
                                double *waited_us);

/* Grid members nx, ny, dx, dy, dt (src/Grid.h:17-21). */
int grlbm_get_grid(const grlbm_ctx *ctx, int64_t *nx, int64_t *ny, double *dx, double *dy,
                   double *dt);

/* ---- inputs (the public buffers callers write, src/Radiation.h:28-39,62-68)
 * Fluid fields kappa0, kappa1, kappaA, eta, ux, uy: nx*ny each. */
int grlbm_set_fields(grlbm_ctx *ctx, const double *kappa0, const double *kappa1,
                     const double *kappaA, const double *eta, const double *ux,
                     const double *uy);
/* isInitialGridPoint (nx*ny bytes), initialI (nx*ny*nDir, cell-major), and
 * initialE_LF..initialPyy_LF (nx*ny each; used when initial_data_type is
 * GRLBM_MOMENTS, may be NULL otherwise).  The source intensities are derived
 * here once, as Radiation::LoadInitialData would (src/Radiation.cpp:103-182). */
int grlbm_set_initial_data(grlbm_ctx *ctx, const uint8_t *is_initial, const double *initial_I,
                           const double *E_LF, const double *Fx_LF, const double *Fy_LF,
                           const double *Pxx_LF, const double *Pxy_LF, const double *Pyy_LF);
/* initialFluxAngle_IF (src/Radiation.h:39, nx*ny): the rotation angles
 * LoadInitialData gives the source nodes under the adaptive streaming types
 * with InitialDataType::Intensities (default 0).  Call before
 * grlbm_set_initial_data. */
int grlbm_set_initial_flux_angle(grlbm_ctx *ctx, const double *angle);
/* Radiation::LoadInitialData (src/Radiation.cpp:128-182): writes the source
 * intensities into the current intensity buffer. */
int grlbm_load_initial_data(grlbm_ctx *ctx);
/* The public member I (src/Radiation.h:71), cell-major, nx*ny*nDir. */
int grlbm_set_intensity(grlbm_ctx *ctx, const double *I);
int grlbm_get_intensity(grlbm_ctx *ctx, double *I);

/* ---- geodesic tables ----------------------------------------------------
 * Radiation::UpdateFourierCoefficients (src/Radiation.cpp:191-237): one FP64
 * RK45 backtrace over dt per interior cell and streaming direction
 * (src/GeodesicEquationSolver.cpp:80-188, tolerance rk_tol; the reference's
 * maxTE is 1e-4), the Fourier projection of 1/s, x, y, vx, vy
 * (src/FourierHarmonics.cpp:33-45), then the per-(cell, direction) departure
 * records the stream reads.  max_substeps bounds each backtrace (0: 1e6);
 * a backtrace that hits it is counted in grlbm_stats.rk_nonconverged and the
 * call returns GRLBM_ERR_NONCONVERGED after finishing the others. */
int grlbm_update_fourier_coefficients(grlbm_ctx *ctx, double rk_tol, int32_t max_substeps);
/* The public coefficient buffers coefficientsS/X/Y/Cx/Cy
 * (src/Radiation.h:75-79, [ij*nF + k]), nx*ny*nF each: set them (as a caller
 * of the reference may) and rebuild the departure records from them, or read
 * them back. */
int grlbm_set_fourier_coefficients(grlbm_ctx *ctx, const double *S, const double *X, const double *Y,
                                   const double *Cx, const double *Cy);
int grlbm_get_fourier_coefficients(grlbm_ctx *ctx, double *S, double *X, double *Y,
                                   double *Cx, double *Cy);

/* ---- time steps -----------------------------------------------------------
 * n_steps iterations of the loop body of Radiation::RunSimulation
 * (src/Radiation.cpp:789-822): LoadInitialData when
 * keep_source_nodes_active, StreamFlatFixed (:380-414) or StreamCurvedFixed
 * (:454-512), ComputeMomentsIF (:239-269) and Collide (:641-736), fused into
 * one kernel per step and replayed from a CUDA graph. */
int grlbm_step(grlbm_ctx *ctx, int32_t n_steps);
/* Same, but only enqueues the work on the context's stream and returns
 * without waiting (for timing with events); grlbm_sync() waits. */
int grlbm_step_async(grlbm_ctx *ctx, int32_t n_steps);
/* No counterpart in the reference.  One step enqueued in parts: updates node
 * rows [j_first, j_end) (within the band of grlbm_set_rows) of the next state
 * from the current one, on the context's stream, without waiting; the first
 * part of a step also applies the active sources.  finish = 1 ends the step
 * (the next state becomes the current one); j_first == j_end with finish = 1
 * only ends it.  The parts of one step must not overlap, and together cover
 * the band.  A slab decomposition steps the band's inner rows while the
 * rows next to it are being exchanged, and its edge rows after.  Not for
 * adaptive streaming or tables rebuilt every step (GRLBM_ERR_UNSUPPORTED). */
int grlbm_step_rows_async(grlbm_ctx *ctx, int64_t j_first, int64_t j_end, int32_t finish);
int grlbm_sync(grlbm_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * work around the library's launches. */
void *grlbm_stream(grlbm_ctx *ctx);

/* Inertial-frame moments E, Fx, Fy, Pxx, Pxy, Pyy as left by the last step
 * (src/Radiation.h:46-51), nx*ny each; any pointer may be NULL. */
int grlbm_get_moments_if(grlbm_ctx *ctx, double *E, double *Fx, double *Fy, double *Pxx,
                         double *Pxy, double *Pyy);
/* Radiation::ComputeMomentsLF (src/Radiation.cpp:270-301): lab-frame moments
 * E_LF, Fx_LF, Fy_LF, Pxx_LF, Pxy_LF, Pyy_LF, F_LF; any pointer may be NULL. */
int grlbm_compute_moments_lf(grlbm_ctx *ctx, double *E, double *Fx, double *Fy, double *Pxx,
                             double *Pxy, double *Pyy, double *F);
/* Global energy: sum of the inertial-frame E over the interior cells, in FP64
 * with a fixed reduction order (bitwise reproducible).  No reference
 * counterpart; the conservation check of the precision form. */
int grlbm_energy(grlbm_ctx *ctx, double *total);
/* Global energy without any device allocation: sum of the interior E of a
 * caller-owned FP64 device array in the per-node layout (nx*ny entries, nx =
 * nx_ + 2), written to the caller-owned device scalar *total, with the work
 * enqueued on `stream` (a cudaStream_t; NULL for the legacy default stream).
 * No counterpart in the reference: it exists for callers that cannot
 * allocate device memory when they need the sum -- loops whose device-memory
 * budget is fixed up front, and host applications that route every device
 * allocation through their own pool (a library cudaMalloc would bypass its
 * accounting and synchronise the device).  Its partial sums live in a fixed
 * file-scope device array of 8192 doubles shared by every call on a device:
 * at most 2,097,152 interior cells (larger grids return GRLBM_ERR_ARGUMENT);
 * calls that overlap on the GPU race on that array; the first call on each
 * device looks the array up and must come before any stream capture.  The
 * call returns once the work is enqueued (asynchronous). */
int grlbm_energy_noalloc(const double *E, int64_t nx_, int64_t ny_, double *total, void *stream);
/* ---- slab decomposition ---------------------------------------------------
 * No counterpart in the reference (it runs on one node, Readme.txt:5-6): one
 * context per GPU holds the whole grid but steps only a band of interior node
 * rows; neighbouring ranks exchange the rows next to their bands between
 * steps.  grlbm_step and grlbm_energy then cover interior node rows
 * [j_first, j_end) only (1 <= j_first < j_end <= ny - 1; the default is all
 * interior rows). */
int grlbm_set_rows(grlbm_ctx *ctx, int64_t j_first, int64_t j_end);
/* (A table build -- grlbm_update_fourier_coefficients or
 * grlbm_set_fourier_coefficients -- covers the interior cells of the band
 * set at that time only; stepping a band outside them returns
 * GRLBM_ERR_STATE.  Set the band first so that each rank builds its own
 * cells' tables.) */
/* Bytes of one node row of the intensity state over all directions:
 * nx * nDir * 8 for GRLBM_PLAIN_FP64; for GRLBM_PRECISION_FP32 with fixed
 * streaming nx * dp * 4, each node holding dp = (nDir + 4 rounded up to a
 * multiple of 4) floats (its directions, then directions 0..3 again); for
 * GRLBM_FAST_FP64 nx * dp * 8 with dp = nDir + 4 rounded up to a multiple of
 * 2 doubles. */
int grlbm_row_bytes(const grlbm_ctx *ctx, int64_t *bytes);
/* Copies node rows [j_first, j_first + n) of the current intensity state
 * (every direction) to (to_buffer = 1) or from (to_buffer = 0) a contiguous
 * device buffer, n * row_bytes bytes, laid out [direction][row][i] for
 * GRLBM_PLAIN_FP64 and [row][i][direction] for GRLBM_PRECISION_FP32 and
 * GRLBM_FAST_FP64.
 * Enqueued on the context's stream; returns before it completes. */
int grlbm_copy_rows(grlbm_ctx *ctx, int64_t j_first, int64_t n, void *buffer, int32_t to_buffer);
/* The per-node fields a band of an adaptive-streaming run also takes from its
 * neighbours before each step, besides the intensities: the current rotation
 * angles (the stream rotates each corner's intensities by that node's angle)
 * and the moments (the angle update averages the flux over the 3x3
 * neighbourhood, src/Radiation.cpp:361-378). */
#define GRLBM_ROWS_ANGLES 1  /* FP64, nx per row; adaptive streaming only */
#define GRLBM_ROWS_MOMENTS 2 /* E, Fx, Fy, Pxx, Pxy, Pyy: 6 x nx values per row, FP32 in the precision form */
/* Bytes of one node row of that field (GRLBM_ERR_UNSUPPORTED for angles
 * without adaptive streaming). */
int grlbm_node_row_bytes(const grlbm_ctx *ctx, int32_t what, int64_t *bytes);
/* Copies node rows [j_first, j_first + n) of that field to (to_buffer = 1) or
 * from (0) a contiguous device buffer of n * bytes-per-row, laid out [row][i]
 * for the angles and [moment][row][i] for the moments.  Enqueued on the
 * context's stream; returns before it completes. */
int grlbm_copy_node_rows(grlbm_ctx *ctx, int32_t what, int64_t j_first, int64_t n, void *buffer, int32_t to_buffer);
/* ---- tiles of the tiled steps -----------------------------------------------
 * No counterpart in the reference.  The GRLBM_PRECISION_FP32 and
 * GRLBM_FAST_FP64 steps of the fixed streaming types run as warps that each
 * take tiles of tile_x x tile_y cells (at most 16), staging each tile's
 * (tile_x + 2) x (tile_y + 2) node patch of the state in shared memory.  The
 * default tile maximises its cells times the kernel's resident blocks per SM
 * (counted up to three), over 8x2, 4x4, 16x1, 4x3, 3x4, 4x2, 2x4, 3x3, 2x2,
 * 2x1, 1x1 in that order of preference; on small grids, with fewer 16-cell
 * tiles than 0.4 (0.2) times the warps then resident, over the tiles of at
 * most 12 (8) cells.  The result does not depend on the tile.
 * GRLBM_ERR_ARGUMENT for more than 16 cells or buffers that do not fit in
 * shared memory; GRLBM_ERR_UNSUPPORTED for other contexts. */
int grlbm_set_tile_shape(grlbm_ctx *ctx, int32_t tile_x, int32_t tile_y);
int grlbm_get_tile_shape(const grlbm_ctx *ctx, int32_t *tile_x, int32_t *tile_y);
/* The most node rows away from its cell that any stream gather reads: the
 * ghost depth a band needs on each side.  From the departure records of the
 * last table build (curved fixed streaming); from the stencil (flat fixed);
 * from dt / dy for any rotated direction (flat adaptive); and for curved
 * adaptive streaming from a bound of the departure's y series over every
 * angle, |c_0 - y| + sqrt 2 sum_k |c_k|, over the band's cells outside the
 * excision. */
int grlbm_departure_rows(grlbm_ctx *ctx, int32_t *rows);
/* ---- batches ----------------------------------------------------------------
 * No counterpart in the reference.  Many problems on one GPU (any form, grid
 * size, direction count and streaming type, with or without active source
 * nodes) stepped together, replayed from CUDA graphs of 32 steps, in one of
 * two kinds of launch shape: each problem's own step with the problems'
 * launch chains running concurrently inside the graph (the default: shape -4
 * below), or one persistent kernel launch per time step over all problems'
 * tiles (only when every problem is a GRLBM_PRECISION_FP32 fixed-streaming
 * one without active source nodes).  Each problem's result is bit-identical
 * to stepping it alone; its context stays usable (moments, intensities,
 * statistics) between batch steps.  Problems that rebuild their tables every
 * step (grlbm_set_update_tables_each_step) are not batched
 * (GRLBM_ERR_UNSUPPORTED).  A batch refers to its contexts: destroy it before
 * them. */
typedef struct grlbm_batch grlbm_batch;
int grlbm_batch_create(grlbm_ctx *const *ctxs, int32_t n, grlbm_batch **out);
void grlbm_batch_destroy(grlbm_batch *batch);
/* Describes the last failure of a batch call (batch may be NULL for
 * grlbm_batch_create). */
const char *grlbm_batch_last_error(const grlbm_batch *batch);
/* n_steps time steps of every problem (synchronous). */
int grlbm_batch_step(grlbm_batch *batch, int32_t n_steps);
/* Sets the launch shape: blocks_per_sm in [1, occupancy limit] for the
 * persistent launch (with the problems' tiles as given or largest problem
 * first; GRLBM_ERR_UNSUPPORTED when the batch holds problems it does not
 * step); 0 for the problems' own steps launched concurrently, each on its own
 * grid; -m (m = 1..8) for the same concurrent launches with the grid of each
 * tiled-form problem k (FP32 and fast FP64 fixed streaming) cut to
 * ceil(m G_k w_k / sum w), at least one block, where G_k is its own grid (its
 * kernel's resident blocks on every SM) and w_k its estimated cost (cells x
 * (directions + 48), x 1.6 for curved streaming, x the form's cost against
 * the FP32 fixed-streaming step): m GPUs' worth of resident blocks shared
 * out, so that the problems' kernels run side by side instead of each
 * filling the GPU in turn. */
int grlbm_batch_set_shape(grlbm_batch *batch, int32_t blocks_per_sm, int32_t largest_first);
/* Times trial_steps steps (rounded up to whole 32-step graphs, replayed as
 * grlbm_batch_step replays them, after an untimed one) for each launch shape
 * -- the persistent launch at resident blocks per SM (the occupancy limit and
 * up to two fewer) with the problems in the order given or largest problem
 * first, where the batch allows it, and the concurrent launches (0, -1, ...,
 * -8) -- and keeps the fastest; then, per size class (tiled-form problems of
 * one form, grid size and direction count) holding at least 2% of the
 * batch's estimated cost, largest class first, times candidate tile shapes
 * (grlbm_set_tile_shape) with the other classes fixed and keeps the
 * fastest.  Every problem is put back in the state it had before the
 * call.  The launch shape is returned in *blocks_per_sm and *largest_first
 * (either may be NULL), the tiles by grlbm_get_tile_shape. */
int grlbm_batch_autotune(grlbm_batch *batch, int32_t trial_steps, int32_t *blocks_per_sm, int32_t *largest_first);
/* ---- adjoint ------------------------------------------------------------------
 * No counterpart in the reference.  Gradients of a loss of the final
 * inertial-frame E with respect to the emissivity, absorption and scattering
 * fields, by a hand-written adjoint of the plain step (GRLBM_PLAIN_FP64) for a
 * fluid at rest without anisotropic scattering (ux = uy = kappa1 = 0; other
 * fields give GRLBM_ERR_UNSUPPORTED).  The stream is transposed through an
 * inverse (CSR) table of its gather built on the device; the adjoint state is
 * FP32 and the gradients accumulate in FP64.  The forward keeps the state
 * every checkpoint_every steps and the backward recomputes each segment. */
typedef struct grlbm_adjoint grlbm_adjoint;
/* After the context's fields and geodesic tables are set; the context must
 * step all interior rows. */
int grlbm_adjoint_create(grlbm_ctx *ctx, int32_t checkpoint_every, grlbm_adjoint **out);
void grlbm_adjoint_destroy(grlbm_adjoint *adj);
const char *grlbm_adjoint_last_error(const grlbm_adjoint *adj);
/* n_steps plain steps of the context from its current intensities, with
 * checkpoints; the context then holds the final state as after grlbm_step. */
int grlbm_adjoint_forward(grlbm_adjoint *adj, int32_t n_steps);
/* dL_dE: dL/dE of the final inertial-frame E (host, nx*ny; only interior
 * nodes matter).  Writes dL/deta, dL/dkappaA, dL/dkappa0 (host, nx*ny each,
 * any may be NULL) for the last forward, with the fields as they were then. */
int grlbm_adjoint_backward(grlbm_adjoint *adj, const double *dL_dE, double *g_eta, double *g_kappaA,
                           double *g_kappa0);
/* Config::updateFourierHarmonics (src/Config.hh:51, src/Radiation.cpp:790-791):
 * when enabled, every step first rebuilds the geodesic tables
 * (grlbm_update_fourier_coefficients with rk_tol and max_substeps), as the
 * reference does at the top of each step; steps are then launched one by one. */
int grlbm_set_update_tables_each_step(grlbm_ctx *ctx, int32_t enabled, double rk_tol, int32_t max_substeps);

/* ---- frames and the simulation loop ---------------------------------------
 * Grid::WriteFrametoCsv (src/Grid.cpp:110-137) for host arrays: writes
 * directory + name + Format(time, 3) + "t <nx>x <ny>y.csv" ("data" when name
 * is NULL or empty; the directory string is used as given, so end it with
 * '/'), creating the directory if needed.  Byte-identical to the
 * reference's file for the same arrays.  No GPU needed. */
int grlbm_host_write_frame_csv(const grlbm_grid_desc *grid, float time, const double *r, const double *g,
                               const double *b, const double *a, const char *directory, const char *name);
/* The frame RunSimulation writes (src/Radiation.cpp:778-781): ComputeMomentsIF
 * of the current intensities (which then become the context's inertial-frame
 * moments), ComputeMomentsLF, and E_LF, Fx_LF, Fy_LF, F_LF to a CSV file. */
int grlbm_write_frame_csv(grlbm_ctx *ctx, float time, const char *directory, const char *name);
/* The time loop of Radiation::RunSimulation (src/Radiation.cpp:748-832) after
 * its set-up (build the tables first): ceil(sim_time / dt) steps from time
 * t0, a frame at t0 when save_initial, one each time write_period has passed,
 * and a final one; no frames when directory is NULL.  *steps_out (may be
 * NULL) receives the step count. */
int grlbm_run_simulation(grlbm_ctx *ctx, double t0, double sim_time, double write_period, int32_t save_initial,
                         const char *directory, int64_t *steps_out);
/* Logger::Write (src/Logger.hh:48-97) after the last grlbm_run_simulation:
 * directory + "/Log.txt" (the directory is created) with the run's creation
 * date, spacetime, grid, stencils, lambda-iteration counts (the average over
 * the run's steps; the maximum since the context was created), its time
 * measurements in seconds -- "Total Time" (the loop), the frame writer under
 * Grid::WriteFrametoCsv's profiler name, the step calls, and the last table
 * build under UpdateFourierCoefficients' -- the computation time (total
 * minus frame writing) and MLUPS, in the reference's format.
 * GRLBM_ERR_STATE before any run. */
int grlbm_write_log(grlbm_ctx *ctx, const char *directory);
/* The same file from given values, without a context or GPU (dates and
 * times as the caller measured them). */
int grlbm_host_write_log(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric, int32_t n_dir,
                         int32_t n_fourier, const char *date, int64_t time_steps, int32_t max_iterations,
                         double average_iterations, const char *const *time_names, const double *seconds,
                         int32_t n_times, const char *directory);
/* A profile session (Profiler::Session::Start/End, src/Profiler.hh:77-141):
 * between grlbm_trace_begin and grlbm_trace_end every table build, step call
 * (grlbm_step), frame write and run loop of the context is recorded with its
 * host start time and duration (microseconds of the profiler's clock), and
 * grlbm_trace_end writes them to `path` in the reference's Chrome-trace JSON
 * (directories created).  GRLBM_ERR_STATE for a second begin or an end
 * without a begin. */
int grlbm_trace_begin(grlbm_ctx *ctx, const char *path);
int grlbm_trace_end(grlbm_ctx *ctx);
/* Lambda-iteration and table-build statistics (src/Radiation.cpp:723-733,
 * 855-857). */
int grlbm_get_stats(grlbm_ctx *ctx, grlbm_stats *stats);

/* ---- host-only helpers (no GPU needed) ----------------------------------
 * The set-up tables the context uploads, for inspection and tests.
 * Stencil(n_order, 0, is_intensity): w, phi, cx, cy (n_order each) and, for an
 * intensity stencil, the cubic interpolation grid InterpolationGrid(10*n_order)
 * (src/Stencil.cpp:4-162, 177-297): ig_index and ig_weight hold 4 entries per
 * row (40*n_order each).  Any output pointer may be NULL. */
int grlbm_host_stencil(int32_t n_order, int32_t is_intensity, double *w, double *phi,
                       double *cx, double *cy, int64_t *ig_index, double *ig_weight);
/* Stencil::fluxToSigmaTable / fluxToNormalizationTable
 * (src/Stencil.cpp:378-455): *size receives the entry count; up to capacity
 * entries are written to inputs, sigma and normalization (may be NULL). */
int grlbm_host_flux_table(int32_t n_order, int32_t *size, double *inputs, double *sigma,
                          double *normalization, int32_t capacity);
/* The 102 per-node metric arrays of the Metric class, in the member order of
 * src/Metric.h:19-65 (102*nx*ny doubles). */
int grlbm_host_metric_arrays(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric,
                             double *out);
/* Number of metric arrays written by grlbm_host_metric_arrays. */
int32_t grlbm_metric_array_count(void);

#ifdef __cplusplus
}
#endif
#endif
