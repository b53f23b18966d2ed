// Types and launch entry points shared by the kernel translation units.
//
// Translation units and their floating-point contracts:
//   kernels_tables.cu    geodesic backtrace, Fourier projection, departure
//                        records, alpha-ratio cubes -- FP64, built with
//                        -fmad=false (every product rounded once, as on the
//                        reference's CPU)
//   kernels_plain.cu     the plain FP64 step (stream + moments + collide),
//                        LF moments, sources, energy, layout transposes --
//                        FP64, -fmad=false; it evaluates the reference's
//                        expressions in the reference's association order, so
//                        identical inputs give identical bits
//   kernels_step32.cu    the FP32 precision step of the fixed streaming types
//                        and its batched form -- contracted FMAs, packed
//                        records, moment-space lambda iteration
//   kernels_step64.cu    the fast FP64 step of the fixed streaming types --
//                        the same scheme in FP64, contracted FMAs
//   kernels_precision.cu the FP32 precision step of the adaptive streaming
//                        types
//   adjoint.cu           the adjoint of the plain step
//
// Device layouts (one problem, all in HBM):
//   plain state  I[d * nxy + ij]          direction-major FP64, two buffers
//   FP32 adaptive state                   J[d * plane + i + j * pitch], rows
//                                         padded to 16 bytes
//   tiled states (FP32 fixed, fast FP64)  J[ij * dp + d], cell-major, directions
//                                         0..3 repeated after the last (dp = nd + 4
//                                         rounded up to 16 bytes); J = I / alpha^3
//                                         for curved streaming
//   plain record rec64[d * ncell + c]     {i_dep, j_dep, angle coordinate, s^3}
//                                         (absolute grid coordinates of the
//                                         departure point; angle < 0 marks a
//                                         departure inside the excision)
//   FP32 record  rec32[c * nd + d]        packed32 (below), with side records
//                                         {i_dep - i, j_dep - j, angle coordinate,
//                                         s^3 alpha_c^3} for far departures
//   FP64 record  recf[c * nd + d]         packed64 (below), with FP64 side records
//   rk fields    rkf[ij * kRkStride + f]  node-major pack of the 21 metric arrays
//                                         the geodesic right-hand side reads and
//                                         the 2x2 spatial tetrad blocks
//   alpha cubes  acube[ij * 9 + 3(dj+1) + (di+1)] = (alpha_ij / alpha_n)^3 for
//                                         the 3x3 neighbours n of interior ij
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace grlbm
{
constexpr int kRkStride = 32;
enum RkField : int
{
    RF_ALPHA, RF_B1, RF_B2, RF_DA1, RF_DA2, RF_DB11, RF_DB12, RF_DB21, RF_DB22,
    RF_K11, RF_K12, RF_K22, RF_GU11, RF_GU12, RF_GU22,
    RF_DG111, RF_DG112, RF_DG122, RF_DG211, RF_DG212, RF_DG222,
    RF_PAD, // zero: the tetrad blocks start on 16-byte boundaries
    RF_T11, RF_T12, RF_T21, RF_T22, RF_TI11, RF_TI12, RF_TI21, RF_TI22,
    RF_COUNT
};
static_assert(RF_COUNT <= kRkStride, "rk pack stride");
static_assert(RF_DG222 % 2 == 0 && RF_T11 % 2 == 0 && RF_TI11 % 2 == 0 && kRkStride % 2 == 0,
              "fields read in pairs (16-byte loads)");

constexpr int kStepBlock = 128;
// Threads per block of the curved adaptive stream kernels: 16 cells of a row
// times kAdaptiveBlock / 16 directions sharing the row's staged coefficients.
#ifndef GRLBM_ADAPTIVE_BLOCK
#define GRLBM_ADAPTIVE_BLOCK 256
#endif
constexpr int kAdaptiveBlock = GRLBM_ADAPTIVE_BLOCK;
static_assert(kAdaptiveBlock % 32 == 0 && kAdaptiveBlock >= 32 && kAdaptiveBlock <= 1024,
              "whole warps of 16 cells x 2 directions, within the block limit");
constexpr int kMaxDirs = 256;
constexpr int kMaxFourier = 64;

// Directions 0..kStateMirror-1 repeated after the last direction in the
// cell-major states, so that every 5-direction angular window of a node is
// one contiguous run.
constexpr int kStateMirror = 4;

// Where intensity (node ij = i + j nx, direction d) sits in a state buffer:
// element at(ij) * sp + d * plane.  Direction-major layouts have sp = 1 and
// plane = the plane stride; the cell-major layout has sp = dp (the direction
// pitch) and plane = 1, and repeats directions 0..mirror-1 after the last.
struct StateLayout
{
    int64_t nx, pitch, plane; // grid row length, state row pitch (nodes), direction stride (elements)
    int64_t sp = 1;           // node stride (elements)
    int mirror = 0;           // directions repeated after the last one
    __host__ __device__ int64_t at(int64_t ij) const { return pitch == nx ? ij : ij + (ij / nx) * (pitch - nx); }
    __host__ __device__ int64_t elem(int64_t ij, int64_t d) const { return at(ij) * sp + d * plane; }
    static StateLayout dense(int64_t nx, int64_t ny) { return StateLayout{nx, nx, nx * ny}; }
    // FP32 state of the adaptive streaming types: direction-major, rows padded to 16 bytes
    static StateLayout padded32(int64_t nx, int64_t ny)
    {
        const int64_t pitch = (nx + 3) & ~(int64_t)3;
        return StateLayout{nx, pitch, pitch * ny};
    }
    // FP32 state of the fixed streaming types: cell-major, [ij * dp + d] with
    // dp = nd + kStateMirror rounded up to 4 floats (16-byte node records)
    static int direction_pitch(int nd) { return (nd + kStateMirror + 3) & ~3; }
    static StateLayout cell_major32(int64_t nx, int nd)
    {
        return StateLayout{nx, nx, 1, (int64_t)direction_pitch(nd), kStateMirror};
    }
    // FP64 state of the fast form: cell-major, dp = nd + kStateMirror rounded
    // up to 2 doubles (16-byte node records)
    static int direction_pitch64(int nd) { return (nd + kStateMirror + 1) & ~1; }
    static StateLayout cell_major64(int64_t nx, int nd)
    {
        return StateLayout{nx, nx, 1, (int64_t)direction_pitch64(nd), kStateMirror};
    }
    // elements of a buffer of ny rows and nd directions
    int64_t elements(int64_t ny, int nd) const { return sp == 1 ? plane * nd : pitch * ny * sp; }
};

struct GridDev
{
    int64_t nx, ny, nxy, nx_, ny_, ncell;
    // interior node rows [jlo, jhi) the step updates (a slab; all rows by
    // default: 1, ny - 1)
    int64_t jlo, jhi;
    double dx, dy, dt, startx, starty, endx, endy;
    int kind;
    double excision2;
};

#ifdef __CUDACC__
__device__ __forceinline__ bool dev_outside(const GridDev &g, double x, double y)
{
    return x > g.endx || x < g.startx || y > g.endy || y < g.starty;
}
__device__ __forceinline__ bool dev_inside_bh(const GridDev &g, double x, double y)
{
    return g.kind != 0 && x * x + y * y <= g.excision2;
}
#endif

struct GeodesicArgs
{
    GridDev g;
    const double *rkf;
    const double *ss_cx, *ss_cy; // streaming stencil directions (nf)
    int nf;
    double tol;
    int max_trials;
    double *data; // out: [5][cn][nf]: 1/s, x, y, vIF_x, vIF_y of the built cells
    unsigned long long *trials_total;
    int *nonconverged;
    int64_t c0, cn; // the interior cells built: [c0, c0 + cn)
};

struct ProjectArgs
{
    GridDev g;
    int nf;
    const double *data;  // [5][ncell][nf]
    const double *ss_w;  // nf
    const double *basis; // [f][k] = Basis(k, phi_f)
    double *coef;        // [5][nxy][nf]
    int64_t c0, cn;      // the interior cells built (data holds them): [c0, c0 + cn)
};

// Directions per chunk of the adaptive precision-form kernels' moment loops.
constexpr int kChunk = 8;

// Packed departure record of the precision form (uint4, [c * nd + d]):
//   .x  bits  0-17  t, the blend between interpolation rows, in units of 2^-18
//       bits 18-22  row type of the departure's interpolation row
//       bits 23-30  first direction of the 5-direction angular window
//   .y  fx = i_dep - i0, the bilinear fraction, with bit 31 set when the
//       corner column i0 is i (clear: i - 1)
//   .z  fy likewise for the corner row
//   .w  s^3 alpha_c^3 (0 when the departure is excised), with bit 31 set when
//       the departure lies outside the cell's 3x3 neighbourhood (far: read
//       the side record {i_dep - i, j_dep - j, angle coordinate, s^3 alpha_c^3})
namespace packed32
{
constexpr unsigned kTBits = 18, kTypeShift = 18, kStartShift = 23;
} // namespace packed32

// Packed departure record of the fast FP64 form (double4, [c * nd + d]): the
// fractions are stored as 1 + f in [1, 2), whose exponent field is always
// 1023, so the field and the sign bit carry the record's small integers (the
// reader restores the exponent and subtracts 1, exactly):
//   .x  1 + fx, fx = i_dep - i0; sign set when the corner column i0 is i
//       (clear: i - 1); exponent bits 0-4: row type of the interpolation row
//   .y  1 + fy likewise for the corner row (exponent unused)
//   .z  1 + t, the blend between interpolation rows; exponent bits 0-7: the
//       first direction of the 5-direction angular window
//   .w  s^3 alpha_c^3 (0 when excised); sign set when the departure lies
//       outside the cell's 3x3 neighbourhood (far: read the side record
//       {i_dep - i, j_dep - j, angle coordinate, s^3 alpha_c^3})
namespace packed64
{
constexpr unsigned kExpShift = 20;            // the exponent field in the high word
constexpr unsigned kMantHi = 0x000FFFFFu;     // the high word's mantissa bits
constexpr unsigned kOne = 0x3FF00000u;        // the high word of 1.0
} // namespace packed64

struct DepartureArgs
{
    GridDev g;
    int nf, nd, ng;
    const double *coef;  // [5][nxy][nf]
    const double *eval;  // [k][d] = Basis(k, phi_d) at the intensity directions
    const double *alpha; // nxy
    double rot_c, rot_s; // RotationMatrix(0) entries
    double4 *rec64;      // plain records [d * ncell + c] or null
    uint4 *rec32;        // precision records (packed32) [c * nd + d] or null
    float4 *side32;      // precision side records [c * nd + d] or null
    double4 *recf;       // fast FP64 records (packed64) [c * nd + d] or null
    double4 *sidef;      // fast FP64 side records [c * nd + d] or null
    int q, p;            // interpolation row period (row types) and its direction shift
    int row_base[32];    // first window direction of each row type
    int *clamped;
    unsigned long long *far; // packed records marked far (precision form)
    int *row_extent;     // max over departures of the node rows away from the cell a gather reads
    int64_t c0, cn;      // the interior cells built: [c0, c0 + cn)
};

// What a recording plain step writes for the adjoint (indices over the
// interior cells c and directions d of the whole grid).
struct StepRecord
{
    uint8_t *clamp; // [d * ncell + c]: bit q set where corner q was not clamped
    int *cycles;    // [c]: lambda-iteration cycles of the cell (0: no collide)
    double *e0;     // [c]: E of the streamed intensities (first iterate)
};

// One row of the cubic interpolation grid: 4 directions and their weights.
struct __align__(16) IgRow
{
    int4 idx;
    double2 w01, w23;
};
// The same with the weights rounded to FP32 (the precision form).
struct __align__(16) IgRow32
{
    int4 idx;
    float4 w;
};

struct PlainStepArgs
{
    GridDev g;
    int nd, ng;
    const double *Iin;
    double *Iout;
    const double4 *rec;
    const double *w, *n1, *n2; // nd
    const double *cx, *cy;     // nd (flat departures)
    const IgRow *ig_rows;      // ng
    const double *alpha;       // nxy
    const double *acube;       // nxy*9
    const uint8_t *flags;      // nxy: bit0 excised node (no collide), bit1 stream writes 0
    const double *u1, *u2, *lor, *adt, *eta, *k0, *k3, *ka; // k3 = 3 kappa1
    double *mom;               // 6*nxy
    unsigned long long *iter_sum;
    unsigned int *iter_max;
    // adaptive streaming only (null otherwise): rotation angles before and
    // after this step's update (nxy), and the Fourier coefficients
    const double *ang_old, *ang_new;
    const double2 *rot_inv, *rot_new; // per node {sin, cos}: inverse previous rotation, new rotation
    const double *coef; // [5][nf][nxy]: the Fourier coefficients, node index fastest
    int nf;
    double *S; // the streamed values of the step, [d * nxy + ij]
    // 64-bit element offsets in the curved gather: set when the state has 2^32
    // elements or more (and, for tests, when GRLBM_WIDE_OFFSETS=1 at creation)
    bool wide;
};

// The adaptive streaming types in the precision form (direction-major state).
struct PrecStepArgs
{
    GridDev g;
    int nd, ng;
    const float *Iin;
    float *Iout;
    const float *ia3;         // nxy: 1/alpha^3 (scale of the stored state)
    const uint8_t *flags;
    const float *u1, *u2, *lor, *adt, *eta, *k0, *k3, *ka;
    float *mom;               // 6*nxy
    unsigned long long *iter_sum;
    unsigned int *iter_max;
    unsigned pitch, plane;    // state row pitch (a multiple of 4 floats) and plane stride
    const double *ang_old, *ang_new; // rotation angles before and after this step's update (nxy)
    const float2 *rot_inv, *rot_new; // per node {sin, cos}: inverse previous rotation, new rotation
    // [5][nf][nxy]: the Fourier coefficients in FP32, node index fastest, with
    // the X and Y series taken about the node (its coordinates subtracted)
    const float *coef32;
    float inv_dx, inv_dy;            // 1 / dx, 1 / dy
    const float *cx, *cy;            // nd: the stencil's unrotated directions
    const IgRow32 *ig_rows;          // ng: the interpolation grid
    float *S;                        // [d * nxy + ij]: the streamed values of the step
    int nf;
};

// Direction tables of the precision form, passed by value as a kernel
// parameter (uniform constant-bank reads): quadrature weights, rotated
// directions, flat-space departure offsets in cells, and the 18 stencil sums
// of the affine collide map (sum_d w mu_q, times n1, times n2 for
// mu = 1, n1, n2, n1^2, n1 n2, n2^2).
//
// The angular interpolation rows: row g of the interpolation grid blended
// with row g+1 is a 5-direction window with weights W0 + t D.  The grid has
// nGrid = 10 nDir rows, so with q = nGrid / gcd(nDir, nGrid) and
// p = nDir / gcd(nDir, nGrid) row g = q m + r has the weights of row r and
// starts p m directions further on: q row types of 12 floats
// {W0[0..3]}, {D[0..3]}, {W0[4], D[4], first direction of row r, 0}.
constexpr int kMaxRowTypes = 32;
struct __align__(16) DirTable
{
    float w[kMaxDirs], n1[kMaxDirs], n2[kMaxDirs], ox[kMaxDirs], oy[kMaxDirs];
    float wmom[18];
    // both read as float4 (from the parameter space, or from global memory in
    // a batch), so 16-byte aligned
    __align__(16) float rowtab[kMaxRowTypes * 12];
    // moment-sum coefficients per direction: {w, w n1, w n2, w n1^2}, {w n1 n2, w n2^2, n1, n2}
    __align__(16) float dirc[kMaxDirs * 8];
    int q, p;
    float inv_q;
};
static_assert(offsetof(DirTable, rowtab) % 16 == 0 && offsetof(DirTable, dirc) % 16 == 0 &&
                  sizeof(DirTable) % 16 == 0,
              "DirTable float4 members");

struct AdjEntryArgs
{
    GridDev g;
    int nd, ng, curved;
    const double4 *rec;   // plain departure records (curved)
    const IgRow *ig_rows; // interpolation rows (curved)
    const double *alpha, *acube;
    const uint8_t *flags;
    const double *cx, *cy; // intensity directions (flat)
};

struct AdjCollideArgs
{
    GridDev g;
    int nd;
    const double *w;                   // nd
    const uint8_t *flags;              // nxy
    const double *adt, *eta, *k0, *ka; // nxy
    const float *lam;                  // [d * nxy + ij]: adjoint of the step's output intensities
    const double *Iout;                // [d * nxy + ij]: the step's output intensities
    const int *cycles;                 // [c]
    const double *e0;                  // [c]
    float *lamS;                       // [d * ncell + c]: adjoint of the streamed intensities
    double *g_eta, *g_ka, *g_k0;       // nxy: gradients, accumulated
};

// The precision-form step of the fixed streaming types (cell-major state,
// kernels_step32.cu): warps of kStep32Warps per block, each taking tiles of
// tx x ty <= kStep32UnitCells cells from a counter.
constexpr int kStep32Warps = 6;
constexpr int kStep32UnitCells = 16;
constexpr int kStep32MaxSmem = 227 * 1024;
struct Step32Args
{
    GridDev g;
    int nd, ng, dp;          // directions, interpolation rows, direction pitch of the state
    int dps;                 // a node's floats in the staged patch (dp padded to a multiple of 32)
    int tx, ty;              // cells per tile; a warp stages (tx + 2) x (ty + 2) nodes
    int ss, patch_floats;    // row stride of the streamed-value buffer, floats of the patch buffer
    int tiles_x, ntiles;     // tiles per row of tiles, tiles over the slab rows
    const float *Iin;
    float *Iout;
    const uint4 *rec;        // packed records (curved)
    const float4 *side;      // side records (curved)
    const float *ia3;        // nxy: 1/alpha^3, the scale of the stored state (curved)
    const uint8_t *flags;    // nxy: bit0 excised node (no collide), bit1 stream writes 0
    const float *u1, *u2, *lor, *adt, *eta, *k0, *k3, *ka;
    float *mom;              // 6*nxy
    unsigned long long *iter_sum;
    unsigned int *iter_max;
    unsigned *fault;         // set to 1 when a staging copy does not land within its time limit
    // [0] the next tile to take, [1] warps done: zero between launches (the
    // launch's last warp clears both)
    unsigned *tiles;
    CUtensorMap in_map;      // Iin as a 4D tensor, one box per tile patch (encode_state_map32)
};

// The fast FP64 step of the fixed streaming types (cell-major FP64 state,
// kernels_step64.cu): the same warp-per-tile scheme with kStep64Warps warps
// per block.
constexpr int kStep64Warps = 4;
struct Step64Args
{
    GridDev g;
    int nd, ng, dp;          // directions, interpolation rows, direction pitch of the state
    int q;                   // row types of the angular windows (the DirTable64's q)
    int dps;                 // a node's doubles in the staged patch (dp padded to a multiple of 16)
    int tx, ty;              // cells per tile
    int ss, patch_elems;     // row stride of the streamed-value buffer, doubles of the patch buffer
    int tiles_x, ntiles;
    const double *Iin;
    double *Iout;
    const double4 *rec;      // packed records (packed64, curved)
    const double4 *side;     // side records (curved)
    const double *ia3;       // nxy: 1/alpha^3, the scale of the stored state (curved)
    const uint8_t *flags;
    const double *u1, *u2, *lor, *adt, *eta, *k0, *k3, *ka;
    double *mom;             // 6*nxy
    unsigned long long *iter_sum;
    unsigned int *iter_max;
    unsigned *fault;
    unsigned *tiles;         // [0] next tile, [1] warps done (zero between launches)
    CUtensorMap in_map;      // Iin as a 4D tensor, one box per tile patch (encode_state_map64)
};

// Direction tables of the fast FP64 step (device memory, copied into each
// block's shared memory): the angular rows and moment coefficients of
// DirTable in FP64, and the flat departures' products c dt.
struct __align__(16) DirTable64
{
    double rowtab[kMaxRowTypes * 12];
    double dirc[kMaxDirs * 8];
    double wmom[18];
    double cxdt[kMaxDirs], cydt[kMaxDirs];
    int q, p;
    double inv_q;
};

// One problem of a batched precision-form step: its step arguments for
// either buffer parity and its direction tables (device memory).
struct Batch32Item
{
    Step32Args a[2]; // a[k]: the step that reads intensity buffer k
    const DirTable *dt;
    int curved, cur0;
    int mode; // step32_mode(nd): 0 half-warp mode, else the passes per lane
};

int64_t adj_entries_per_source(bool curved);
// slice_start: adj_slices(nd * nxy) + 1 entries
int64_t adj_slices(int64_t n_targets);
cudaError_t adj_build_table(const AdjEntryArgs &a, int64_t *slice_start, unsigned **srcq, float **coef,
                            int64_t *n_entries, cudaStream_t s);
void launch_adj_seed(const GridDev &g, int nd, const double *w, const uint8_t *flags, const double *dLdE, float *lam,
                     cudaStream_t s);
void launch_adj_collide(const AdjCollideArgs &a, cudaStream_t s);
void launch_adj_stream(const int64_t *slice_start, const unsigned *srcq, const float *coef, const uint8_t *clamp,
                       const float *lamS, int64_t n_targets, float *lam, cudaStream_t s);

// Records a message for grlbm_last_error(NULL) (defined in grlbm_capi.cu).
void set_global_error(const char *msg);

// ---- launchers (defined in the kernel translation units) ----
void launch_geodesic(const GeodesicArgs &a, cudaStream_t s);
void launch_project(const ProjectArgs &a, cudaStream_t s);
void launch_departure(const DepartureArgs &a, cudaStream_t s);
void launch_alpha_cube(const GridDev &g, const double *alpha, double *acube, cudaStream_t s);

cudaError_t prepare_step_plain(int smem_bytes);
void launch_step_plain(const PlainStepArgs &a, bool curved, cudaStream_t s, const StepRecord *record = nullptr);
// One block's bounded wait on an mbarrier phase nothing (arrive = 0) or one
// arrival (arrive = 1) completes; synchronous.
cudaError_t run_wait_selftest(int arrive, unsigned long long limit_ns, int *completed, unsigned long long *waited_ns);
// the adaptive streaming types in the precision form: stream, then moments
// and collide (and the rotation update before, the halo moments after)
void launch_step_prec_adaptive(const PrecStepArgs &a, const DirTable &dt, bool curved, cudaStream_t s);

// The fixed streaming types in the precision form (kernels_step32.cu).
// Passes per lane for nd directions (an instantiated count >= nd / 32), or -1.
int step32_passes(int nd);
// Warp buffers: the patch (floats) and the streamed values of the tile's
// cells (row stride s, s = 2 mod 32 >= nd: conflict-free for lanes over the
// directions and for two lanes per cell over interleaved directions).
int step32_s_stride(int nd);
// A node's floats in the staged patch: dp padded to a multiple of 32 (while
// that stays within the TMA box's 256), so that lanes reading neighbouring
// nodes at the same direction offset hit disjoint banks.
int step32_patch_node_floats(int dp);
int step32_patch_floats(int tx, int ty, int dp);
int step32_warp_stride(int tx, int ty, int dp, int nd);
// shared memory of a block of the single-problem kernel, and of the batch kernel
size_t step32_smem(int tx, int ty, int dp, int nd);
size_t step32_batch_smem(int warp_stride);
// bytes at the start of each warp's batch buffer for its copy of the current
// problem's arguments, direction scalars and q row types
int step32_batch_item_bytes(int q);
cudaError_t prepare_step32();
cudaError_t step32_occupancy(int P, bool curved, bool batch, size_t smem, int *blocks, int nd);
// The step's mode for nd directions: 0 for half-warp mode (at most 16
// directions: phases 1 and 3 take two cells at a time), else its passes.
int step32_mode(int nd);
// blocks: the persistent grid (resident blocks per SM times the SMs)
void launch_step32(const Step32Args &a, const DirTable &dt, bool curved, int P, int blocks, cudaStream_t s);
void launch_step_batch32(const Batch32Item *items, const int *first_tile, int n_items, int total_tiles, int flip,
                         unsigned *counters, int P, int blocks, size_t smem, int warp_stride, int s_offset,
                         int item_bytes, cudaStream_t s);
// The TMA map the step stages a cell-major state of nx x ny nodes through,
// for tiles of tx x ty cells.
cudaError_t encode_state_map32(CUtensorMap *map, const float *state, int64_t nx, int64_t ny, int dp, int tx, int ty);

// The fast FP64 step of the fixed streaming types (kernels_step64.cu), with
// the same roles as the step32 functions above.
int step64_passes(int nd);
int step64_s_stride(int nd);
int step64_patch_node_elems(int dp);
int step64_warp_stride(int tx, int ty, int dp, int nd);
size_t step64_smem(int tx, int ty, int dp, int nd, int q);
cudaError_t prepare_step64();
cudaError_t step64_occupancy(int P, bool curved, size_t smem, int *blocks);
void launch_step64(const Step64Args &a, const DirTable64 *dt, bool curved, int P, int blocks, cudaStream_t s);
cudaError_t encode_state_map64(CUtensorMap *map, const double *state, int64_t nx, int64_t ny, int dp, int tx, int ty);

void launch_sources64(double *I, int64_t nxy, int nd, const int64_t *nodes, const double *vals, int64_t nsrc,
                      cudaStream_t s);
// the same into a state of layout L (the fast FP64 form's cell-major state)
void launch_sources64L(double *I, const StateLayout &L, int nd, const int64_t *nodes, const double *vals,
                       int64_t nsrc, cudaStream_t s);
void launch_sources32(float *I, const StateLayout &L, int nd, const int64_t *nodes, const float *vals, int64_t nsrc,
                      cudaStream_t s);
// [5][nxy][nf] -> [5][nf][nxy]
void launch_coef_k_major(const double *coef, double *coef_k, int64_t nxy, int nf, cudaStream_t s);
void launch_moments_lf64(int64_t nxy, const double *mom, const double *lfp, const uint8_t *bh, double *out,
                         cudaStream_t s);
void launch_moments_lf32(int64_t nxy, const float *mom, const double *lfp, const uint8_t *bh, double *out,
                         cudaStream_t s);
void launch_energy64(const GridDev &g, const double *E, double *partial, int nblocks, double *out, cudaStream_t s);
void launch_energy32(const GridDev &g, const float *E, double *partial, int nblocks, double *out, cudaStream_t s);
void launch_to_dirmajor64(const double *in, double *out, int64_t nxy, int nd, cudaStream_t s);
void launch_to_dirmajor32(const double *in, float *out, int64_t nxy, const StateLayout &L, int nd,
                          const float *scale, cudaStream_t s);
void launch_to_cellmajor64(const double *in, double *out, int64_t nxy, int nd, cudaStream_t s);
void launch_to_cellmajor32(const float *in, double *out, int64_t nxy, const StateLayout &L, int nd,
                           const float *scale, cudaStream_t s);
void launch_widen32(const float *in, double *out, int64_t n, cudaStream_t s);
// The fast FP64 form's cell-major state (layout L, stored as I * scale where
// scale is given): from and to the boundary's cell-major [ij][d], and
// ComputeMomentsIF of it.
void launch_to_state64(const double *in, double *out, int64_t nxy, const StateLayout &L, int nd, const double *scale,
                       cudaStream_t s);
void launch_from_state64(const double *in, double *out, int64_t nxy, const StateLayout &L, int nd, const double *scale,
                         cudaStream_t s);
void launch_moments_from_state64(const double *J, int64_t nxy, const StateLayout &L, int nd, const double *w,
                                 const double *n1, const double *n2, const double *scale, double *mom, cudaStream_t s);
// ComputeMomentsIF from the current intensities (FP64 out, 6 * nxy)
// (ang: per-node rotation angles of adaptive streaming, with n1/n2 the
// unrotated stencil directions; null otherwise)
void launch_moments_from_I64(const double *I, int64_t nxy, int nd, const double *w, const double *n1,
                             const double *n2, const double *ang, double *mom, cudaStream_t s);
void launch_moments_from_I32(const float *J, int64_t nxy, const StateLayout &L, int nd, const double *w,
                             const double *n1, const double *n2, const float *scale, const double *ang, double *mom,
                             cudaStream_t s);
// Per node {sin, cos} of the inverse of the previous rotation and of the new
// rotation of an adaptive step (the reference's polynomial trigonometry,
// evaluated once per node instead of once per gather).
void launch_rotation_trig(int64_t nxy, const double *ang_old, const double *ang_new, double2 *rot_inv,
                          double2 *rot_new, cudaStream_t s);
// The same, rounded to FP32 (the precision form).
void launch_rotation_trig32(int64_t nxy, const double *ang_old, const double *ang_new, float2 *rot_inv,
                            float2 *rot_new, cudaStream_t s);
// The FP32 coefficient copy of adaptive streaming in the precision form:
// coef [5][nxy][nf] (FP64) to [5][nf][nxy] (FP32), the node's x and y
// subtracted from the constant terms of the X and Y series in FP64 first.
void launch_coef_about_node32(const GridDev &g, const double *coef, float *coef32, int nf, cudaStream_t s);
void launch_rotation_update32(const GridDev &g, const float *mom, const double *ang_old, double *ang_new,
                              cudaStream_t s);
void launch_zero_halo_moments32(const GridDev &g, float *mom, cudaStream_t s);
} // namespace grlbm
