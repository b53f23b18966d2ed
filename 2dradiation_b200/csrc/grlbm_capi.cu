// C-ABI of include/grlbm.h: context management, host<->device transfers,
// the geodesic-table build and the graph-replayed time steps.  Kernels live
// in kernels_tables.cu, kernels_plain.cu and kernels_precision.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/grlbm.h"
#include "approx_math.hpp"
#include "device_common.cuh"
#include "frames.hpp"
#include "host_setup.hpp"
#include "runlog.hpp"

using namespace grlbm;

namespace
{
thread_local std::string g_create_error;

struct DevBuf
{
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf()
    {
        if (p)
            cudaFree(p);
    }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};
} // namespace

struct grlbm_ctx
{
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    // host tables
    GridGeom geo;
    grlbm_metric_desc mdesc{};
    grlbm_run_desc run{};
    StencilTables st, ss;
    MetricArrays M;
    bool fp32 = false;
    bool fast64 = false; // GRLBM_FAST_FP64: cell-major FP64 state, the fast FP64 step
    GridDev gd{};
    StateLayout sl{};          // node positions in the state buffers
    // precision form, fixed streaming: the step's tile shape, passes per lane,
    // persistent grid, and the TMA maps of the state buffers for that tile
    int tile_x = 4, tile_y = 4, passes = 1, step_blocks = 1;
    CUtensorMap in_map[2];
    unsigned *fault = nullptr; // mapped host word: a precision step's staging wait timed out
    int64_t ncell = 0;
    int ng = 0;
    // device buffers (storage type T = double for the plain form, float for the precision form)
    DevBuf I[2], rec, side, w, n1, n2, cx, cy, flags, bhmask, alpha, acube;
    DevBuf cx32, cy32; // the precision form's adaptive streaming: the stencil directions in FP32
    DevBuf dirs64, frame_mom; // FP64 {w, n1, n2} and moments for frame output
    // adaptive streaming: rotation angles (ang[cur] current, ang[cur ^ 1] the
    // next), the source nodes' angles, and initialFluxAngle_IF
    DevBuf ang[2], src_ang_nodes, src_ang_vals;
    DevBuf rot; // adaptive: per node {sin, cos} of the inverse previous and the new rotation
    bool wide_offsets = false; // GRLBM_WIDE_OFFSETS=1 at creation: the 64-bit gather at any size
    int64_t nsrc_ang = 0;
    std::vector<double> flux_angle;
    DevBuf ig_rows, ia3;
    DevBuf coef32; // adaptive streaming in the precision form: FP32 coefficients, X and Y about the node
    DevBuf streamed; // plain form: the streamed values of a step
    DevBuf coef_k;   // adaptive streaming: the coefficients as [5][nf][nxy]
    DirTable dirs{}; // precision-form direction tables (kernel parameter)
    DevBuf dirs64t;  // the fast FP64 form's direction tables (a DirTable64 in device memory)
    DevBuf cu1, cu2, clor, cadt, ceta, ck0, ck3, cka, mom, rkf, lfp;
    DevBuf coef, ss_cx, ss_cy, ss_w, proj_basis, eval_basis, stage;
    DevBuf src_nodes, src_vals, lf_out, energy_partial, energy_out;
    DevBuf tile_ctr; // precision form, fixed streaming: the step's tile counter and retired warps
    // counters: [0] iteration sum, [1] iteration max (low 32 bits), [2] RK45
    // trials, [3] capped backtraces, [4] departures off the grid, [5] row
    // extent of the gathers, [6] far precision-form departures
    DevBuf counters;
    int64_t nsrc = 0;
    int cur = 0;
    bool tables = false;
    // node rows whose interior cells have tables (coefficients and records):
    // the band when they were built
    int64_t table_jlo = 0, table_jhi = 0;
    bool partial = false; // a step enqueued in row ranges (grlbm_step_rows_async) is open
    // the tiled forms keep the records of the built cells only: rec and side
    // hold cells [rec_c0, rec_c0 + rec.bytes / (record size * nd))
    int64_t rec_c0 = 0;
    // config.updateFourierHarmonics: rebuild the tables before every step
    bool update_each_step = false;
    double update_tol = 1e-4;
    int32_t update_max_substeps = 0;
    int64_t steps = 0;
    double table_ms = 0;
    // the last grlbm_run_simulation's Log.txt contents, and a profile session
    RunLog runlog;
    double frame_s = 0; // host time spent writing CSV frames
    bool tracing = false;
    std::string trace_path;
    std::vector<TraceEvent> trace;
    cudaGraphExec_t graph[2] = {nullptr, nullptr}; // kGraphSteps steps from buffer 0 / 1
    ~grlbm_ctx()
    {
        for (auto &g : graph)
            if (g)
                cudaGraphExecDestroy(g);
        if (stream)
            cudaStreamDestroy(stream);
        if (fault)
            cudaFreeHost(fault);
    }
};

namespace grlbm
{
void set_global_error(const char *msg) { g_create_error = msg; }
} // namespace grlbm

namespace
{
// One traced entry point of a profile session (grlbm_trace_begin): the
// event is recorded when the scope ends.
struct TraceScope
{
    grlbm_ctx *ctx;
    const char *name;
    long long t0;
    TraceScope(grlbm_ctx *c, const char *n) : ctx(c), name(n), t0(c && c->tracing ? trace_now_us() : 0) {}
    ~TraceScope()
    {
        if (ctx && ctx->tracing)
            ctx->trace.push_back(TraceEvent{name, t0, trace_now_us(), trace_thread_id()});
    }
};

constexpr const char *kStepName = "grlbm_step (stream, moments, collide)";
constexpr const char *kTablesName = "void Radiation::UpdateFourierCoefficients()";

constexpr int kGraphSteps = 32;
constexpr int kPartialBlocks = 592; // 4 x 148 SMs

int fail(grlbm_ctx *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c)
        c->err = buf;
    else
        g_create_error = buf;
    return code;
}

#define CU(call)                                                                               \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ctx, GRLBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// The precision step gives up on a tile whose staged planes do not land
// within the kernel's time limit and raises the context's fault word; the
// state is then invalid.  Read after a stream synchronisation.
int check_fault(grlbm_ctx *ctx)
{
    if (ctx->fault && *reinterpret_cast<volatile unsigned *>(ctx->fault))
        return fail(ctx, GRLBM_ERR_CUDA,
                    "a precision step's shared-memory staging did not complete within its time limit");
    return GRLBM_OK;
}

int alloc(grlbm_ctx *ctx, DevBuf &b, size_t bytes)
{
    if (b.p && b.bytes == bytes)
        return GRLBM_OK;
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    if (bytes == 0)
        return GRLBM_OK;
    CU(cudaMalloc(&b.p, bytes));
    b.bytes = bytes;
    return GRLBM_OK;
}

template <class T>
int upload(grlbm_ctx *ctx, DevBuf &b, const std::vector<T> &v)
{
    int rc = alloc(ctx, b, v.size() * sizeof(T));
    if (rc)
        return rc;
    if (!v.empty())
        CU(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return GRLBM_OK;
}

// doubles stored in the form's type
int upload_t(grlbm_ctx *ctx, DevBuf &b, const std::vector<double> &v)
{
    if (!ctx->fp32)
        return upload(ctx, b, v);
    std::vector<float> f(v.begin(), v.end());
    return upload(ctx, b, f);
}

size_t tsize(const grlbm_ctx *ctx) { return ctx->fp32 ? sizeof(float) : sizeof(double); }

void invalidate_graphs(grlbm_ctx *ctx)
{
    for (auto &g : ctx->graph)
        if (g)
        {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// per-node factor between the precision form's stored state and I (null: none)
const float *state_scale(const grlbm_ctx *ctx)
{
    const int st = ctx->run.streaming_type;
    return (ctx->fp32 && (st == GRLBM_CURVED_FIXED || st == GRLBM_CURVED_ADAPTIVE)) ? ctx->ia3.as<float>() : nullptr;
}

// Arguments of the adaptive precision-form step that reads intensity buffer `from`.
PrecStepArgs prec_args(grlbm_ctx *ctx, int from)
{
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    PrecStepArgs a{};
    a.g = ctx->gd;
    a.nd = ctx->st.n;
    a.ng = ctx->ng;
    a.Iin = ctx->I[from].as<float>();
    a.Iout = ctx->I[from ^ 1].as<float>();
    a.ia3 = ctx->ia3.as<float>();
    a.flags = ctx->flags.as<uint8_t>();
    a.u1 = ctx->cu1.as<float>();
    a.u2 = ctx->cu2.as<float>();
    a.lor = ctx->clor.as<float>();
    a.adt = ctx->cadt.as<float>();
    a.eta = ctx->ceta.as<float>();
    a.k0 = ctx->ck0.as<float>();
    a.k3 = ctx->ck3.as<float>();
    a.ka = ctx->cka.as<float>();
    a.mom = ctx->mom.as<float>();
    a.iter_sum = cnt;
    a.iter_max = reinterpret_cast<unsigned int *>(cnt + 1);
    a.pitch = (unsigned)ctx->sl.pitch;
    a.plane = (unsigned)ctx->sl.plane;
    // the angles are set per step
    a.coef32 = ctx->coef32.as<float>();
    a.inv_dx = (float)(1.0 / ctx->gd.dx);
    a.inv_dy = (float)(1.0 / ctx->gd.dy);
    a.cx = ctx->cx32.as<float>();
    a.cy = ctx->cy32.as<float>();
    a.ig_rows = ctx->ig_rows.as<IgRow32>();
    a.S = ctx->streamed.as<float>();
    a.nf = ctx->ss.n;
    return a;
}

bool is_fixed32(const grlbm_ctx *ctx)
{
    return ctx->fp32 && (ctx->run.streaming_type == GRLBM_FLAT_FIXED || ctx->run.streaming_type == GRLBM_CURVED_FIXED);
}
// the warp-per-tile steps on a cell-major state: FP32 fixed streaming and the fast FP64 form
bool is_tiled(const grlbm_ctx *ctx) { return is_fixed32(ctx) || ctx->fast64; }

// per-node factor between the fast FP64 form's stored state and I (null: none)
const double *state_scale64(const grlbm_ctx *ctx)
{
    return (ctx->fast64 && ctx->run.streaming_type == GRLBM_CURVED_FIXED) ? ctx->ia3.as<double>() : nullptr;
}

int step32_tiles_x(const grlbm_ctx *ctx) { return (int)((ctx->gd.nx_ + ctx->tile_x - 1) / ctx->tile_x); }
int step32_tiles(const grlbm_ctx *ctx)
{
    const int64_t rows = ctx->gd.jhi - ctx->gd.jlo;
    return rows <= 0 ? 0 : step32_tiles_x(ctx) * (int)((rows + ctx->tile_y - 1) / ctx->tile_y);
}

// Arguments of the precision-form step of the fixed streaming types that
// reads intensity buffer `from`.
Step32Args step32_args(grlbm_ctx *ctx, int from)
{
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    Step32Args a{};
    a.g = ctx->gd;
    a.nd = ctx->st.n;
    a.ng = ctx->ng;
    a.dp = (int)ctx->sl.sp;
    a.dps = step32_patch_node_floats(a.dp);
    a.tx = ctx->tile_x;
    a.ty = ctx->tile_y;
    a.ss = step32_s_stride(a.nd);
    a.patch_floats = step32_patch_floats(a.tx, a.ty, a.dp);
    a.tiles_x = step32_tiles_x(ctx);
    a.ntiles = step32_tiles(ctx);
    a.Iin = ctx->I[from].as<float>();
    a.Iout = ctx->I[from ^ 1].as<float>();
    a.rec = ctx->rec.as<uint4>() - ctx->rec_c0 * a.nd;
    a.side = ctx->side.as<float4>() - ctx->rec_c0 * a.nd;
    a.ia3 = ctx->ia3.as<float>();
    a.flags = ctx->flags.as<uint8_t>();
    a.u1 = ctx->cu1.as<float>();
    a.u2 = ctx->cu2.as<float>();
    a.lor = ctx->clor.as<float>();
    a.adt = ctx->cadt.as<float>();
    a.eta = ctx->ceta.as<float>();
    a.k0 = ctx->ck0.as<float>();
    a.k3 = ctx->ck3.as<float>();
    a.ka = ctx->cka.as<float>();
    a.mom = ctx->mom.as<float>();
    a.iter_sum = cnt;
    a.iter_max = reinterpret_cast<unsigned int *>(cnt + 1);
    a.fault = ctx->fault;
    a.tiles = ctx->tile_ctr.as<unsigned>();
    a.in_map = ctx->in_map[from];
    return a;
}

// Arguments of the fast FP64 step that reads intensity buffer `from`.
Step64Args step64_args(grlbm_ctx *ctx, int from)
{
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    Step64Args a{};
    a.g = ctx->gd;
    a.nd = ctx->st.n;
    a.ng = ctx->ng;
    a.dp = (int)ctx->sl.sp;
    a.q = ctx->dirs.q;
    a.dps = step64_patch_node_elems(a.dp);
    a.tx = ctx->tile_x;
    a.ty = ctx->tile_y;
    a.ss = step64_s_stride(a.nd);
    a.patch_elems = (((a.tx + 2) * (a.ty + 2) * a.dps + 15) / 16) * 16;
    a.tiles_x = step32_tiles_x(ctx);
    a.ntiles = step32_tiles(ctx);
    a.Iin = ctx->I[from].as<double>();
    a.Iout = ctx->I[from ^ 1].as<double>();
    a.rec = ctx->rec.as<double4>() - ctx->rec_c0 * a.nd;
    a.side = ctx->side.as<double4>() - ctx->rec_c0 * a.nd;
    a.ia3 = ctx->ia3.as<double>();
    a.flags = ctx->flags.as<uint8_t>();
    a.u1 = ctx->cu1.as<double>();
    a.u2 = ctx->cu2.as<double>();
    a.lor = ctx->clor.as<double>();
    a.adt = ctx->cadt.as<double>();
    a.eta = ctx->ceta.as<double>();
    a.k0 = ctx->ck0.as<double>();
    a.k3 = ctx->ck3.as<double>();
    a.ka = ctx->cka.as<double>();
    a.mom = ctx->mom.as<double>();
    a.iter_sum = cnt;
    a.iter_max = reinterpret_cast<unsigned int *>(cnt + 1);
    a.fault = ctx->fault;
    a.tiles = ctx->tile_ctr.as<unsigned>();
    a.in_map = ctx->in_map[from];
    return a;
}

// shared memory and resident blocks per SM of the context's tiled step at a tile shape
int tiled_fit(grlbm_ctx *ctx, int tx, int ty, size_t *smem, int *per_sm)
{
    const int dp = (int)ctx->sl.sp;
    const bool curved = ctx->run.streaming_type == GRLBM_CURVED_FIXED;
    *smem = ctx->fast64 ? step64_smem(tx, ty, dp, ctx->st.n, curved ? ctx->dirs.q : 0) : step32_smem(tx, ty, dp, ctx->st.n);
    *per_sm = 0;
    if (*smem > (size_t)kStep32MaxSmem)
        return GRLBM_OK;
    if (ctx->fast64)
        CU(step64_occupancy(ctx->passes, curved, *smem, per_sm));
    else
        CU(step32_occupancy(ctx->passes, curved, false, *smem, per_sm, ctx->st.n));
    return GRLBM_OK;
}

// Sets the tile shape of the tiled step (FP32 fixed streaming, fast FP64):
// the TMA maps of the state buffers for its patch, and the persistent grid at
// its occupancy.
int set_step32_tile(grlbm_ctx *ctx, int tx, int ty)
{
    const int dp = (int)ctx->sl.sp;
    if (tx < 1 || ty < 1 || tx * ty > kStep32UnitCells)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "tile %dx%d: at least 1 and at most %d cells", tx, ty, kStep32UnitCells);
    size_t smem = 0;
    int per_sm = 0, sms = 0;
    int rc = tiled_fit(ctx, tx, ty, &smem, &per_sm);
    if (rc)
        return rc;
    if (smem > (size_t)kStep32MaxSmem)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "tile %dx%d: its patch of %d directions needs %zu bytes of shared memory",
                    tx, ty, ctx->st.n, smem);
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (per_sm < 1)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "tile %dx%d does not fit on an SM", tx, ty);
    for (int k = 0; k < 2; k++)
    {
        const cudaError_t e =
            ctx->fast64
                ? encode_state_map64(&ctx->in_map[k], ctx->I[k].as<double>(), ctx->geo.nx, ctx->geo.ny, dp, tx, ty)
                : encode_state_map32(&ctx->in_map[k], ctx->I[k].as<float>(), ctx->geo.nx, ctx->geo.ny, dp, tx, ty);
        if (e != cudaSuccess)
            return fail(ctx, GRLBM_ERR_CUDA, "TMA map of the state: %s", cudaGetErrorString(e));
    }
    ctx->tile_x = tx;
    ctx->tile_y = ty;
    ctx->step_blocks = per_sm * sms;
    invalidate_graphs(ctx);
    return GRLBM_OK;
}

// The node rows a curved adaptive step reads away from the band's cells: the
// series of the departure's y about the node, c_0 - y + sum_k c_k b_k(phi)
// with |b_k| <= sqrt 2, is bounded by |c_0 - y| + sqrt 2 sum_k |c_k| for every
// angle; cells inside the excision stream zeros and are skipped.  The corners
// are floor(jt) and floor(jt) + 1, and 1e-3 row absorbs the FP32 form's
// roundings of the series and of jt.
int adaptive_departure_rows(grlbm_ctx *ctx, int32_t *rows)
{
    if (!ctx->tables)
        return fail(ctx, GRLBM_ERR_STATE, "departure rows need the Fourier coefficients");
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    const int nf = ctx->ss.n;
    const int64_t nx = ctx->gd.nx, nxy = ctx->gd.nxy, per = nxy * nf;
    const int64_t first = ctx->gd.jlo * nx, count = (ctx->gd.jhi - ctx->gd.jlo) * nx;
    std::vector<double> cy((size_t)count * nf);
    std::vector<uint8_t> fl((size_t)count);
    CU(cudaMemcpy(cy.data(), ctx->coef.as<double>() + 2 * per + first * nf, cy.size() * sizeof(double),
                  cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(fl.data(), ctx->flags.as<uint8_t>() + first, fl.size(), cudaMemcpyDeviceToHost));
    double far = 0.0;
    for (int64_t n = 0; n < count; n++)
    {
        const int64_t i = (first + n) % nx, j = (first + n) / nx;
        if (i < 1 || i > ctx->gd.nx_ || (fl[(size_t)n] & 2))
            continue;
        const double *c = cy.data() + (size_t)n * nf;
        double b = std::fabs(c[0] - (ctx->geo.starty + (double)j * ctx->geo.dy));
        for (int k = 1; k < nf; k++)
            b += std::sqrt(2.0) * std::fabs(c[k]);
        far = std::max(far, b / ctx->geo.dy);
    }
    *rows = (int32_t)std::floor(far + 1e-3) + 1;
    return GRLBM_OK;
}

// The default tile: the candidate with the most cells times resident blocks
// per SM (counted up to three), the first in this order on a tie.  Tile
// sweeps at 400^2 curved scattering with 16 to 96 directions found this
// rule's pick within 1% of the fastest in both tiled forms: 8x2 where 16-cell
// tiles keep their occupancy; 4x4 for FP32 at 32 directions (three blocks
// per SM against two for 8x2's wider patch: 64.5 against 72.6 us) and at 64
// (8x2 drops to one block per SM: 128 against 91 us); 4x3 for FP64 at 64
// directions (172 us, against 243-248 us for the 16-cell tiles at one block).
//
// Small grids leave most warps without a tile: with fewer 16-cell tiles (of
// the rows stepped) than 0.4 (0.2) times the warps resident at that pick, the
// rule picks among tiles of at most 12 (8) cells.  Swept at 64^2-128^2 with
// 16-64 directions in both tiled forms, this took the FP32 step within 3% and
// the fast FP64 step within 8% of the fastest shape, where the 16-cell pick
// was up to 27% slower (64^2 x 64 curved, FP32: 11.3 against 15.1 us; the
// 100^2 x 20 flat beam: 9.3 against 9.9 us).  Not covered: tile counts just
// above one wave of warps (fast FP64 at 200^2 x 32: 4x4 34.8 us, its second
// wave 40% full, against 31.6 us for 4x3).
int default_step32_tile(grlbm_ctx *ctx)
{
    static const int cand[][2] = {{8, 2}, {4, 4}, {16, 1}, {4, 3}, {3, 4}, {4, 2}, {2, 4}, {3, 3}, {2, 2}, {2, 1}, {1, 1}};
    const int nc = (int)(sizeof cand / sizeof cand[0]);
    int max_cells = kStep32UnitCells;
    for (int pass = 0; pass < 2; pass++)
    {
        int best = -1, best_score = 0, best_per_sm = 0;
        for (int ci = 0; ci < nc; ci++)
        {
            if (cand[ci][0] * cand[ci][1] > max_cells)
                continue;
            size_t smem = 0;
            int per_sm = 0;
            const int rc = tiled_fit(ctx, cand[ci][0], cand[ci][1], &smem, &per_sm);
            if (rc)
                return rc;
            const int score = cand[ci][0] * cand[ci][1] * std::min(per_sm, 3);
            if (score > best_score)
                best = ci, best_score = score, best_per_sm = per_sm;
        }
        if (best < 0)
            return fail(ctx, GRLBM_ERR_ARGUMENT, "no tile of %d directions fits on an SM", ctx->st.n);
        if (pass == 0)
        {
            int sms = 0;
            CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
            const double warps = (double)best_per_sm * sms * (ctx->fast64 ? kStep64Warps : kStep32Warps);
            const double tiles16 = (double)(ctx->gd.jhi - ctx->gd.jlo) * ctx->gd.nx_ / kStep32UnitCells;
            max_cells = tiles16 < 0.2 * warps ? 8 : (tiles16 < 0.4 * warps ? 12 : kStep32UnitCells);
            if (max_cells < kStep32UnitCells)
                continue;
        }
        return set_step32_tile(ctx, cand[best][0], cand[best][1]);
    }
    return GRLBM_OK;
}


// Arguments of the plain step that reads intensity buffer `from`.
PlainStepArgs plain_args(grlbm_ctx *ctx, int from)
{
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    PlainStepArgs a{};
    a.g = ctx->gd;
    a.nd = ctx->st.n;
    a.ng = ctx->ng;
    a.wide = ctx->wide_offsets || (uint64_t)ctx->st.n * (uint64_t)ctx->gd.nxy > 0xFFFFFFFFull;
    a.Iin = ctx->I[from].as<double>();
    a.Iout = ctx->I[from ^ 1].as<double>();
    a.rec = ctx->rec.as<double4>();
    a.w = ctx->w.as<double>();
    a.n1 = ctx->n1.as<double>();
    a.n2 = ctx->n2.as<double>();
    a.cx = ctx->cx.as<double>();
    a.cy = ctx->cy.as<double>();
    a.ig_rows = ctx->ig_rows.as<IgRow>();
    a.alpha = ctx->alpha.as<double>();
    a.acube = ctx->acube.as<double>();
    a.flags = ctx->flags.as<uint8_t>();
    a.u1 = ctx->cu1.as<double>();
    a.u2 = ctx->cu2.as<double>();
    a.lor = ctx->clor.as<double>();
    a.adt = ctx->cadt.as<double>();
    a.eta = ctx->ceta.as<double>();
    a.k0 = ctx->ck0.as<double>();
    a.k3 = ctx->ck3.as<double>();
    a.ka = ctx->cka.as<double>();
    a.mom = ctx->mom.as<double>();
    a.iter_sum = cnt;
    a.iter_max = reinterpret_cast<unsigned int *>(cnt + 1);
    a.S = ctx->streamed.as<double>();
    return a;
}

bool is_curved(const grlbm_ctx *ctx)
{
    return ctx->run.streaming_type == GRLBM_CURVED_FIXED || ctx->run.streaming_type == GRLBM_CURVED_ADAPTIVE;
}
bool is_adaptive(const grlbm_ctx *ctx)
{
    return ctx->run.streaming_type == GRLBM_FLAT_ADAPTIVE || ctx->run.streaming_type == GRLBM_CURVED_ADAPTIVE;
}

// The step's tables exist for the band (curved streaming).
int check_tables(grlbm_ctx *ctx)
{
    if (!is_curved(ctx))
        return GRLBM_OK;
    if (!ctx->tables)
        return fail(ctx, GRLBM_ERR_STATE, "curved streaming needs grlbm_update_fourier_coefficients first");
    if (ctx->gd.jlo < ctx->table_jlo || ctx->gd.jhi > ctx->table_jhi)
        return fail(ctx, GRLBM_ERR_STATE,
                    "the geodesic tables cover rows [%lld, %lld) only; rebuild them for the band [%lld, %lld)",
                    (long long)ctx->table_jlo, (long long)ctx->table_jhi, (long long)ctx->gd.jlo,
                    (long long)ctx->gd.jhi);
    return GRLBM_OK;
}

// Enqueue one step starting from buffer `from` (no sync).
// (sources: LoadInitialData at the top of the step; off for the second and
// later row ranges of a step enqueued in parts.  blocks: the tiled forms'
// grid, 0 for the context's own)
int enqueue_step(grlbm_ctx *ctx, int from, bool sources = true, int blocks = 0)
{
    const bool curved = is_curved(ctx);
    if (blocks <= 0)
        blocks = ctx->step_blocks;
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    if (ctx->fast64)
    {
        if (sources && ctx->run.keep_source_nodes_active && ctx->nsrc > 0)
            launch_sources64L(ctx->I[from].as<double>(), ctx->sl, ctx->st.n, ctx->src_nodes.as<int64_t>(),
                              ctx->src_vals.as<double>(), ctx->nsrc, ctx->stream);
        launch_step64(step64_args(ctx, from), ctx->dirs64t.as<DirTable64>(), curved, ctx->passes, blocks,
                      ctx->stream);
    }
    else if (ctx->fp32)
    {
        if (sources && ctx->run.keep_source_nodes_active && ctx->nsrc > 0)
            launch_sources32(ctx->I[from].as<float>(), ctx->sl, ctx->st.n, ctx->src_nodes.as<int64_t>(),
                             ctx->src_vals.as<float>(), ctx->nsrc, ctx->stream);
        if (!is_adaptive(ctx))
            launch_step32(step32_args(ctx, from), ctx->dirs, curved, ctx->passes, blocks, ctx->stream);
        else
        {
            PrecStepArgs a = prec_args(ctx, from);
            // LoadInitialData also sets the source nodes' angles (src/Radiation.cpp:170-176)
            if (sources && ctx->run.keep_source_nodes_active && ctx->nsrc_ang > 0)
                launch_sources64(ctx->ang[from].as<double>(), ctx->gd.nxy, 1, ctx->src_ang_nodes.as<int64_t>(),
                                 ctx->src_ang_vals.as<double>(), ctx->nsrc_ang, ctx->stream);
            a.ang_old = ctx->ang[from].as<double>();
            a.ang_new = ctx->ang[from ^ 1].as<double>();
            a.rot_inv = ctx->rot.as<float2>();
            a.rot_new = ctx->rot.as<float2>() + ctx->gd.nxy;
            launch_step_prec_adaptive(a, ctx->dirs, curved, ctx->stream);
        }
    }
    else
    {
        if (sources && ctx->run.keep_source_nodes_active && ctx->nsrc > 0)
            launch_sources64(ctx->I[from].as<double>(), ctx->gd.nxy, ctx->st.n, ctx->src_nodes.as<int64_t>(),
                             ctx->src_vals.as<double>(), ctx->nsrc, ctx->stream);
        PlainStepArgs a = plain_args(ctx, from);
        if (is_adaptive(ctx))
        {
            // LoadInitialData also sets the source nodes' angles (src/Radiation.cpp:170-176)
            if (sources && ctx->run.keep_source_nodes_active && ctx->nsrc_ang > 0)
                launch_sources64(ctx->ang[from].as<double>(), ctx->gd.nxy, 1, ctx->src_ang_nodes.as<int64_t>(),
                                 ctx->src_ang_vals.as<double>(), ctx->nsrc_ang, ctx->stream);
            a.ang_old = ctx->ang[from].as<double>();
            a.ang_new = ctx->ang[from ^ 1].as<double>();
            a.rot_inv = ctx->rot.as<double2>();
            a.rot_new = ctx->rot.as<double2>() + ctx->gd.nxy;
            a.coef = ctx->coef_k.as<double>();
            a.nf = ctx->ss.n;
        }
        launch_step_plain(a, curved, ctx->stream);
    }
    CU(cudaGetLastError());
    return GRLBM_OK;
}

int build_graph(grlbm_ctx *ctx, int from)
{
    cudaGraph_t g = nullptr;
    CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = GRLBM_OK;
    int b = from;
    for (int s = 0; s < kGraphSteps && rc == GRLBM_OK; s++, b ^= 1)
        rc = enqueue_step(ctx, b);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != GRLBM_OK)
    {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess)
        return fail(ctx, GRLBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->graph[from], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return fail(ctx, GRLBM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    return GRLBM_OK;
}

// departure records from the current Fourier coefficients
int build_records(grlbm_ctx *ctx)
{
    DepartureArgs da{};
    da.g = ctx->gd;
    da.nf = ctx->ss.n;
    da.nd = ctx->st.n;
    da.ng = ctx->ng;
    da.coef = ctx->coef.as<double>();
    da.eval = ctx->eval_basis.as<double>();
    da.alpha = ctx->alpha.as<double>();
    da.rot_c = approx_cos(0.0);
    da.rot_s = approx_sin(0.0);
    if (ctx->fp32 || ctx->fast64)
    {
        // the cell-major records of the band's cells only, addressed by
        // interior cell index through a base shifted by the first cell
        const int64_t c0 = (ctx->gd.jlo - 1) * ctx->gd.nx_, cn = (ctx->gd.jhi - ctx->gd.jlo) * ctx->gd.nx_;
        const size_t rs = ctx->fp32 ? sizeof(float4) : sizeof(double4);
        void *old_rec = ctx->rec.p;
        int rc = alloc(ctx, ctx->rec, (size_t)cn * ctx->st.n * rs);
        if (!rc)
            rc = alloc(ctx, ctx->side, (size_t)cn * ctx->st.n * rs);
        if (rc)
            return rc;
        if (ctx->rec.p != old_rec || ctx->rec_c0 != c0)
            invalidate_graphs(ctx); // captured steps hold the old records' base
        ctx->rec_c0 = c0;
    }
    da.rec64 = ctx->fp32 || ctx->fast64 ? nullptr : ctx->rec.as<double4>();
    da.rec32 = ctx->fp32 ? ctx->rec.as<uint4>() - ctx->rec_c0 * ctx->st.n : nullptr;
    da.side32 = ctx->fp32 ? ctx->side.as<float4>() - ctx->rec_c0 * ctx->st.n : nullptr;
    da.recf = ctx->fast64 ? ctx->rec.as<double4>() - ctx->rec_c0 * ctx->st.n : nullptr;
    da.sidef = ctx->fast64 ? ctx->side.as<double4>() - ctx->rec_c0 * ctx->st.n : nullptr;
    da.q = ctx->dirs.q;
    da.p = ctx->dirs.p;
    for (int r = 0; r < ctx->dirs.q && r < kMaxRowTypes; r++)
        da.row_base[r] = (int)ctx->dirs.rowtab[r * 12 + 10];
    da.c0 = (ctx->gd.jlo - 1) * ctx->gd.nx_;
    da.cn = (ctx->gd.jhi - ctx->gd.jlo) * ctx->gd.nx_;
    da.clamped = reinterpret_cast<int *>(ctx->counters.as<unsigned long long>() + 4);
    da.row_extent = reinterpret_cast<int *>(ctx->counters.as<unsigned long long>() + 5);
    da.far = ctx->counters.as<unsigned long long>() + 6;
    CU(cudaMemsetAsync(ctx->counters.as<unsigned long long>() + 4, 0, 3 * sizeof(unsigned long long), ctx->stream));
    launch_departure(da, ctx->stream);
    if (is_adaptive(ctx))
    {
        // adaptive streaming evaluates the series at run time: a copy with
        // the coefficients of neighbouring nodes side by side (FP32, X and Y
        // about the node, for the precision form)
        if (ctx->fp32)
        {
            int rc = alloc(ctx, ctx->coef32, ctx->coef.bytes / 2);
            if (rc)
                return rc;
            launch_coef_about_node32(ctx->gd, ctx->coef.as<double>(), ctx->coef32.as<float>(), ctx->ss.n,
                                     ctx->stream);
        }
        else
        {
            int rc = alloc(ctx, ctx->coef_k, ctx->coef.bytes);
            if (rc)
                return rc;
            launch_coef_k_major(ctx->coef.as<double>(), ctx->coef_k.as<double>(), ctx->gd.nxy, ctx->ss.n,
                                ctx->stream);
        }
    }
    CU(cudaGetLastError());
    return GRLBM_OK;
}

std::vector<double> identity_coefficients(const grlbm_ctx *ctx)
{
    const int nf = ctx->ss.n;
    const int64_t nxy = ctx->geo.nxy;
    std::vector<double> coef((size_t)5 * nxy * nf, 0.0);
    std::vector<double> B((size_t)nf * nf);
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < nf; k++)
            B[f * nf + k] = fourier_basis(k, ctx->ss.phi[f]);
    std::vector<double> data(5 * (size_t)nf);
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        const double x = ctx->geo.x((double)(ij % ctx->geo.nx)), y = ctx->geo.y((double)(ij / ctx->geo.nx));
        for (int f = 0; f < nf; f++)
        {
            data[f] = 1.0;
            data[nf + f] = x;
            data[2 * nf + f] = y;
            // the reference fills these from the intensity stencil
            data[3 * nf + f] = f < ctx->st.n ? ctx->st.cx[f] : 0.0;
            data[4 * nf + f] = f < ctx->st.n ? ctx->st.cy[f] : 0.0;
        }
        for (int field = 0; field < 5; field++)
        {
            double *out = &coef[(size_t)field * nxy * nf + ij * nf];
            for (int f = 0; f < nf; f++)
            {
                const double c = data[field * nf + f] * ctx->ss.w[f];
                for (int k = 0; k < nf; k++)
                    out[k] += c * B[f * nf + k];
            }
        }
    }
    return coef;
}
} // namespace


// =========================================================================
extern "C" {

const char *grlbm_last_error(const grlbm_ctx *ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int grlbm_selftest_staging_wait(int32_t device, int32_t arrive, int32_t limit_us, int32_t *completed,
                                double *waited_us)
{
    if (!completed || !waited_us || limit_us < 1 || limit_us > 1000000)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "need outputs and a limit in [1, 1000000] us");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, GRLBM_ERR_CUDA, "no CUDA device available");
    if (device >= ndev)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "device %d does not exist", device);
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess)
        return fail(nullptr, GRLBM_ERR_CUDA, "cudaSetDevice failed");
    int done = -1;
    unsigned long long ns = 0;
    const cudaError_t e = run_wait_selftest(arrive != 0, (unsigned long long)limit_us * 1000ull, &done, &ns);
    if (e != cudaSuccess)
        return fail(nullptr, GRLBM_ERR_CUDA, "staging-wait self-test: %s", cudaGetErrorString(e));
    *completed = done;
    *waited_us = (double)ns / 1e3;
    return GRLBM_OK;
}

int32_t grlbm_metric_array_count(void) { return kMetricArrays; }

int grlbm_create(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric, const grlbm_run_desc *run,
                 int32_t device, grlbm_ctx **out)
{
    if (!grid || !metric || !run || !out)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    if (grid->nx_ < 2 || grid->ny_ < 2)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "Grid must have at least 2 LP in each Dimension.");
    if (grid->endx < grid->startx || grid->endy < grid->starty)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "Grid x/y range has end < start");
    if (!(grid->cfl > 0))
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "cfl must be positive");
    if (metric->kind < GRLBM_MINKOWSKI || metric->kind > GRLBM_KERRSCHILD)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "unknown metric kind %d", metric->kind);
    if (run->streaming_type < GRLBM_FLAT_FIXED || run->streaming_type > GRLBM_GEODESIC_FIXED)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "Invalid StreamingType");
    if (run->streaming_type == GRLBM_GEODESIC_FIXED)
        return fail(nullptr, GRLBM_ERR_UNSUPPORTED,
                    "GeodesicFixed (a performance test of the reference) is not built");
    if (run->precision != GRLBM_PLAIN_FP64 && run->precision != GRLBM_PRECISION_FP32 &&
        run->precision != GRLBM_FAST_FP64)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "unknown precision %d", run->precision);
    const int maxdir = kMaxDirs;
    if (run->n_dir < 4 || run->n_dir > maxdir)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "n_dir must be in [4, %d]", maxdir);
    const bool adaptive_type =
        run->streaming_type == GRLBM_FLAT_ADAPTIVE || run->streaming_type == GRLBM_CURVED_ADAPTIVE;
    if (run->precision == GRLBM_PRECISION_FP32 &&
        (adaptive_type ? (double)StateLayout::padded32(grid->nx_ + 2, grid->ny_ + 2).plane * (double)run->n_dir
                       : (double)(grid->nx_ + 2) * (double)(grid->ny_ + 2) *
                             (double)StateLayout::direction_pitch(run->n_dir)) >= 2147483648.0)
        return fail(nullptr, GRLBM_ERR_ARGUMENT,
                    "the precision form indexes its state with 32 bits: it must hold fewer than 2^31 values");
    if (run->precision == GRLBM_FAST_FP64)
    {
        if (adaptive_type)
            return fail(nullptr, GRLBM_ERR_UNSUPPORTED, "the fast FP64 form steps the fixed streaming types only");
        if ((double)(grid->nx_ + 2) * (double)(grid->ny_ + 2) * (double)StateLayout::direction_pitch64(run->n_dir) >=
            2147483648.0)
            return fail(nullptr, GRLBM_ERR_ARGUMENT,
                        "the fast FP64 form indexes its nodes with 32 bits: its state must hold fewer than 2^31 values");
    }
    if (run->n_fourier < 1 || run->n_fourier > kMaxFourier)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "n_fourier must be in [1, %d]", kMaxFourier);
    if (run->initial_data_type != GRLBM_MOMENTS && run->initial_data_type != GRLBM_INTENSITIES)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "unknown initial data type");

    std::unique_ptr<grlbm_ctx> owner(new (std::nothrow) grlbm_ctx);
    if (!owner)
        return fail(nullptr, GRLBM_ERR_HOST, "out of host memory");
    grlbm_ctx *ctx = owner.get();
    ctx->run = *run;
    ctx->mdesc = *metric;
    ctx->fp32 = run->precision == GRLBM_PRECISION_FP32;
    ctx->fast64 = run->precision == GRLBM_FAST_FP64;
    if (const char *w = std::getenv("GRLBM_WIDE_OFFSETS"))
        ctx->wide_offsets = w[0] == '1';
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, GRLBM_ERR_CUDA, "no CUDA device available");
    if (device >= 0)
    {
        if (device >= ndev)
            return fail(nullptr, GRLBM_ERR_ARGUMENT, "device %d does not exist", device);
        if (cudaSetDevice(device) != cudaSuccess)
            return fail(nullptr, GRLBM_ERR_CUDA, "cudaSetDevice failed");
    }
    cudaGetDevice(&ctx->device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(nullptr, GRLBM_ERR_CUDA, "cudaStreamCreate failed");

    try
    {
        ctx->geo = GridGeom::from(*grid);
        ctx->st = StencilTables::build(run->n_dir, true);
        ctx->ss = StencilTables::build(run->n_fourier, false);
        ctx->M = MetricArrays::build(ctx->geo, *metric);
    }
    catch (const std::exception &e)
    {
        return fail(nullptr, GRLBM_ERR_HOST, "host set-up failed: %s", e.what());
    }
    const GridGeom &G = ctx->geo;
    const int64_t nxy = G.nxy;
    const int nd = run->n_dir, nf = run->n_fourier;
    ctx->ncell = grid->nx_ * grid->ny_;
    ctx->ng = ctx->st.ng;
    GridDev &gd = ctx->gd;
    gd.nx = G.nx;
    gd.ny = G.ny;
    gd.nxy = nxy;
    gd.nx_ = grid->nx_;
    gd.ny_ = grid->ny_;
    gd.ncell = ctx->ncell;
    gd.jlo = 1;
    gd.jhi = G.ny - 1;
    gd.dx = G.dx;
    gd.dy = G.dy;
    gd.dt = G.dt;
    gd.startx = G.startx;
    gd.starty = G.starty;
    gd.endx = G.endx;
    gd.endy = G.endy;
    gd.kind = metric->kind;
    gd.excision2 = ctx->M.excision2;

    int rc;
#define TRY(x)                           \
    do                                   \
    {                                    \
        if ((rc = (x)) != GRLBM_OK)      \
        {                                \
            g_create_error = ctx->err;   \
            return rc;                   \
        }                                \
    } while (0)

    // directions rotated by RotationMatrix(0) (src/DataTypes.hh:630-635)
    const double rc0 = approx_cos(0.0), rs0 = approx_sin(0.0);
    std::vector<double> n1(nd), n2(nd);
    for (int d = 0; d < nd; d++)
    {
        n1[d] = ctx->st.cx[d] * rc0 - ctx->st.cy[d] * rs0;
        n2[d] = ctx->st.cx[d] * rs0 + ctx->st.cy[d] * rc0;
    }
    {
        std::vector<double> d64(ctx->st.w.begin(), ctx->st.w.end());
        d64.insert(d64.end(), n1.begin(), n1.end());
        d64.insert(d64.end(), n2.begin(), n2.end());
        TRY(upload(ctx, ctx->dirs64, d64));
    }
    TRY(upload_t(ctx, ctx->w, ctx->st.w));
    TRY(upload_t(ctx, ctx->n1, n1));
    TRY(upload_t(ctx, ctx->n2, n2));
    TRY(upload(ctx, ctx->cx, ctx->st.cx));
    TRY(upload(ctx, ctx->cy, ctx->st.cy));
    // the fast FP64 form's tables, built beside the FP32 ones
    std::unique_ptr<DirTable64> t64(ctx->fast64 ? new DirTable64{} : nullptr);
    if (ctx->fp32 || ctx->fast64)
    {
        // each cubic row g of the reference's interpolation grid blended with
        // row g+1 into one 5-direction window starting at row g's first
        // direction: weights W0 + t D.  The rows repeat with period q (shifted
        // by p directions per period); the kernel keeps the q row types and
        // every row is checked against its type here.
        const int ng = ctx->ng;
        std::vector<int> base(ng);
        for (int g = 0; g < ng; g++)
        {
            base[g] = (int)ctx->st.ig_index[4 * g];
            for (int k = 1; k < 4; k++)
                if (ctx->st.ig_index[4 * g + k] != (base[g] + k) % nd)
                    return fail(nullptr, GRLBM_ERR_HOST, "interpolation row %d is not 4 consecutive directions", g);
        }
        int gcd = nd, b = ng;
        while (b)
        {
            const int r = gcd % b;
            gcd = b;
            b = r;
        }
        const int q = ng / gcd, pstep = nd / gcd;
        if (q > kMaxRowTypes)
            return fail(nullptr, GRLBM_ERR_UNSUPPORTED, "interpolation grid period %d exceeds %d row types", q,
                        kMaxRowTypes);
        DirTable &dt = ctx->dirs;
        std::vector<double> eff_row(2 * nd), eff_type(2 * nd);
        for (int g = 0; g < ng; g++)
        {
            const int g1 = (g + 1) % ng;
            const int shift = ((base[g1] - base[g]) % nd + nd) % nd;
            if (shift > 1)
                return fail(nullptr, GRLBM_ERR_HOST, "interpolation rows %d, %d are %d directions apart", g, g1, shift);
            double W0[5] = {0, 0, 0, 0, 0}, W1[5] = {0, 0, 0, 0, 0};
            for (int k = 0; k < 4; k++)
            {
                W0[k] = ctx->st.ig_weight[4 * g + k];
                W1[k + shift] = ctx->st.ig_weight[4 * g1 + k];
            }
            double rowd[12];
            for (int k = 0; k < 4; k++)
            {
                rowd[k] = W0[k];
                rowd[4 + k] = W1[k] - W0[k];
            }
            rowd[8] = W0[4];
            rowd[9] = W1[4] - W0[4];
            rowd[10] = (double)base[g];
            rowd[11] = 0.0;
            float row[12];
            for (int k = 0; k < 12; k++)
                row[k] = (float)rowd[k];
            const int r = g % q, m = g / q;
            float *t = &dt.rowtab[r * 12];
            if (m == 0)
            {
                std::memcpy(t, row, sizeof row);
                if (t64)
                    std::memcpy(&t64->rowtab[r * 12], rowd, sizeof rowd);
            }
            else
            {
                // The row must act on the same directions with the same
                // weights as its type shifted by p m directions.  (A row that
                // sits exactly on a direction may list its 4 neighbours one
                // place earlier or later, with that direction's weight 1 and
                // the others 0: the same interpolation.)
                std::fill(eff_row.begin(), eff_row.end(), 0.0);
                std::fill(eff_type.begin(), eff_type.end(), 0.0);
                const int tb = ((int)t[10] + pstep * m) % nd;
                for (int k = 0; k < 5; k++)
                {
                    const float rw0 = k < 4 ? row[k] : row[8], rdd = k < 4 ? row[4 + k] : row[9];
                    const float tw0 = k < 4 ? t[k] : t[8], tdd = k < 4 ? t[4 + k] : t[9];
                    eff_row[(base[g] + k) % nd] += rw0;
                    eff_row[nd + (base[g] + k) % nd] += rdd;
                    eff_type[(tb + k) % nd] += tw0;
                    eff_type[nd + (tb + k) % nd] += tdd;
                }
                for (int k = 0; k < 2 * nd; k++)
                    if (std::fabs(eff_row[k] - eff_type[k]) > 1e-6)
                        return fail(nullptr, GRLBM_ERR_HOST, "interpolation row %d does not repeat row %d", g, r);
                if (t64)
                {
                    // the same in FP64: the rows of a type may differ in the
                    // reference's rounding only
                    std::fill(eff_row.begin(), eff_row.end(), 0.0);
                    std::fill(eff_type.begin(), eff_type.end(), 0.0);
                    const double *td = &t64->rowtab[r * 12];
                    for (int k = 0; k < 5; k++)
                    {
                        eff_row[(base[g] + k) % nd] += k < 4 ? rowd[k] : rowd[8];
                        eff_row[nd + (base[g] + k) % nd] += k < 4 ? rowd[4 + k] : rowd[9];
                        eff_type[(tb + k) % nd] += k < 4 ? td[k] : td[8];
                        eff_type[nd + (tb + k) % nd] += k < 4 ? td[4 + k] : td[9];
                    }
                    for (int k = 0; k < 2 * nd; k++)
                        if (std::fabs(eff_row[k] - eff_type[k]) > 1e-12)
                            return fail(nullptr, GRLBM_ERR_HOST,
                                        "interpolation row %d repeats row %d only to %.3g in FP64", g, r,
                                        std::fabs(eff_row[k] - eff_type[k]));
                }
            }
        }
        dt.q = q;
        dt.p = pstep;
        dt.inv_q = 1.0f / (float)q;
        // direction tables: weights, rotated directions, flat departures, and
        // the stencil sums of the affine collide map
        double wm[18] = {0};
        for (int d = 0; d < nd; d++)
        {
            dt.w[d] = (float)ctx->st.w[d];
            dt.n1[d] = (float)n1[d];
            dt.n2[d] = (float)n2[d];
            const double wd = ctx->st.w[d];
            const double cf[8] = {wd, wd * n1[d], wd * n2[d], wd * n1[d] * n1[d], wd * n1[d] * n2[d],
                                  wd * n2[d] * n2[d], n1[d], n2[d]};
            for (int k = 0; k < 8; k++)
                dt.dirc[8 * d + k] = (float)cf[k];
            dt.ox[d] = (float)(-ctx->st.cx[d] * G.dt / G.dx);
            dt.oy[d] = (float)(-ctx->st.cy[d] * G.dt / G.dy);
            const double mu[6] = {1.0, n1[d], n2[d], n1[d] * n1[d], n1[d] * n2[d], n2[d] * n2[d]};
            for (int q = 0; q < 6; q++)
            {
                wm[q] += ctx->st.w[d] * mu[q];
                wm[6 + q] += ctx->st.w[d] * mu[q] * n1[d];
                wm[12 + q] += ctx->st.w[d] * mu[q] * n2[d];
            }
        }
        for (int q = 0; q < 18; q++)
            dt.wmom[q] = (float)wm[q];
        if (t64)
        {
            t64->q = q;
            t64->p = pstep;
            t64->inv_q = 1.0 / (double)q;
            for (int d = 0; d < nd; d++)
            {
                const double wd = ctx->st.w[d];
                const double cf[8] = {wd, wd * n1[d], wd * n2[d], wd * n1[d] * n1[d], wd * n1[d] * n2[d],
                                      wd * n2[d] * n2[d], n1[d], n2[d]};
                for (int k = 0; k < 8; k++)
                    t64->dirc[8 * d + k] = cf[k];
                // the products c dt of the reference's flat departure (src/Radiation.cpp:398-399)
                t64->cxdt[d] = ctx->st.cx[d] * G.dt;
                t64->cydt[d] = ctx->st.cy[d] * G.dt;
            }
            for (int q = 0; q < 18; q++)
                t64->wmom[q] = wm[q];
            std::vector<DirTable64> one(1, *t64);
            TRY(upload(ctx, ctx->dirs64t, one));
        }
    }
    // the interpolation grid's rows: the plain form's stream, and adaptive
    // streaming in either form
    if (!ctx->fp32)
    {
        std::vector<IgRow> rows(ctx->ng);
        for (int g = 0; g < ctx->ng; g++)
        {
            const int64_t *x = &ctx->st.ig_index[4 * g];
            const double *w = &ctx->st.ig_weight[4 * g];
            rows[g].idx = make_int4((int)x[0], (int)x[1], (int)x[2], (int)x[3]);
            rows[g].w01 = make_double2(w[0], w[1]);
            rows[g].w23 = make_double2(w[2], w[3]);
        }
        TRY(upload(ctx, ctx->ig_rows, rows));
    }
    else if (is_adaptive(ctx))
    {
        std::vector<IgRow32> rows(ctx->ng);
        for (int g = 0; g < ctx->ng; g++)
        {
            const int64_t *x = &ctx->st.ig_index[4 * g];
            const double *w = &ctx->st.ig_weight[4 * g];
            rows[g].idx = make_int4((int)x[0], (int)x[1], (int)x[2], (int)x[3]);
            rows[g].w = make_float4((float)w[0], (float)w[1], (float)w[2], (float)w[3]);
        }
        TRY(upload(ctx, ctx->ig_rows, rows));
    }

    // per-node metric data
    const MetricArrays &M = ctx->M;
    std::vector<double> rkf((size_t)nxy * kRkStride, 0.0), lfp((size_t)nxy * 12), ia3(nxy), alpha(nxy);
    std::vector<uint8_t> flags(nxy), bh(nxy);
    static const int rkmap[RF_COUNT] = {ALPHA, BETA1U, BETA2U, D1ALPHA, D2ALPHA, D1BETA1LU, D1BETA2LU,
                                        D2BETA1LU, D2BETA2LU, K11L, K12L, K22L, GAM11U, GAM12U, GAM22U,
                                        D1GAM11LLL, D1GAM12LLL, D1GAM22LLL, D2GAM11LLL, D2GAM12LLL, D2GAM22LLL,
                                        -1, TET11, TET12, TET21, TET22, ITET11, ITET12, ITET21, ITET22};
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        for (int f = 0; f < RF_COUNT; f++)
            rkf[ij * kRkStride + f] = rkmap[f] < 0 ? 0.0 : M.at(rkmap[f], ij);
        for (int q = 0; q < 9; q++)
            lfp[ij * 12 + q] = M.at(TET00 + q, ij);
        lfp[ij * 12 + 9] = M.at(GAM11L, ij);
        lfp[ij * 12 + 10] = M.at(GAM12L, ij);
        lfp[ij * 12 + 11] = M.at(GAM22L, ij);
        const double a = M.at(ALPHA, ij);
        alpha[ij] = a;
        // A node exactly on the singularity has alpha = 0; it lies inside the
        // excision, keeps its intensity, and stores it unscaled.
        const double s = 1.0 / (a * a * a);
        ia3[ij] = (std::isfinite(s) && std::isfinite((float)s) && (float)s > 0.f) ? s : 1.0;
        const bool inside = M.inside_bh(G.x((double)(ij % G.nx)), G.y((double)(ij / G.nx)));
        bh[ij] = inside;
        flags[ij] = inside ? 3 : 0;
    }
    TRY(upload(ctx, ctx->rkf, rkf));
    TRY(upload(ctx, ctx->lfp, lfp));
    TRY(upload(ctx, ctx->alpha, alpha));
    TRY(upload(ctx, ctx->flags, flags));
    TRY(upload(ctx, ctx->bhmask, bh));
    if (ctx->fp32 || ctx->fast64)
        TRY(upload_t(ctx, ctx->ia3, ia3));
    else
    {
        TRY(alloc(ctx, ctx->acube, (size_t)nxy * 9 * sizeof(double)));
        cudaMemset(ctx->acube.p, 0, ctx->acube.bytes);
        launch_alpha_cube(gd, ctx->alpha.as<double>(), ctx->acube.as<double>(), ctx->stream);
    }

    // streaming stencil and the two Fourier bases
    std::vector<double> pb((size_t)nf * nf), eb((size_t)nf * nd);
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < nf; k++)
            pb[f * nf + k] = fourier_basis(k, ctx->ss.phi[f]);
    for (int k = 0; k < nf; k++)
        for (int d = 0; d < nd; d++)
            eb[k * nd + d] = fourier_basis(k, ctx->st.phi[d]);
    TRY(upload(ctx, ctx->ss_cx, ctx->ss.cx));
    TRY(upload(ctx, ctx->ss_cy, ctx->ss.cy));
    TRY(upload(ctx, ctx->ss_w, ctx->ss.w));
    TRY(upload(ctx, ctx->proj_basis, pb));
    TRY(upload(ctx, ctx->eval_basis, eb));
    TRY(upload(ctx, ctx->coef, identity_coefficients(ctx)));

    // state
    ctx->sl = ctx->fast64 ? StateLayout::cell_major64(G.nx, nd)
              : !ctx->fp32 ? StateLayout::dense(G.nx, G.ny)
                           : (is_adaptive(ctx) ? StateLayout::padded32(G.nx, G.ny) : StateLayout::cell_major32(G.nx, nd));
    const size_t ib = (size_t)ctx->sl.elements(G.ny, nd) * tsize(ctx);
    if (ctx->fp32 || ctx->fast64)
    {
        if (cudaHostAlloc(reinterpret_cast<void **>(&ctx->fault), sizeof(unsigned),
                          cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
            return fail(nullptr, GRLBM_ERR_CUDA, "cudaHostAlloc of the fault word failed");
        *ctx->fault = 0;
    }
    TRY(alloc(ctx, ctx->I[0], ib));
    TRY(alloc(ctx, ctx->I[1], ib));
    if ((!ctx->fp32 && !ctx->fast64) || is_adaptive(ctx))
        TRY(alloc(ctx, ctx->streamed, (size_t)nxy * nd * tsize(ctx)));
    TRY(alloc(ctx, ctx->mom, (size_t)6 * nxy * tsize(ctx)));
    // (the tiled forms allocate their records with the first table build, for the band's cells)
    if (!ctx->fp32 && !ctx->fast64)
        TRY(alloc(ctx, ctx->rec, (size_t)ctx->ncell * nd * sizeof(double4)));
    TRY(alloc(ctx, ctx->counters, 8 * sizeof(unsigned long long)));
    TRY(alloc(ctx, ctx->tile_ctr, 2 * sizeof(unsigned)));
    cudaMemset(ctx->tile_ctr.p, 0, ctx->tile_ctr.bytes);
    TRY(alloc(ctx, ctx->energy_partial, kPartialBlocks * sizeof(double)));
    TRY(alloc(ctx, ctx->energy_out, sizeof(double)));
    cudaMemset(ctx->I[0].p, 0, ib);
    cudaMemset(ctx->I[1].p, 0, ib);
    if (is_tiled(ctx))
    {
        ctx->passes = ctx->fast64 ? step64_passes(nd) : step32_passes(nd);
        if (ctx->passes < 1)
            return fail(nullptr, GRLBM_ERR_ARGUMENT, "n_dir %d exceeds the tiled step's passes", nd);
        if ((ctx->fast64 ? prepare_step64() : prepare_step32()) != cudaSuccess)
            return fail(nullptr, GRLBM_ERR_CUDA, "cannot reserve shared memory for the tiled step");
        TRY(default_step32_tile(ctx));
    }
    if (is_adaptive(ctx))
    {
        // rotationAngle and rotationAngleNew start at zero (src/Radiation.cpp:3-60)
        for (auto &b : ctx->ang)
        {
            TRY(alloc(ctx, b, (size_t)nxy * sizeof(double)));
            cudaMemset(b.p, 0, b.bytes);
        }
        TRY(alloc(ctx, ctx->rot, 2 * (size_t)nxy * (ctx->fp32 ? sizeof(float2) : sizeof(double2))));
        if (ctx->fp32)
        {
            std::vector<float> cx32(ctx->st.cx.begin(), ctx->st.cx.end()), cy32(ctx->st.cy.begin(), ctx->st.cy.end());
            TRY(upload(ctx, ctx->cx32, cx32));
            TRY(upload(ctx, ctx->cy32, cy32));
        }
        ctx->flux_angle.assign(nxy, 0.0);
    }
    cudaMemset(ctx->mom.p, 0, ctx->mom.bytes);
    cudaMemset(ctx->counters.p, 0, ctx->counters.bytes);
    if (ctx->rec.p)
        cudaMemset(ctx->rec.p, 0, ctx->rec.bytes);
    // fields default to zero (the reference's buffers are value-initialised)
    std::vector<double> zeros(nxy, 0.0);
    TRY(grlbm_set_fields(ctx, zeros.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data()));
    if (!ctx->fp32 && prepare_step_plain(0) != cudaSuccess)
        return fail(nullptr, GRLBM_ERR_CUDA, "cannot reserve shared memory for the step kernel");
    if (cudaDeviceSynchronize() != cudaSuccess)
        return fail(nullptr, GRLBM_ERR_CUDA, "device error during set-up");
#undef TRY
    *out = owner.release();
    return GRLBM_OK;
}

void grlbm_destroy(grlbm_ctx *ctx)
{
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

int grlbm_get_grid(const grlbm_ctx *ctx, int64_t *nx, int64_t *ny, double *dx, double *dy, double *dt)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (nx)
        *nx = ctx->geo.nx;
    if (ny)
        *ny = ctx->geo.ny;
    if (dx)
        *dx = ctx->geo.dx;
    if (dy)
        *dy = ctx->geo.dy;
    if (dt)
        *dt = ctx->geo.dt;
    return GRLBM_OK;
}

void *grlbm_stream(grlbm_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int grlbm_set_fields(grlbm_ctx *ctx, const double *kappa0, const double *kappa1, const double *kappaA,
                     const double *eta, const double *ux, const double *uy)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!kappa0 || !kappa1 || !kappaA || !eta || !ux || !uy)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null field");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->geo.nxy;
    const MetricArrays &M = ctx->M;
    std::vector<double> u1(nxy), u2(nxy), lor(nxy), adt(nxy), k3(nxy);
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        // TransformLFtoIF(uLF, GetTetrad(ij)) as Collide calls it (src/Radiation.cpp:652-657)
        const double a = M.at(TET11, ij) * ux[ij] + M.at(TET12, ij) * uy[ij];
        const double b = M.at(TET21, ij) * ux[ij] + M.at(TET22, ij) * uy[ij];
        u1[ij] = a;
        u2[ij] = b;
        lor[ij] = 1.0 / std::sqrt(1.0 - (a * a + b * b));
        adt[ij] = M.at(ALPHA, ij) * ctx->geo.dt;
        k3[ij] = 3.0 * kappa1[ij];
    }
    int rc;
    if ((rc = upload_t(ctx, ctx->cu1, u1)) || (rc = upload_t(ctx, ctx->cu2, u2)) ||
        (rc = upload_t(ctx, ctx->clor, lor)) || (rc = upload_t(ctx, ctx->cadt, adt)) ||
        (rc = upload_t(ctx, ctx->ck3, k3)))
        return rc;
    const double *src[3] = {eta, kappa0, kappaA};
    DevBuf *dst[3] = {&ctx->ceta, &ctx->ck0, &ctx->cka};
    for (int q = 0; q < 3; q++)
        if ((rc = upload_t(ctx, *dst[q], std::vector<double>(src[q], src[q] + nxy))))
            return rc;
    invalidate_graphs(ctx);
    return GRLBM_OK;
}

int grlbm_set_initial_data(grlbm_ctx *ctx, const uint8_t *is_initial, const double *initial_I, const double *E_LF,
                           const double *Fx_LF, const double *Fy_LF, const double *Pxx_LF, const double *Pxy_LF,
                           const double *Pyy_LF)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!is_initial)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null is_initial");
    if (ctx->run.initial_data_type == GRLBM_INTENSITIES && !initial_I)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "initial_I is required for InitialDataType::Intensities");
    if (ctx->run.initial_data_type == GRLBM_MOMENTS && (!E_LF || !Fx_LF || !Fy_LF || !Pxx_LF || !Pxy_LF || !Pyy_LF))
        return fail(ctx, GRLBM_ERR_ARGUMENT, "initial moments are required for InitialDataType::Moments");
    cudaSetDevice(ctx->device);
    Sources S;
    try
    {
        S = build_sources(ctx->M, ctx->st, ctx->run.initial_data_type, is_initial, initial_I, E_LF, Fx_LF, Fy_LF,
                          Pxx_LF, Pxy_LF, Pyy_LF, is_adaptive(ctx),
                          ctx->flux_angle.empty() ? nullptr : ctx->flux_angle.data());
    }
    catch (const std::exception &e)
    {
        return fail(ctx, GRLBM_ERR_HOST, "source set-up failed: %s", e.what());
    }
    ctx->nsrc = (int64_t)S.nodes.size();
    if (ctx->fast64 && is_curved(ctx))
    {
        // the fast FP64 form stores I / alpha^3
        const int nd = ctx->st.n;
        for (size_t s_ = 0; s_ < S.nodes.size(); s_++)
        {
            const double a = ctx->M.at(ALPHA, S.nodes[s_]);
            const double s3 = 1.0 / (a * a * a);
            const double scale = (std::isfinite(s3) && s3 > 0.0) ? s3 : 1.0;
            for (int d = 0; d < nd; d++)
                S.intensities[s_ * nd + d] *= scale;
        }
    }
    if (ctx->fp32 && is_curved(ctx))
    {
        // the precision form stores I / alpha^3
        const int nd = ctx->st.n;
        for (size_t s_ = 0; s_ < S.nodes.size(); s_++)
        {
            const double a = ctx->M.at(ALPHA, S.nodes[s_]);
            const float scale = (float)(1.0 / (a * a * a));
            for (int d = 0; d < nd; d++)
                S.intensities[s_ * nd + d] = (double)((float)S.intensities[s_ * nd + d] * scale);
        }
    }
    int rc;
    if ((rc = upload(ctx, ctx->src_nodes, S.nodes)) || (rc = upload_t(ctx, ctx->src_vals, S.intensities)))
        return rc;
    if (is_adaptive(ctx))
    {
        ctx->nsrc_ang = (int64_t)S.angle_nodes.size();
        if ((rc = upload(ctx, ctx->src_ang_nodes, S.angle_nodes)) || (rc = upload(ctx, ctx->src_ang_vals, S.angles)))
            return rc;
    }
    invalidate_graphs(ctx);
    return GRLBM_OK;
}

int grlbm_load_initial_data(grlbm_ctx *ctx)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (ctx->nsrc == 0)
        return GRLBM_OK;
    // both buffers: halo and excised nodes are read from whichever is current
    for (int b = 0; b < 2; b++)
    {
        if (ctx->fast64)
            launch_sources64L(ctx->I[b].as<double>(), ctx->sl, ctx->st.n, ctx->src_nodes.as<int64_t>(),
                              ctx->src_vals.as<double>(), ctx->nsrc, ctx->stream);
        else if (ctx->fp32)
            launch_sources32(ctx->I[b].as<float>(), ctx->sl, ctx->st.n, ctx->src_nodes.as<int64_t>(),
                             ctx->src_vals.as<float>(), ctx->nsrc, ctx->stream);
        else
            launch_sources64(ctx->I[b].as<double>(), ctx->gd.nxy, ctx->st.n, ctx->src_nodes.as<int64_t>(),
                             ctx->src_vals.as<double>(), ctx->nsrc, ctx->stream);
    }
    // and the source nodes' rotation angles, into the current angles only
    if (is_adaptive(ctx) && ctx->nsrc_ang > 0)
        launch_sources64(ctx->ang[ctx->cur].as<double>(), ctx->gd.nxy, 1, ctx->src_ang_nodes.as<int64_t>(),
                         ctx->src_ang_vals.as<double>(), ctx->nsrc_ang, ctx->stream);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_set_initial_flux_angle(grlbm_ctx *ctx, const double *angle)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!angle)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null angles");
    if (!is_adaptive(ctx))
        return fail(ctx, GRLBM_ERR_STATE, "initialFluxAngle_IF is read by the adaptive streaming types only");
    ctx->flux_angle.assign(angle, angle + ctx->gd.nxy);
    return GRLBM_OK;
}

int grlbm_set_intensity(grlbm_ctx *ctx, const double *I)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!I)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null intensities");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    const int nd = ctx->st.n;
    int rc = alloc(ctx, ctx->stage, (size_t)nxy * nd * sizeof(double));
    if (rc)
        return rc;
    CU(cudaMemcpyAsync(ctx->stage.p, I, ctx->stage.bytes, cudaMemcpyHostToDevice, ctx->stream));
    for (int b = 0; b < 2; b++)
    {
        if (ctx->fast64)
            launch_to_state64(ctx->stage.as<double>(), ctx->I[b].as<double>(), nxy, ctx->sl, nd, state_scale64(ctx),
                              ctx->stream);
        else if (ctx->fp32)
            launch_to_dirmajor32(ctx->stage.as<double>(), ctx->I[b].as<float>(), nxy, ctx->sl, nd,
                                 state_scale(ctx), ctx->stream);
        else
            launch_to_dirmajor64(ctx->stage.as<double>(), ctx->I[b].as<double>(), nxy, nd, ctx->stream);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_get_intensity(grlbm_ctx *ctx, double *I)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!I)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null intensities");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    const int nd = ctx->st.n;
    int rc = alloc(ctx, ctx->stage, (size_t)nxy * nd * sizeof(double));
    if (rc)
        return rc;
    if (ctx->fast64)
        launch_from_state64(ctx->I[ctx->cur].as<double>(), ctx->stage.as<double>(), nxy, ctx->sl, nd, state_scale64(ctx),
                            ctx->stream);
    else if (ctx->fp32)
        launch_to_cellmajor32(ctx->I[ctx->cur].as<float>(), ctx->stage.as<double>(), nxy, ctx->sl, nd, state_scale(ctx),
                              ctx->stream);
    else
        launch_to_cellmajor64(ctx->I[ctx->cur].as<double>(), ctx->stage.as<double>(), nxy, nd, ctx->stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(I, ctx->stage.p, ctx->stage.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_update_fourier_coefficients(grlbm_ctx *ctx, double rk_tol, int32_t max_substeps)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    TraceScope trace(ctx, kTablesName);
    if (!(rk_tol > 0))
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rk_tol must be positive");
    cudaSetDevice(ctx->device);
    const int nf = ctx->ss.n;
    // the cells of the band's rows (all interior cells unless grlbm_set_rows narrowed it)
    const int64_t c0 = (ctx->gd.jlo - 1) * ctx->gd.nx_, cn = (ctx->gd.jhi - ctx->gd.jlo) * ctx->gd.nx_;
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    CU(cudaMemsetAsync(cnt + 2, 0, 2 * sizeof(unsigned long long), ctx->stream));
    void *data = nullptr;
    CU(cudaMallocAsync(&data, (size_t)5 * cn * nf * sizeof(double), ctx->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);

    GeodesicArgs ga{};
    ga.g = ctx->gd;
    ga.rkf = ctx->rkf.as<double>();
    ga.ss_cx = ctx->ss_cx.as<double>();
    ga.ss_cy = ctx->ss_cy.as<double>();
    ga.nf = nf;
    ga.tol = rk_tol;
    ga.max_trials = max_substeps > 0 ? max_substeps : 1000000;
    ga.data = static_cast<double *>(data);
    ga.trials_total = cnt + 2;
    ga.nonconverged = reinterpret_cast<int *>(cnt + 3);
    ga.c0 = c0;
    ga.cn = cn;
    launch_geodesic(ga, ctx->stream);

    ProjectArgs pa{};
    pa.g = ctx->gd;
    pa.nf = nf;
    pa.data = ga.data;
    pa.ss_w = ctx->ss_w.as<double>();
    pa.basis = ctx->proj_basis.as<double>();
    pa.coef = ctx->coef.as<double>();
    pa.c0 = c0;
    pa.cn = cn;
    launch_project(pa, ctx->stream);
    int rc = build_records(ctx);
    cudaEventRecord(e1, ctx->stream);
    cudaError_t le = cudaGetLastError();
    cudaFreeAsync(data, ctx->stream);
    cudaError_t se = cudaStreamSynchronize(ctx->stream);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    if (le != cudaSuccess || se != cudaSuccess)
        return fail(ctx, GRLBM_ERR_CUDA, "table build failed: %s", cudaGetErrorString(le != cudaSuccess ? le : se));
    ctx->table_ms = ms;
    ctx->tables = true;
    ctx->table_jlo = ctx->gd.jlo;
    ctx->table_jhi = ctx->gd.jhi;
    unsigned long long h[5];
    CU(cudaMemcpy(h, cnt, sizeof h, cudaMemcpyDeviceToHost));
    const int nonconv = (int)(unsigned)h[3];
    if (nonconv > 0)
        return fail(ctx, GRLBM_ERR_NONCONVERGED, "%d RK45 backtraces hit the substep cap", nonconv);
    return GRLBM_OK;
}

int grlbm_set_fourier_coefficients(grlbm_ctx *ctx, const double *S, const double *X, const double *Y,
                                   const double *Cx, const double *Cy)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!S || !X || !Y || !Cx || !Cy)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null coefficient array");
    cudaSetDevice(ctx->device);
    const size_t per = (size_t)ctx->gd.nxy * ctx->ss.n;
    const double *src[5] = {S, X, Y, Cx, Cy};
    for (int q = 0; q < 5; q++)
        CU(cudaMemcpyAsync(ctx->coef.as<double>() + q * per, src[q], per * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
    int rc = build_records(ctx);
    if (rc)
        return rc;
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->tables = true;
    ctx->table_jlo = ctx->gd.jlo;
    ctx->table_jhi = ctx->gd.jhi;
    return GRLBM_OK;
}

int grlbm_get_fourier_coefficients(grlbm_ctx *ctx, double *S, double *X, double *Y, double *Cx, double *Cy)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    const size_t per = (size_t)ctx->gd.nxy * ctx->ss.n;
    double *dst[5] = {S, X, Y, Cx, Cy};
    for (int q = 0; q < 5; q++)
        if (dst[q])
            CU(cudaMemcpy(dst[q], ctx->coef.as<double>() + q * per, per * sizeof(double), cudaMemcpyDeviceToHost));
    return GRLBM_OK;
}

int grlbm_step_async(grlbm_ctx *ctx, int32_t n_steps)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (n_steps < 0)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "negative step count");
    int rc = check_tables(ctx);
    if (rc)
        return rc;
    if (ctx->partial)
        return fail(ctx, GRLBM_ERR_STATE, "a step enqueued in row ranges is not finished");
    cudaSetDevice(ctx->device);
    if (ctx->update_each_step)
    {
        // UpdateFourierCoefficients at the top of every step (src/Radiation.cpp:790-791)
        for (int k = 0; k < n_steps; k++)
        {
            if ((rc = grlbm_update_fourier_coefficients(ctx, ctx->update_tol, ctx->update_max_substeps)))
                return rc;
            if ((rc = enqueue_step(ctx, ctx->cur)))
                return rc;
            ctx->cur ^= 1;
            ctx->steps++;
        }
        return GRLBM_OK;
    }
    int left = n_steps;
    while (left >= kGraphSteps)
    {
        if (!ctx->graph[ctx->cur] && (rc = build_graph(ctx, ctx->cur)))
            return rc;
        CU(cudaGraphLaunch(ctx->graph[ctx->cur], ctx->stream));
        left -= kGraphSteps; // an even count: the current buffer is unchanged
    }
    for (; left > 0; left--)
    {
        if ((rc = enqueue_step(ctx, ctx->cur)))
            return rc;
        ctx->cur ^= 1;
    }
    ctx->steps += n_steps;
    return GRLBM_OK;
}

int grlbm_step_rows_async(grlbm_ctx *ctx, int64_t j_first, int64_t j_end, int32_t finish)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (j_first < ctx->gd.jlo || j_end > ctx->gd.jhi || j_first > j_end)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rows [%lld, %lld) outside the band [%lld, %lld)", (long long)j_first,
                    (long long)j_end, (long long)ctx->gd.jlo, (long long)ctx->gd.jhi);
    if (ctx->update_each_step)
        return fail(ctx, GRLBM_ERR_UNSUPPORTED, "tables rebuilt every step are not stepped in row ranges");
    if (is_adaptive(ctx))
        return fail(ctx, GRLBM_ERR_UNSUPPORTED, "adaptive streaming is not split into row ranges");
    int rc = check_tables(ctx);
    if (rc)
        return rc;
    cudaSetDevice(ctx->device);
    if (j_end > j_first)
    {
        const int64_t lo = ctx->gd.jlo, hi = ctx->gd.jhi;
        ctx->gd.jlo = j_first;
        ctx->gd.jhi = j_end;
        rc = enqueue_step(ctx, ctx->cur, !ctx->partial);
        ctx->gd.jlo = lo;
        ctx->gd.jhi = hi;
        if (rc)
            return rc;
        ctx->partial = true;
    }
    if (finish)
    {
        ctx->cur ^= 1;
        ctx->steps++;
        ctx->partial = false;
    }
    return GRLBM_OK;
}

int grlbm_sync(grlbm_ctx *ctx)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    CU(cudaStreamSynchronize(ctx->stream));
    return check_fault(ctx);
}

int grlbm_step(grlbm_ctx *ctx, int32_t n_steps)
{
    TraceScope trace(ctx, kStepName);
    int rc = grlbm_step_async(ctx, n_steps);
    if (rc)
        return rc;
    return grlbm_sync(ctx);
}

int grlbm_get_moments_if(grlbm_ctx *ctx, double *E, double *Fx, double *Fy, double *Pxx, double *Pxy, double *Pyy)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    double *dst[6] = {E, Fx, Fy, Pxx, Pxy, Pyy};
    const double *from = ctx->mom.as<double>();
    if (ctx->fp32)
    {
        int rc = alloc(ctx, ctx->lf_out, (size_t)7 * nxy * sizeof(double));
        if (rc)
            return rc;
        launch_widen32(ctx->mom.as<float>(), ctx->lf_out.as<double>(), 6 * nxy, ctx->stream);
        CU(cudaGetLastError());
        from = ctx->lf_out.as<double>();
    }
    for (int q = 0; q < 6; q++)
        if (dst[q])
            CU(cudaMemcpyAsync(dst[q], from + q * nxy, nxy * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_compute_moments_lf(grlbm_ctx *ctx, double *E, double *Fx, double *Fy, double *Pxx, double *Pxy,
                             double *Pyy, double *F)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    int rc = alloc(ctx, ctx->lf_out, (size_t)7 * nxy * sizeof(double));
    if (rc)
        return rc;
    if (ctx->fp32)
        launch_moments_lf32(nxy, ctx->mom.as<float>(), ctx->lfp.as<double>(), ctx->bhmask.as<uint8_t>(),
                            ctx->lf_out.as<double>(), ctx->stream);
    else
        launch_moments_lf64(nxy, ctx->mom.as<double>(), ctx->lfp.as<double>(), ctx->bhmask.as<uint8_t>(),
                            ctx->lf_out.as<double>(), ctx->stream);
    CU(cudaGetLastError());
    double *dst[7] = {E, Fx, Fy, Pxx, Pxy, Pyy, F};
    for (int q = 0; q < 7; q++)
        if (dst[q])
            CU(cudaMemcpyAsync(dst[q], ctx->lf_out.as<double>() + q * nxy, nxy * sizeof(double),
                               cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_set_update_tables_each_step(grlbm_ctx *ctx, int32_t enabled, double rk_tol, int32_t max_substeps)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (enabled && !(rk_tol > 0))
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rk_tol must be positive");
    ctx->update_each_step = enabled != 0;
    ctx->update_tol = rk_tol;
    ctx->update_max_substeps = max_substeps;
    return GRLBM_OK;
}

int grlbm_host_write_frame_csv(const grlbm_grid_desc *grid, float time, const double *r, const double *g,
                               const double *b, const double *a, const char *directory, const char *name)
{
    if (!grid || !r || !g || !b || !a || !directory)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_host_write_frame_csv: null argument");
    GridGeom G;
    try
    {
        G = GridGeom::from(*grid);
    }
    catch (const std::exception &e)
    {
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_host_write_frame_csv: %s", e.what());
    }
    std::string err;
    if (!write_frame_csv(G, time, r, g, b, a, directory, name ? name : "", err))
        return fail(nullptr, GRLBM_ERR_HOST, "%s", err.c_str());
    return GRLBM_OK;
}

int grlbm_write_frame_csv(grlbm_ctx *ctx, float time, const char *directory, const char *name)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!directory)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null directory");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    const int nd = ctx->st.n;
    int rc;
    if ((rc = alloc(ctx, ctx->frame_mom, (size_t)6 * nxy * sizeof(double))) ||
        (rc = alloc(ctx, ctx->lf_out, (size_t)7 * nxy * sizeof(double))))
        return rc;
    // ComputeMomentsIF from the current intensities, then ComputeMomentsLF
    // (src/Radiation.cpp:239-301), as RunSimulation does before each frame
    const double *d64 = ctx->dirs64.as<double>();
    if (ctx->fp32)
    {
        if (is_adaptive(ctx))
            launch_moments_from_I32(ctx->I[ctx->cur].as<float>(), nxy, ctx->sl, nd, d64, ctx->cx.as<double>(),
                                    ctx->cy.as<double>(), state_scale(ctx), ctx->ang[ctx->cur].as<double>(),
                                    ctx->frame_mom.as<double>(), ctx->stream);
        else
            launch_moments_from_I32(ctx->I[ctx->cur].as<float>(), nxy, ctx->sl, nd, d64, d64 + nd, d64 + 2 * nd,
                                    state_scale(ctx), nullptr, ctx->frame_mom.as<double>(), ctx->stream);
    }
    else
    {
        if (ctx->fast64)
            launch_moments_from_state64(ctx->I[ctx->cur].as<double>(), nxy, ctx->sl, nd, d64, d64 + nd, d64 + 2 * nd,
                                        state_scale64(ctx), ctx->frame_mom.as<double>(), ctx->stream);
        else if (is_adaptive(ctx))
            launch_moments_from_I64(ctx->I[ctx->cur].as<double>(), nxy, nd, d64, ctx->cx.as<double>(),
                                    ctx->cy.as<double>(), ctx->ang[ctx->cur].as<double>(),
                                    ctx->frame_mom.as<double>(), ctx->stream);
        else
            launch_moments_from_I64(ctx->I[ctx->cur].as<double>(), nxy, nd, d64, d64 + nd, d64 + 2 * nd, nullptr,
                                    ctx->frame_mom.as<double>(), ctx->stream);
        // the moments E..Pyy now hold ComputeMomentsIF's values, as in the reference
        CU(cudaMemcpyAsync(ctx->mom.p, ctx->frame_mom.p, (size_t)6 * nxy * sizeof(double),
                           cudaMemcpyDeviceToDevice, ctx->stream));
    }
    launch_moments_lf64(nxy, ctx->frame_mom.as<double>(), ctx->lfp.as<double>(), ctx->bhmask.as<uint8_t>(),
                        ctx->lf_out.as<double>(), ctx->stream);
    CU(cudaGetLastError());
    std::vector<double> h((size_t)7 * nxy);
    CU(cudaMemcpyAsync(h.data(), ctx->lf_out.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    std::string err;
    // E_LF, Fx_LF, Fy_LF, F_LF (src/Radiation.cpp:780)
    const long long t0 = trace_now_us();
    bool ok;
    {
        TraceScope trace(ctx, kFrameWriterName);
        ok = write_frame_csv(ctx->geo, time, h.data(), h.data() + nxy, h.data() + 2 * nxy, h.data() + 6 * nxy,
                             directory, name ? name : "", err);
    }
    ctx->frame_s += (double)(trace_now_us() - t0) / 1e6;
    if (!ok)
        return fail(ctx, GRLBM_ERR_HOST, "%s", err.c_str());
    return GRLBM_OK;
}

int grlbm_run_simulation(grlbm_ctx *ctx, double t0, double sim_time, double write_period, int32_t save_initial,
                         const char *directory, int64_t *steps_out)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!(sim_time >= 0.0) || !(write_period > 0.0))
        return fail(ctx, GRLBM_ERR_ARGUMENT, "sim_time must be >= 0 and write_period > 0");
    // src/Radiation.cpp:748-750, 772-832 (the tables are built beforehand,
    // grlbm_update_fourier_coefficients; no console output).  The run's own
    // measurements are kept for grlbm_write_log, as Logger::SetValues and
    // the profiler's totals are (src/Radiation.cpp:750, 862-880).
    cudaSetDevice(ctx->device);
    const int64_t time_steps = (int64_t)std::ceil(sim_time / ctx->geo.dt);
    RunLog log;
    log.date = log_date_now();
    unsigned long long it0 = 0;
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaMemcpy(&it0, ctx->counters.p, sizeof it0, cudaMemcpyDeviceToHost));
    ctx->frame_s = 0;
    double step_s = 0;
    auto steps = [&](int64_t n) {
        const long long a = trace_now_us();
        const int rc_ = grlbm_step(ctx, (int32_t)n);
        step_s += (double)(trace_now_us() - a) / 1e6;
        return rc_;
    };
    const long long total0 = trace_now_us();
    {
        TraceScope total(ctx, "Total Time");
        double current = t0, since = 0.0;
        int rc;
        const bool write = directory != nullptr;
        if (write && save_initial)
        {
            if ((rc = grlbm_write_frame_csv(ctx, (float)current, directory, "")))
                return rc;
            since = 0.0;
        }
        int64_t pending = 0; // steps enqueued since the last frame
        for (int64_t n = 0; n < time_steps; n++)
        {
            pending++;
            current += ctx->geo.dt;
            since += ctx->geo.dt;
            if (write && since >= write_period - 1e-8)
            {
                if ((rc = steps(pending)))
                    return rc;
                pending = 0;
                if ((rc = grlbm_write_frame_csv(ctx, (float)current, directory, "")))
                    return rc;
                since = 0.0;
            }
        }
        if (pending && (rc = steps(pending)))
            return rc;
        if (write && since != 0.0)
        {
            if ((rc = grlbm_write_frame_csv(ctx, (float)current, directory, "")))
                return rc;
        }
    }
    const double total_s = (double)(trace_now_us() - total0) / 1e6;
    unsigned long long h[2];
    CU(cudaMemcpy(h, ctx->counters.p, sizeof h, cudaMemcpyDeviceToHost));
    log.time_steps = time_steps;
    log.sim_time = (double)time_steps * ctx->geo.dt;
    // the run's own lambda-iteration average (src/Radiation.cpp:856); the
    // maximum is the context's since its creation
    const double cells = (double)(ctx->geo.nx - 2) * (double)(ctx->gd.jhi - ctx->gd.jlo);
    log.max_iterations = (int32_t)(unsigned)(h[1] & 0xffffffffu);
    log.average_iterations = time_steps > 0 ? (double)(h[0] - it0) / ((double)time_steps * cells) : 0.0;
    log.times = {{"Total Time", total_s},
                 {kFrameWriterName, ctx->frame_s},
                 {kStepName, step_s},
                 {kTablesName, ctx->table_ms / 1e3}};
    log.valid = true;
    ctx->runlog = log;
    if (steps_out)
        *steps_out = time_steps;
    return GRLBM_OK;
}

int grlbm_write_log(grlbm_ctx *ctx, const char *directory)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!directory)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null directory");
    if (!ctx->runlog.valid)
        return fail(ctx, GRLBM_ERR_STATE, "Log.txt describes a grlbm_run_simulation: run one first");
    std::string err;
    if (!write_log_txt(directory, ctx->geo, ctx->mdesc.kind, ctx->mdesc.m, ctx->mdesc.a, ctx->st, ctx->ss,
                       ctx->runlog, err))
        return fail(ctx, GRLBM_ERR_HOST, "%s", err.c_str());
    return GRLBM_OK;
}

int grlbm_host_write_log(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric, int32_t n_dir,
                         int32_t n_fourier, const char *date, int64_t time_steps, int32_t max_iterations,
                         double average_iterations, const char *const *time_names, const double *seconds,
                         int32_t n_times, const char *directory)
{
    if (!grid || !metric || !date || !directory || (n_times > 0 && (!time_names || !seconds)) || n_times < 0 ||
        n_dir < 1 || n_fourier < 1)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_host_write_log: bad arguments");
    GridGeom G;
    StencilTables st, ss;
    try
    {
        G = GridGeom::from(*grid);
        st = StencilTables::build(n_dir, true);
        ss = StencilTables::build(n_fourier, false);
    }
    catch (const std::exception &e)
    {
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_host_write_log: %s", e.what());
    }
    RunLog log;
    log.date = date;
    log.time_steps = time_steps;
    log.sim_time = (double)time_steps * G.dt;
    log.max_iterations = max_iterations;
    log.average_iterations = average_iterations;
    for (int k = 0; k < n_times; k++)
        log.times.emplace_back(time_names[k] ? time_names[k] : "", seconds[k]);
    log.valid = true;
    std::string err;
    if (!write_log_txt(directory, G, metric->kind, metric->m, metric->a, st, ss, log, err))
        return fail(nullptr, GRLBM_ERR_HOST, "%s", err.c_str());
    return GRLBM_OK;
}

int grlbm_trace_begin(grlbm_ctx *ctx, const char *path)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!path || !*path)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null trace path");
    if (ctx->tracing)
        return fail(ctx, GRLBM_ERR_STATE, "a profile session is already open");
    ctx->tracing = true;
    ctx->trace_path = path;
    ctx->trace.clear();
    return GRLBM_OK;
}

int grlbm_trace_end(grlbm_ctx *ctx)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!ctx->tracing)
        return fail(ctx, GRLBM_ERR_STATE, "no profile session is open");
    ctx->tracing = false;
    std::string err;
    const bool ok = write_trace_json(ctx->trace_path, ctx->trace, err);
    ctx->trace.clear();
    if (!ok)
        return fail(ctx, GRLBM_ERR_HOST, "%s", err.c_str());
    return GRLBM_OK;
}

int grlbm_energy(grlbm_ctx *ctx, double *total)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!total)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null output");
    cudaSetDevice(ctx->device);
    if (ctx->fp32)
        launch_energy32(ctx->gd, ctx->mom.as<float>(), ctx->energy_partial.as<double>(), kPartialBlocks,
                        ctx->energy_out.as<double>(), ctx->stream);
    else
        launch_energy64(ctx->gd, ctx->mom.as<double>(), ctx->energy_partial.as<double>(), kPartialBlocks,
                        ctx->energy_out.as<double>(), ctx->stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(total, ctx->energy_out.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_set_rows(grlbm_ctx *ctx, int64_t j_first, int64_t j_end)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (j_first < 1 || j_end > ctx->geo.ny - 1 || j_first >= j_end)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rows [%lld, %lld) outside the interior rows [1, %lld)",
                    (long long)j_first, (long long)j_end, (long long)(ctx->geo.ny - 1));
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->gd.jlo = j_first;
    ctx->gd.jhi = j_end;
    invalidate_graphs(ctx);
    return GRLBM_OK;
}

int grlbm_row_bytes(const grlbm_ctx *ctx, int64_t *bytes)
{
    if (!ctx || !bytes)
        return GRLBM_ERR_ARGUMENT;
    *bytes = ctx->sl.sp == 1 ? ctx->sl.pitch * (int64_t)ctx->st.n * (int64_t)tsize(ctx)
                             : ctx->sl.pitch * ctx->sl.sp * (int64_t)tsize(ctx);
    return GRLBM_OK;
}

int grlbm_copy_rows(grlbm_ctx *ctx, int64_t j_first, int64_t n, void *buffer, int32_t to_buffer)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!buffer || n < 0 || j_first < 0 || j_first + n > ctx->geo.ny)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rows [%lld, %lld) outside the grid's %lld rows", (long long)j_first,
                    (long long)(j_first + n), (long long)ctx->geo.ny);
    if (n == 0)
        return GRLBM_OK;
    cudaSetDevice(ctx->device);
    const size_t es = tsize(ctx);
    if (ctx->sl.sp != 1)
    {
        // cell-major: the rows are one contiguous run
        const size_t row = (size_t)ctx->sl.pitch * (size_t)ctx->sl.sp * es;
        char *state = static_cast<char *>(ctx->I[ctx->cur].p) + (size_t)j_first * row;
        if (to_buffer)
            CU(cudaMemcpyAsync(buffer, state, (size_t)n * row, cudaMemcpyDeviceToDevice, ctx->stream));
        else
            CU(cudaMemcpyAsync(state, buffer, (size_t)n * row, cudaMemcpyDeviceToDevice, ctx->stream));
        return GRLBM_OK;
    }
    const size_t width = (size_t)n * ctx->sl.pitch * es, pitch = (size_t)ctx->sl.plane * es;
    char *state = static_cast<char *>(ctx->I[ctx->cur].p) + (size_t)j_first * ctx->sl.pitch * es;
    if (to_buffer)
        CU(cudaMemcpy2DAsync(buffer, width, state, pitch, width, (size_t)ctx->st.n, cudaMemcpyDeviceToDevice,
                             ctx->stream));
    else
        CU(cudaMemcpy2DAsync(state, pitch, buffer, width, width, (size_t)ctx->st.n, cudaMemcpyDeviceToDevice,
                             ctx->stream));
    return GRLBM_OK;
}

int grlbm_node_row_bytes(const grlbm_ctx *ctx, int32_t what, int64_t *bytes)
{
    if (!ctx || !bytes)
        return GRLBM_ERR_ARGUMENT;
    if (what == GRLBM_ROWS_ANGLES)
        *bytes = is_adaptive(ctx) ? ctx->gd.nx * (int64_t)sizeof(double) : 0;
    else if (what == GRLBM_ROWS_MOMENTS)
        *bytes = 6 * ctx->gd.nx * (int64_t)tsize(ctx);
    else
        return GRLBM_ERR_ARGUMENT;
    return is_adaptive(ctx) || what == GRLBM_ROWS_MOMENTS ? GRLBM_OK : GRLBM_ERR_UNSUPPORTED;
}

int grlbm_copy_node_rows(grlbm_ctx *ctx, int32_t what, int64_t j_first, int64_t n, void *buffer, int32_t to_buffer)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (what != GRLBM_ROWS_ANGLES && what != GRLBM_ROWS_MOMENTS)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "unknown node-row field %d", what);
    if (what == GRLBM_ROWS_ANGLES && !is_adaptive(ctx))
        return fail(ctx, GRLBM_ERR_UNSUPPORTED, "rotation angles exist for adaptive streaming only");
    if (!buffer || n < 0 || j_first < 0 || j_first + n > ctx->geo.ny)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rows [%lld, %lld) outside the grid's %lld rows", (long long)j_first,
                    (long long)(j_first + n), (long long)ctx->geo.ny);
    if (n == 0)
        return GRLBM_OK;
    cudaSetDevice(ctx->device);
    const size_t nx = (size_t)ctx->gd.nx;
    if (what == GRLBM_ROWS_ANGLES)
    {
        double *ang = ctx->ang[ctx->cur].as<double>() + (size_t)j_first * nx;
        const size_t bytes = (size_t)n * nx * sizeof(double);
        CU(cudaMemcpyAsync(to_buffer ? buffer : ang, to_buffer ? ang : buffer, bytes, cudaMemcpyDeviceToDevice,
                           ctx->stream));
        return GRLBM_OK;
    }
    // the six moment planes: [plane][row][i] in the buffer
    const size_t es = tsize(ctx), width = (size_t)n * nx * es, pitch = (size_t)ctx->gd.nxy * es;
    char *mom = static_cast<char *>(ctx->mom.p) + (size_t)j_first * nx * es;
    if (to_buffer)
        CU(cudaMemcpy2DAsync(buffer, width, mom, pitch, width, 6, cudaMemcpyDeviceToDevice, ctx->stream));
    else
        CU(cudaMemcpy2DAsync(mom, pitch, buffer, width, width, 6, cudaMemcpyDeviceToDevice, ctx->stream));
    return GRLBM_OK;
}

int grlbm_set_tile_shape(grlbm_ctx *ctx, int32_t tile_x, int32_t tile_y)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!is_tiled(ctx))
        return fail(ctx, GRLBM_ERR_UNSUPPORTED,
                    "tiles are a setting of the fixed streaming step of the precision and fast FP64 forms");
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    return set_step32_tile(ctx, tile_x, tile_y);
}

int grlbm_get_tile_shape(const grlbm_ctx *ctx, int32_t *tile_x, int32_t *tile_y)
{
    if (!ctx || !tile_x || !tile_y)
        return GRLBM_ERR_ARGUMENT;
    if (!is_tiled(ctx))
        return GRLBM_ERR_UNSUPPORTED;
    *tile_x = ctx->tile_x;
    *tile_y = ctx->tile_y;
    return GRLBM_OK;
}

int grlbm_departure_rows(grlbm_ctx *ctx, int32_t *rows)
{
    if (!ctx || !rows)
        return GRLBM_ERR_ARGUMENT;
    if (ctx->run.streaming_type == GRLBM_FLAT_ADAPTIVE)
    {
        // any rotated direction: |dy| <= dt, the corners floor(jt) and floor(jt)
        // + 1 (1e-3 row absorbs the FP32 form's rounding of jt)
        *rows = (int32_t)std::floor(ctx->geo.dt / ctx->geo.dy + 1e-3) + 1;
        return GRLBM_OK;
    }
    if (ctx->run.streaming_type == GRLBM_CURVED_ADAPTIVE)
        return adaptive_departure_rows(ctx, rows);
    if (ctx->run.streaming_type == GRLBM_FLAT_FIXED)
    {
        int ext = 0;
        for (int d = 0; d < ctx->st.n; d++)
        {
            const double oy = -ctx->st.cy[d] * ctx->geo.dt / ctx->geo.dy;
            const double jf = std::floor(oy);
            ext = std::max(ext, (int)std::max(std::fabs(jf), std::fabs(jf + 1.0)));
        }
        *rows = ext;
        return GRLBM_OK;
    }
    if (!ctx->tables)
        return fail(ctx, GRLBM_ERR_STATE, "departure rows need the geodesic tables");
    cudaSetDevice(ctx->device);
    unsigned long long h[6];
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaMemcpy(h, ctx->counters.p, sizeof h, cudaMemcpyDeviceToHost));
    *rows = (int32_t)(unsigned)(h[5] & 0xffffffffu);
    return GRLBM_OK;
}

int grlbm_get_stats(grlbm_ctx *ctx, grlbm_stats *s)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!s)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null output");
    cudaSetDevice(ctx->device);
    unsigned long long h[7];
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaMemcpy(h, ctx->counters.p, sizeof h, cudaMemcpyDeviceToHost));
    if (int rc = check_fault(ctx))
        return rc;
    s->steps = ctx->steps;
    s->max_iterations = (int32_t)(unsigned)(h[1] & 0xffffffffu);
    const double denom = (double)ctx->steps * (double)(ctx->geo.nx - 2) * (double)(ctx->gd.jhi - ctx->gd.jlo);
    s->average_iterations = ctx->steps ? (double)h[0] / denom : 0.0;
    s->rk_substeps = (int64_t)h[2];
    s->rk_nonconverged = (int32_t)(unsigned)h[3];
    s->departures_off_grid = (int32_t)(unsigned)h[4];
    s->table_ms = ctx->table_ms;
    s->far_departures = ctx->fp32 || ctx->fast64 ? (int64_t)h[6] : 0;
    return GRLBM_OK;
}

// ---------------------------------------------------------- host helpers
int grlbm_host_stencil(int32_t n_order, int32_t is_intensity, double *w, double *phi, double *cx, double *cy,
                       int64_t *ig_index, double *ig_weight)
{
    if (n_order < 1 || n_order > 4096)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "bad stencil order");
    StencilTables s = StencilTables::build(n_order, is_intensity != 0);
    for (int d = 0; d < n_order; d++)
    {
        if (w)
            w[d] = s.w[d];
        if (phi)
            phi[d] = s.phi[d];
        if (cx)
            cx[d] = s.cx[d];
        if (cy)
            cy[d] = s.cy[d];
    }
    if (is_intensity)
    {
        if (ig_index)
            std::copy(s.ig_index.begin(), s.ig_index.end(), ig_index);
        if (ig_weight)
            std::copy(s.ig_weight.begin(), s.ig_weight.end(), ig_weight);
    }
    return GRLBM_OK;
}

int grlbm_host_flux_table(int32_t n_order, int32_t *size, double *inputs, double *sigma, double *normalization,
                          int32_t capacity)
{
    if (n_order < 4 || n_order > 4096 || !size)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "bad arguments");
    StencilTables s = StencilTables::build(n_order, true);
    *size = (int32_t)s.lut_in.size();
    const int n = std::min<int>(capacity, (int)s.lut_in.size());
    for (int k = 0; k < n; k++)
    {
        if (inputs)
            inputs[k] = s.lut_in[k];
        if (sigma)
            sigma[k] = s.lut_sigma[k];
        if (normalization)
            normalization[k] = s.lut_norm[k];
    }
    return GRLBM_OK;
}

int grlbm_host_metric_arrays(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric, double *out)
{
    if (!grid || !metric || !out || grid->nx_ < 2 || grid->ny_ < 2)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "bad arguments");
    if (metric->kind < GRLBM_MINKOWSKI || metric->kind > GRLBM_KERRSCHILD)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "unknown metric kind");
    const GridGeom g = GridGeom::from(*grid);
    const MetricArrays M = MetricArrays::build(g, *metric);
    std::copy(M.arr.begin(), M.arr.end(), out);
    return GRLBM_OK;
}

} // extern "C"

// ---------------------------------------------------------------- batches
// the concurrent shapes share out at most this many GPUs' worth of resident
// blocks (blocks_per_sm = -1 .. -kBatchMaxShare)
constexpr int kBatchMaxShare = 8;
// a new batch's shape: the concurrent launches on shares of this many GPUs
// (the fastest on the 64-problem benchmark batch, with 6)
constexpr int kBatchDefaultShare = 4;

struct grlbm_batch
{
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<grlbm_ctx *> ctx;
    std::vector<Batch32Item> items; // in launch order
    std::vector<int> order;         // items[k] is context order[k]
    std::vector<int> grid;          // items[k]'s grid in the concurrent shapes
    DevBuf d_items, d_first, d_dirs, counters;
    int total_tiles = 0, passes = 1, warp_stride = 0, s_offset = 0, blocks_per_sm_max = 1, blocks_per_sm = 1, sms = 1;
    int item_bytes = 0; // each warp's copy of its problem's arguments and tables
    // every problem is an FP32 fixed-streaming one without active sources:
    // the persistent kernel can step the batch (else only the concurrent
    // shapes, which run each problem's own step)
    bool persistent_ok = true;
    size_t smem = 0;
    int largest_first = 0;
    int flip = 0; // parity of the steps taken since the items were built
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // blocks_per_sm <= 0: each problem's own step kernel, the problems'
    // launch chains running concurrently on their streams, forked from and
    // joined back to the batch stream by these events (below 0 with the
    // grids cut to shares of -blocks_per_sm GPUs' worth of resident blocks)
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    ~grlbm_batch()
    {
        for (auto &g : graph)
            if (g)
                cudaGraphExecDestroy(g);
        if (fork)
            cudaEventDestroy(fork);
        for (cudaEvent_t e : join)
            if (e)
                cudaEventDestroy(e);
        if (stream)
            cudaStreamDestroy(stream);
    }
};

namespace
{
int bfail(grlbm_batch *b, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b)
        b->err = buf;
    else
        g_create_error = buf;
    return code;
}

#define BCU(call)                                                                                  \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return bfail(b, GRLBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

void batch_drop_graphs(grlbm_batch *b)
{
    for (auto &g : b->graph)
        if (g)
        {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// A problem's estimated step time in arbitrary units: its cells times (its
// directions + 48), times 1.6 for curved streaming, times its form's cost
// against the FP32 fixed-streaming step.  The FP32 step's rates at 512^2 with
// 16, 32 and 64 directions fit a per-cell cost of a + b nd with a between 40
// and 57 b, curved streaming 1.5-1.75 times flat; at 400^2 x 64 the fast FP64
// step takes 1.9 times as long, the plain FP64 step 4.7 times, and adaptive
// streaming 4.9 (FP32) and 10.9 (plain) times.
double batch_cost(const grlbm_ctx *c)
{
    const bool curved = is_curved(c);
    double form = 1.0;
    if (c->fast64)
        form = 1.9;
    else if (is_adaptive(c))
        form = c->fp32 ? 4.9 : 10.9;
    else if (!c->fp32)
        form = 4.7;
    return (double)c->ncell * (c->st.n + 48.0) * (curved ? 1.6 : 1.0) * form;
}

// Passes, shared memory and occupancy of the persistent kernel for the
// problems' current tile shapes.
int batch_geometry(grlbm_batch *b)
{
    if (!b->persistent_ok)
    {
        b->blocks_per_sm_max = 0;
        return GRLBM_OK;
    }
    // each warp's buffer: the largest patch of the problems, then the largest
    // streamed-value rows
    b->passes = 1;
    b->s_offset = 0;
    int s_rows = 0, q = 1;
    for (grlbm_ctx *c : b->ctx)
    {
        b->passes = std::max(b->passes, c->passes);
        b->s_offset = std::max(b->s_offset, step32_patch_floats(c->tile_x, c->tile_y, (int)c->sl.sp));
        s_rows = std::max(s_rows, step32_s_stride(c->st.n));
        q = std::max(q, c->dirs.q);
    }
    b->item_bytes = step32_batch_item_bytes(q);
    b->warp_stride = b->item_bytes + ((b->s_offset + kStep32UnitCells * s_rows) * 4 + 127) / 128 * 128;
    b->smem = step32_batch_smem(b->warp_stride);
    if (b->smem > (size_t)kStep32MaxSmem)
        return bfail(b, GRLBM_ERR_ARGUMENT, "the batch's largest patch needs %zu bytes of shared memory", b->smem);
    BCU(step32_occupancy(b->passes, true, true, b->smem, &b->blocks_per_sm_max, 0));
    if (b->blocks_per_sm_max < 1)
        return bfail(b, GRLBM_ERR_CUDA, "the batched kernel does not fit on an SM");
    if (b->blocks_per_sm > b->blocks_per_sm_max)
        b->blocks_per_sm = b->blocks_per_sm_max;
    return GRLBM_OK;
}

// (Re)build the launch list from the contexts' current buffers and tiles, in
// the chosen order, and upload it.
int batch_build(grlbm_batch *b)
{
    const int n = (int)b->ctx.size();
    int rc = batch_geometry(b);
    if (rc)
        return rc;
    std::vector<int> order(n);
    for (int k = 0; k < n; k++)
        order[k] = k;
    if (b->largest_first)
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return batch_cost(b->ctx[x]) > batch_cost(b->ctx[y]); });
    b->order = order;
    b->items.assign(n, Batch32Item{});
    std::vector<int> first(n + 1, 0);
    const DirTable *dirs = b->d_dirs.as<DirTable>();
    for (int k = 0; k < n; k++)
    {
        grlbm_ctx *c = b->ctx[order[k]];
        Batch32Item &it = b->items[k];
        it.cur0 = c->cur;
        first[k + 1] = first[k];
        if (!b->persistent_ok)
            continue; // the concurrent shapes read cur0 only
        it.a[0] = step32_args(c, 0);
        it.a[1] = step32_args(c, 1);
        it.dt = dirs + order[k];
        it.curved = c->run.streaming_type == GRLBM_CURVED_FIXED;
        it.mode = step32_mode(c->st.n);
        first[k + 1] += step32_tiles(c);
    }
    b->total_tiles = first[n];
    // the concurrent shapes' grids: each problem's own persistent grid, or
    // (blocks_per_sm = -m) its share of m GPUs' worth of resident blocks by
    // its estimated cost, so that the problems' kernels are resident side by
    // side instead of each filling the GPU in turn
    b->grid.assign(n, 0);
    double wsum = 0.0;
    for (int k = 0; k < n; k++)
        wsum += batch_cost(b->ctx[order[k]]);
    for (int k = 0; k < n; k++)
    {
        const grlbm_ctx *c = b->ctx[order[k]];
        b->grid[k] = c->step_blocks;
        if (b->blocks_per_sm < 0 && is_tiled(c)) // the other forms' grids cover their work once
            b->grid[k] = std::max(1, std::min(c->step_blocks, (int)std::ceil(-b->blocks_per_sm * c->step_blocks *
                                                                             batch_cost(c) / wsum)));
    }
    if (alloc(nullptr, b->d_items, n * sizeof(Batch32Item)) || alloc(nullptr, b->d_first, (n + 1) * sizeof(int)))
        return bfail(b, GRLBM_ERR_CUDA, "cannot allocate the batch launch list");
    BCU(cudaMemcpy(b->d_items.p, b->items.data(), n * sizeof(Batch32Item), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_first.p, first.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    b->flip = 0;
    batch_drop_graphs(b);
    return GRLBM_OK;
}

// Enqueue n steps of every problem on the batch stream, the first reading
// the buffers of parity `flip`: one persistent launch per step, or (shapes 0
// and below) each problem's chain of step kernels on its own stream between a
// fork and a join on the batch stream.
int batch_enqueue(grlbm_batch *b, int n, int flip)
{
    if (b->blocks_per_sm > 0)
    {
        for (int s = 0; s < n; s++)
            launch_step_batch32(b->d_items.as<Batch32Item>(), b->d_first.as<int>(), (int)b->items.size(),
                                b->total_tiles, flip ^ (s & 1), b->counters.as<unsigned>(), b->passes,
                                b->sms * b->blocks_per_sm, b->smem, b->warp_stride, b->s_offset, b->item_bytes,
                                b->stream);
        return GRLBM_OK;
    }
    BCU(cudaEventRecord(b->fork, b->stream));
    for (size_t k = 0; k < b->items.size(); k++)
    {
        grlbm_ctx *c = b->ctx[b->order[k]];
        BCU(cudaStreamWaitEvent(c->stream, b->fork, 0));
        for (int s = 0; s < n; s++)
            if (enqueue_step(c, b->items[k].cur0 ^ flip ^ (s & 1), true, b->grid[k]))
                return bfail(b, GRLBM_ERR_CUDA, "problem %zu: %s", k, c->err.c_str());
        BCU(cudaEventRecord(b->join[k], c->stream));
        BCU(cudaStreamWaitEvent(b->stream, b->join[k], 0));
    }
    return GRLBM_OK;
}

// Brings the launch list in line with the contexts (stepped on their own
// since the last batch step, or never batched): rebuilt when any context's
// current buffer is not the one the list expects.
int batch_sync_state(grlbm_batch *b)
{
    for (size_t k = 0; k < b->items.size(); k++)
        if (b->ctx[b->order[k]]->cur != (b->items[k].cur0 ^ b->flip))
            return batch_build(b);
    return GRLBM_OK;
}

// Captures (once) the graph of kGraphSteps batch steps that starts from the
// buffers of parity `flip`.
int batch_graph(grlbm_batch *b, int flip)
{
    if (b->graph[flip])
        return GRLBM_OK;
    cudaGraph_t g = nullptr;
    BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int erc = batch_enqueue(b, kGraphSteps, flip);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (erc)
    {
        if (g)
            cudaGraphDestroy(g);
        return erc;
    }
    if (e != cudaSuccess)
        return bfail(b, GRLBM_ERR_CUDA, "batch graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph[flip], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return bfail(b, GRLBM_ERR_CUDA, "batch graph instantiation failed: %s", cudaGetErrorString(e));
    return GRLBM_OK;
}

int batch_steps(grlbm_batch *b, int n)
{
    for (grlbm_ctx *c : b->ctx)
        BCU(cudaStreamSynchronize(c->stream));
    int rc = batch_sync_state(b);
    if (rc)
        return rc;
    int left = n;
    while (left >= kGraphSteps)
    {
        if ((rc = batch_graph(b, b->flip)))
            return rc;
        BCU(cudaGraphLaunch(b->graph[b->flip], b->stream));
        left -= kGraphSteps; // even: parity unchanged
    }
    if (left > 0)
    {
        if ((rc = batch_enqueue(b, left, b->flip)))
            return rc;
        b->flip ^= left & 1;
    }
    BCU(cudaGetLastError());
    BCU(cudaStreamSynchronize(b->stream));
    for (size_t k = 0; k < b->items.size(); k++)
    {
        grlbm_ctx *c = b->ctx[b->order[k]];
        c->cur = b->items[k].cur0 ^ b->flip;
        c->steps += n;
    }
    for (grlbm_ctx *c : b->ctx)
        if (check_fault(c))
            return bfail(b, GRLBM_ERR_CUDA, "problem %p: %s", (void *)c, c->err.c_str());
    return GRLBM_OK;
}

// The time per step of `trial_steps` batch steps, rounded up to whole
// graphs of kGraphSteps steps and replayed as grlbm_batch_step replays them,
// after one untimed replay; -1 on failure.  (Each problem's launch chain in
// the concurrent shapes spans a whole graph, so a shorter trial would time
// mostly its tail.)
float batch_time(grlbm_batch *b, int trial_steps, cudaEvent_t e0, cudaEvent_t e1, int *rc)
{
    if ((*rc = batch_build(b)) || (*rc = batch_graph(b, 0)))
        return -1.f;
    const int reps = (trial_steps + kGraphSteps - 1) / kGraphSteps;
    bool ok = cudaGraphLaunch(b->graph[0], b->stream) == cudaSuccess &&
              cudaEventRecord(e0, b->stream) == cudaSuccess;
    for (int r = 0; r < reps && ok; r++)
        ok = cudaGraphLaunch(b->graph[0], b->stream) == cudaSuccess;
    ok = ok && cudaEventRecord(e1, b->stream) == cudaSuccess;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess || !ok)
    {
        *rc = bfail(b, GRLBM_ERR_CUDA, "autotune: trial steps failed");
        return -1.f;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / (float)(reps * kGraphSteps);
}
} // namespace

extern "C" {

int grlbm_batch_create(grlbm_ctx *const *ctxs, int32_t n, grlbm_batch **out)
{
    if (!ctxs || !out || n < 1)
        return bfail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_batch_create: no contexts");
    *out = nullptr;
    std::unique_ptr<grlbm_batch> owner(new grlbm_batch);
    grlbm_batch *b = owner.get();
    for (int k = 0; k < n; k++)
    {
        grlbm_ctx *c = ctxs[k];
        if (!c)
            return bfail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_batch_create: context %d is null", k);
        if (c->device != ctxs[0]->device)
            return bfail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_batch_create: contexts on different devices");
        if (is_curved(c) && !c->tables)
            return bfail(nullptr, GRLBM_ERR_STATE, "grlbm_batch_create: context %d has no geodesic tables", k);
        if (c->update_each_step)
            return bfail(nullptr, GRLBM_ERR_UNSUPPORTED,
                         "grlbm_batch_create: context %d rebuilds its tables every step (not batched)", k);
        if (c->partial)
            return bfail(nullptr, GRLBM_ERR_STATE, "grlbm_batch_create: context %d is inside a step taken in row ranges",
                         k);
        if (!is_fixed32(c) || (c->run.keep_source_nodes_active && c->nsrc > 0))
            b->persistent_ok = false;
        for (int j = 0; j < k; j++)
            if (ctxs[j] == c)
                return bfail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_batch_create: context %d appears twice", k);
        b->ctx.push_back(c);
    }
    b->device = ctxs[0]->device;
    cudaSetDevice(b->device);
    BCU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCU(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    b->join.assign(n, nullptr);
    for (int k = 0; k < n; k++)
        BCU(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
    BCU(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    if (alloc(nullptr, b->counters, 2 * sizeof(unsigned)))
        return bfail(nullptr, GRLBM_ERR_CUDA, "grlbm_batch_create: cannot allocate the tile counters");
    BCU(cudaMemset(b->counters.p, 0, b->counters.bytes));
    std::vector<DirTable> dirs(n);
    for (int k = 0; k < n; k++)
        dirs[k] = ctxs[k]->dirs;
    if (upload(nullptr, b->d_dirs, dirs))
        return bfail(nullptr, GRLBM_ERR_CUDA, "grlbm_batch_create: cannot upload the direction tables");
    int rc = batch_geometry(b);
    if (rc)
        return bfail(nullptr, rc, "%s", b->err.c_str());
    b->blocks_per_sm = -kBatchDefaultShare;
    b->largest_first = 1;
    if ((rc = batch_build(b)))
        return bfail(nullptr, rc, "%s", b->err.c_str());
    *out = owner.release();
    return GRLBM_OK;
}

void grlbm_batch_destroy(grlbm_batch *b)
{
    if (b)
    {
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->stream);
        delete b;
    }
}

const char *grlbm_batch_last_error(const grlbm_batch *b) { return b ? b->err.c_str() : g_create_error.c_str(); }

int grlbm_batch_step(grlbm_batch *b, int32_t n_steps)
{
    if (!b)
        return GRLBM_ERR_ARGUMENT;
    if (n_steps < 0)
        return bfail(b, GRLBM_ERR_ARGUMENT, "negative step count");
    cudaSetDevice(b->device);
    return batch_steps(b, n_steps);
}

int grlbm_batch_set_shape(grlbm_batch *b, int32_t blocks_per_sm, int32_t largest_first)
{
    if (!b)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(b->device);
    int rc = batch_geometry(b);
    if (rc)
        return rc;
    if (blocks_per_sm > 0 && !b->persistent_ok)
        return bfail(b, GRLBM_ERR_UNSUPPORTED,
                     "the persistent launch steps FP32 fixed-streaming problems without active sources only");
    if (blocks_per_sm < -kBatchMaxShare || blocks_per_sm > b->blocks_per_sm_max)
        return bfail(b, GRLBM_ERR_ARGUMENT, "blocks_per_sm must be in [%d, %d]", -kBatchMaxShare,
                     b->blocks_per_sm_max);
    for (grlbm_ctx *c : b->ctx)
        BCU(cudaStreamSynchronize(c->stream));
    b->blocks_per_sm = blocks_per_sm;
    b->largest_first = largest_first != 0;
    return batch_build(b);
}

int grlbm_batch_autotune(grlbm_batch *b, int32_t trial_steps, int32_t *blocks_per_sm, int32_t *largest_first)
{
    if (!b)
        return GRLBM_ERR_ARGUMENT;
    if (trial_steps < 1)
        return bfail(b, GRLBM_ERR_ARGUMENT, "trial_steps must be positive");
    cudaSetDevice(b->device);
    for (grlbm_ctx *c : b->ctx)
        BCU(cudaStreamSynchronize(c->stream));
    int rc = batch_sync_state(b);
    if (rc)
        return rc;
    // save every problem's state (current intensities, and rotation angles
    // for adaptive streaming; moments, counters); the trial steps are undone
    // afterwards
    std::vector<std::pair<DevBuf *, std::unique_ptr<DevBuf>>> saved;
    for (grlbm_ctx *c : b->ctx)
    {
        std::vector<DevBuf *> src = {&c->I[c->cur], &c->mom, &c->counters};
        if (is_adaptive(c))
            src.push_back(&c->ang[c->cur]);
        for (DevBuf *d : src)
        {
            std::unique_ptr<DevBuf> copy(new DevBuf);
            if (alloc(nullptr, *copy, d->bytes))
                return bfail(b, GRLBM_ERR_CUDA, "autotune: cannot allocate a state copy");
            BCU(cudaMemcpy(copy->p, d->p, d->bytes, cudaMemcpyDeviceToDevice));
            saved.emplace_back(d, std::move(copy));
        }
    }
    cudaEvent_t e0, e1;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    // 1. the launch shape: persistent launches (largest problem first or not,
    //    at each resident block count down to two below the limit), or the
    //    problems' own kernels launched concurrently, with their own grids or
    //    with shares of one to kBatchMaxShare GPUs' worth of resident blocks
    float best = -1.f;
    int best_bps = b->blocks_per_sm, best_lf = b->largest_first;
    std::vector<std::pair<int, int>> shapes;
    for (int lf = 0; lf <= 1; lf++)
        for (int bps = b->blocks_per_sm_max; bps >= 1 && bps >= b->blocks_per_sm_max - 2; bps--)
            shapes.emplace_back(bps, lf);
    for (int m = 0; m <= kBatchMaxShare; m++)
        shapes.emplace_back(-m, 1);
    for (const auto &shape : shapes)
    {
        b->blocks_per_sm = shape.first;
        b->largest_first = shape.second;
        const float ms = batch_time(b, trial_steps, e0, e1, &rc);
        if (rc)
            break;
        if (best < 0.f || ms < best)
            best = ms, best_bps = shape.first, best_lf = shape.second;
    }
    b->blocks_per_sm = best_bps;
    b->largest_first = best_lf;
    // 2. the tile of each size class (problems of one grid size and
    //    direction count share a tile), largest class first: each class tries
    //    the candidate tiles with the others fixed, and keeps the fastest.
    //    Classes below 2% of the batch's estimated cost keep their tiles: their
    //    share of a trial is within its noise.
    if (!rc)
    {
        double wsum = 0.0;
        for (grlbm_ctx *c : b->ctx)
            wsum += batch_cost(c);
        std::vector<std::pair<int64_t, std::vector<grlbm_ctx *>>> classes;
        for (grlbm_ctx *c : b->ctx)
        {
            if (!is_tiled(c)) // the other forms have no tile
                continue;
            const int64_t key = ((c->gd.nx_ * 65536 + c->gd.ny_) * 512 + c->st.n) * 2 + (c->fast64 ? 1 : 0);
            auto it = std::find_if(classes.begin(), classes.end(), [&](const auto &x) { return x.first == key; });
            if (it == classes.end())
                classes.push_back({key, {c}});
            else
                it->second.push_back(c);
        }
        std::stable_sort(classes.begin(), classes.end(), [](const auto &x, const auto &y) {
            const grlbm_ctx *a = x.second[0], *c = y.second[0];
            return a->ncell * a->st.n * (int64_t)x.second.size() > c->ncell * c->st.n * (int64_t)y.second.size();
        });
        static const int cand[][2] = {{2, 2}, {4, 2}, {2, 4}, {4, 4}, {8, 2}, {2, 8}, {16, 1}};
        for (auto &cls : classes)
        {
            grlbm_ctx *c0 = cls.second[0];
            int bx = c0->tile_x, by = c0->tile_y;
            double wc = 0.0;
            for (grlbm_ctx *c : cls.second)
                wc += batch_cost(c);
            if (wc < 0.02 * wsum)
                continue;
            for (const auto &t : cand)
            {
                if (t[0] == bx && t[1] == by)
                    continue;
                size_t smem = 0;
                int per_sm = 0;
                if ((rc = tiled_fit(c0, t[0], t[1], &smem, &per_sm)))
                    break;
                if (smem > (size_t)kStep32MaxSmem || per_sm < 1)
                    continue;
                for (grlbm_ctx *c : cls.second)
                    if ((rc = set_step32_tile(c, t[0], t[1])))
                        break;
                if (rc)
                    break;
                const float ms = batch_time(b, trial_steps, e0, e1, &rc);
                if (rc)
                    break;
                if (ms < best)
                    best = ms, bx = t[0], by = t[1];
            }
            if (rc)
                break;
            for (grlbm_ctx *c : cls.second)
                if ((rc = set_step32_tile(c, bx, by)))
                    break;
            if (rc)
                break;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // restore the saved state (the trials leave every context's current
    // buffer index as it was)
    for (auto &sv : saved)
        BCU(cudaMemcpy(sv.first->p, sv.second->p, sv.first->bytes, cudaMemcpyDeviceToDevice));
    if (rc)
        return rc;
    if ((rc = batch_build(b)))
        return rc;
    if (blocks_per_sm)
        *blocks_per_sm = b->blocks_per_sm;
    if (largest_first)
        *largest_first = b->largest_first;
    return GRLBM_OK;
}

} // extern "C"

// ---------------------------------------------------------------- adjoint
struct grlbm_adjoint
{
    std::string err;
    grlbm_ctx *ctx = nullptr;
    int every = 20;          // checkpoint interval (steps)
    int64_t n_steps = 0;     // steps of the last forward
    int64_t n_entries = 0;   // inverse-table entries
    DevBuf slices;           // int64: first entry of each slice of the sliced inverse table, and the end
    unsigned *srcq = nullptr;
    float *coef = nullptr;
    std::vector<std::unique_ptr<DevBuf>> ckpt; // states at steps 0, every, 2 every, ...
    std::vector<std::unique_ptr<DevBuf>> seg;  // the recomputed outputs of one segment
    DevBuf clamp, cycles, e0;                  // records of one segment
    DevBuf lam, lamS, grads, dLdE, mom, counters;
    ~grlbm_adjoint()
    {
        cudaFree(srcq);
        cudaFree(coef);
    }
};

namespace
{
int afail(grlbm_adjoint *a, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (a)
        a->err = buf;
    else
        g_create_error = buf;
    return code;
}
#define ACU(call)                                                                                  \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return afail(adj, GRLBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
    } while (0)

bool all_zero(const DevBuf &b, size_t n)
{
    std::vector<double> h(n);
    if (cudaMemcpy(h.data(), b.p, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    for (double v : h)
        if (v != 0.0)
            return false;
    return true;
}
} // namespace

extern "C" {

int grlbm_adjoint_create(grlbm_ctx *ctx, int32_t checkpoint_every, grlbm_adjoint **out)
{
    grlbm_adjoint *adj = nullptr;
    if (!ctx || !out || checkpoint_every < 1)
        return afail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_adjoint_create: null context/output or interval < 1");
    *out = nullptr;
    if (ctx->fp32 || ctx->fast64)
        return afail(nullptr, GRLBM_ERR_UNSUPPORTED, "grlbm_adjoint_create: the adjoint follows GRLBM_PLAIN_FP64");
    if (is_adaptive(ctx))
        return afail(nullptr, GRLBM_ERR_UNSUPPORTED, "grlbm_adjoint_create: the adjoint follows the fixed streaming types");
    const bool curved = ctx->run.streaming_type == GRLBM_CURVED_FIXED;
    if (curved && !ctx->tables)
        return afail(nullptr, GRLBM_ERR_STATE, "grlbm_adjoint_create: build the geodesic tables first");
    if (ctx->run.keep_source_nodes_active && ctx->nsrc > 0)
        return afail(nullptr, GRLBM_ERR_UNSUPPORTED, "grlbm_adjoint_create: active source nodes are not differentiated");
    if (ctx->gd.jlo != 1 || ctx->gd.jhi != ctx->geo.ny - 1)
        return afail(nullptr, GRLBM_ERR_UNSUPPORTED, "grlbm_adjoint_create: the context steps a band of rows only");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    const int64_t nxy = ctx->gd.nxy, ncell = ctx->gd.ncell;
    const int nd = ctx->st.n;
    if (!all_zero(ctx->cu1, nxy) || !all_zero(ctx->cu2, nxy) || !all_zero(ctx->ck3, nxy))
        return afail(nullptr, GRLBM_ERR_UNSUPPORTED,
                     "grlbm_adjoint_create: the adjoint needs a fluid at rest without anisotropic scattering "
                     "(ux = uy = kappa1 = 0)");
    if ((int64_t)nd * ncell >= (int64_t)1 << 30)
        return afail(nullptr, GRLBM_ERR_ARGUMENT, "grlbm_adjoint_create: nDir * cells must stay below 2^30");
    std::unique_ptr<grlbm_adjoint> owner(new grlbm_adjoint);
    adj = owner.get();
    adj->ctx = ctx;
    adj->every = checkpoint_every;
    if (alloc(nullptr, adj->slices, (size_t)(adj_slices((int64_t)nd * nxy) + 1) * sizeof(int64_t)))
        return afail(nullptr, GRLBM_ERR_CUDA, "grlbm_adjoint_create: %s", g_create_error.c_str());
    AdjEntryArgs ea{};
    ea.g = ctx->gd;
    ea.nd = nd;
    ea.ng = ctx->ng;
    ea.curved = curved;
    ea.rec = ctx->rec.as<double4>();
    ea.ig_rows = ctx->ig_rows.as<IgRow>();
    ea.alpha = ctx->alpha.as<double>();
    ea.acube = ctx->acube.as<double>();
    ea.flags = ctx->flags.as<uint8_t>();
    ea.cx = ctx->cx.as<double>();
    ea.cy = ctx->cy.as<double>();
    cudaError_t e = adj_build_table(ea, adj->slices.as<int64_t>(), &adj->srcq, &adj->coef, &adj->n_entries,
                                    ctx->stream);
    if (e != cudaSuccess)
        return afail(nullptr, GRLBM_ERR_CUDA, "grlbm_adjoint_create: inverse table: %s", cudaGetErrorString(e));
    const size_t sb = (size_t)nd * nxy * sizeof(double);
    adj->seg.resize(checkpoint_every);
    for (auto &b : adj->seg)
    {
        b.reset(new DevBuf);
        if (alloc(nullptr, *b, sb))
            return afail(nullptr, GRLBM_ERR_CUDA, "grlbm_adjoint_create: %s", g_create_error.c_str());
    }
    if (alloc(nullptr, adj->clamp, (size_t)checkpoint_every * nd * ncell) ||
        alloc(nullptr, adj->cycles, (size_t)checkpoint_every * ncell * sizeof(int)) ||
        alloc(nullptr, adj->e0, (size_t)checkpoint_every * ncell * sizeof(double)) ||
        alloc(nullptr, adj->lam, (size_t)nd * nxy * sizeof(float)) ||
        alloc(nullptr, adj->lamS, (size_t)nd * ncell * sizeof(float)) ||
        alloc(nullptr, adj->grads, (size_t)3 * nxy * sizeof(double)) ||
        alloc(nullptr, adj->dLdE, (size_t)nxy * sizeof(double)) ||
        alloc(nullptr, adj->mom, (size_t)6 * nxy * sizeof(double)) ||
        alloc(nullptr, adj->counters, 8 * sizeof(unsigned long long)))
        return afail(nullptr, GRLBM_ERR_CUDA, "grlbm_adjoint_create: %s", g_create_error.c_str());
    *out = owner.release();
    return GRLBM_OK;
}

void grlbm_adjoint_destroy(grlbm_adjoint *adj)
{
    if (adj)
    {
        cudaSetDevice(adj->ctx->device);
        cudaStreamSynchronize(adj->ctx->stream);
        delete adj;
    }
}

const char *grlbm_adjoint_last_error(const grlbm_adjoint *adj)
{
    return adj ? adj->err.c_str() : g_create_error.c_str();
}

int grlbm_adjoint_forward(grlbm_adjoint *adj, int32_t n_steps)
{
    if (!adj)
        return GRLBM_ERR_ARGUMENT;
    if (n_steps < 1)
        return afail(adj, GRLBM_ERR_ARGUMENT, "n_steps must be positive");
    grlbm_ctx *ctx = adj->ctx;
    cudaSetDevice(ctx->device);
    const size_t sb = (size_t)ctx->st.n * ctx->gd.nxy * sizeof(double);
    const int n_ckpt = (n_steps + adj->every - 1) / adj->every;
    while ((int)adj->ckpt.size() < n_ckpt)
    {
        adj->ckpt.emplace_back(new DevBuf);
        if (alloc(nullptr, *adj->ckpt.back(), sb))
            return afail(adj, GRLBM_ERR_CUDA, "checkpoint: %s", g_create_error.c_str());
    }
    // nodes the step never writes (halo, excision) keep the initial values in
    // every state: the recompute buffers start from the initial state
    for (auto &b : adj->seg)
        ACU(cudaMemcpyAsync(b->p, ctx->I[ctx->cur].p, sb, cudaMemcpyDeviceToDevice, ctx->stream));
    int rc;
    for (int k = 0; k < n_ckpt; k++)
    {
        ACU(cudaMemcpyAsync(adj->ckpt[k]->p, ctx->I[ctx->cur].p, sb, cudaMemcpyDeviceToDevice, ctx->stream));
        const int len = std::min(adj->every, n_steps - k * adj->every);
        if ((rc = grlbm_step_async(ctx, len)))
            return afail(adj, rc, "forward: %s", ctx->err.c_str());
    }
    ACU(cudaStreamSynchronize(ctx->stream));
    adj->n_steps = n_steps;
    return GRLBM_OK;
}

int grlbm_adjoint_backward(grlbm_adjoint *adj, const double *dL_dE, double *g_eta, double *g_kappaA,
                           double *g_kappa0)
{
    if (!adj)
        return GRLBM_ERR_ARGUMENT;
    if (!dL_dE)
        return afail(adj, GRLBM_ERR_ARGUMENT, "null dL/dE");
    if (adj->n_steps < 1)
        return afail(adj, GRLBM_ERR_STATE, "run grlbm_adjoint_forward first");
    grlbm_ctx *ctx = adj->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const bool curved = ctx->run.streaming_type == GRLBM_CURVED_FIXED;
    const int64_t nxy = ctx->gd.nxy, ncell = ctx->gd.ncell;
    const int nd = ctx->st.n;
    ACU(cudaMemcpyAsync(adj->dLdE.p, dL_dE, nxy * sizeof(double), cudaMemcpyHostToDevice, s));
    ACU(cudaMemsetAsync(adj->grads.p, 0, adj->grads.bytes, s));
    launch_adj_seed(ctx->gd, nd, ctx->w.as<double>(), ctx->flags.as<uint8_t>(), adj->dLdE.as<double>(),
                    adj->lam.as<float>(), s);
    double *g = adj->grads.as<double>();
    const int n_seg = (int)((adj->n_steps + adj->every - 1) / adj->every);
    for (int k = n_seg - 1; k >= 0; k--)
    {
        const int len = (int)std::min<int64_t>(adj->every, adj->n_steps - (int64_t)k * adj->every);
        // recompute the segment, recording clamps, cycles and first iterates
        const double *in = adj->ckpt[k]->as<double>();
        for (int jj = 0; jj < len; jj++)
        {
            PlainStepArgs a = plain_args(ctx, 0);
            a.Iin = in;
            a.Iout = adj->seg[jj]->as<double>();
            a.mom = adj->mom.as<double>();
            a.iter_sum = adj->counters.as<unsigned long long>();
            a.iter_max = reinterpret_cast<unsigned int *>(adj->counters.as<unsigned long long>() + 1);
            StepRecord rec{};
            rec.clamp = adj->clamp.as<uint8_t>() + (size_t)jj * nd * ncell;
            rec.cycles = adj->cycles.as<int>() + (size_t)jj * ncell;
            rec.e0 = adj->e0.as<double>() + (size_t)jj * ncell;
            launch_step_plain(a, curved, s, &rec);
            in = a.Iout;
        }
        ACU(cudaGetLastError());
        // adjoint steps of the segment, last first
        for (int jj = len - 1; jj >= 0; jj--)
        {
            AdjCollideArgs c{};
            c.g = ctx->gd;
            c.nd = nd;
            c.w = ctx->w.as<double>();
            c.flags = ctx->flags.as<uint8_t>();
            c.adt = ctx->cadt.as<double>();
            c.eta = ctx->ceta.as<double>();
            c.k0 = ctx->ck0.as<double>();
            c.ka = ctx->cka.as<double>();
            c.lam = adj->lam.as<float>();
            c.Iout = adj->seg[jj]->as<double>();
            c.cycles = adj->cycles.as<int>() + (size_t)jj * ncell;
            c.e0 = adj->e0.as<double>() + (size_t)jj * ncell;
            c.lamS = adj->lamS.as<float>();
            c.g_eta = g;
            c.g_ka = g + nxy;
            c.g_k0 = g + 2 * nxy;
            launch_adj_collide(c, s);
            launch_adj_stream(adj->slices.as<int64_t>(), adj->srcq, adj->coef,
                              curved ? adj->clamp.as<uint8_t>() + (size_t)jj * nd * ncell : nullptr,
                              adj->lamS.as<float>(), (int64_t)nd * nxy, adj->lam.as<float>(), s);
        }
        ACU(cudaGetLastError());
    }
    double *outs[3] = {g_eta, g_kappaA, g_kappa0};
    for (int q = 0; q < 3; q++)
        if (outs[q])
            ACU(cudaMemcpyAsync(outs[q], g + q * nxy, nxy * sizeof(double), cudaMemcpyDeviceToHost, s));
    ACU(cudaStreamSynchronize(s));
    return GRLBM_OK;
}

} // extern "C"
