// C-ABI of include/grlbm.h: context management, host<->device transfers,
// the geodesic-table build and the graph-replayed time steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/grlbm.h"
#include "approx_math.hpp"
#include "host_setup.hpp"
#include "kernels.cuh"

using namespace grlbm;

namespace
{
thread_local std::string g_create_error;

struct DevBuf
{
    void *p = nullptr;
    size_t bytes = 0;
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
    GridDev gd{};
    int64_t ncell = 0;
    int ng = 0;
    // device buffers
    DevBuf I[2], rec, w, n1, n2, cx, cy, ig_base, ig_shift, ig_w, ia3, flags, bhmask;
    DevBuf cu1, cu2, clor, cadt, ceta, ck0, ck1, cka, mom, rkf, lfp, alpha;
    DevBuf coef, ss_cx, ss_cy, ss_w, proj_basis, eval_basis, stage;
    DevBuf src_nodes, src_vals, lf_out, energy_partial, energy_out;
    DevBuf counters; // [0] iter sum (u64), [1] iter max (u32 in low), [2] rk trials (u64), [3] nonconverged, [4] clamped
    int64_t nsrc = 0;
    int cur = 0;
    bool tables = false;
    int64_t steps = 0;
    double table_ms = 0;
    // graphs of kGraphSteps steps starting from buffer 0 / 1
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    ~grlbm_ctx()
    {
        for (auto &g : graph)
            if (g)
                cudaGraphExecDestroy(g);
        if (stream)
            cudaStreamDestroy(stream);
    }
};

namespace
{
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

#define CU(call)                                                                                  \
    do                                                                                            \
    {                                                                                             \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(ctx, GRLBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));    \
    } while (0)

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

// upload doubles as the context's storage type
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

// cell-major double [ij][d] <-> direction-major T [d][ij]
template <class T>
__global__ void k_to_dirmajor(const double *in, T *out, int64_t nxy, int nd)
{
    __shared__ double tile[32][33];
    const int64_t ij0 = (int64_t)blockIdx.x * 32;
    const int d0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int64_t ij = ij0 + r;
        const int d = d0 + threadIdx.x;
        if (ij < nxy && d < nd)
            tile[r][threadIdx.x] = in[ij * nd + d];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int d = d0 + r;
        const int64_t ij = ij0 + threadIdx.x;
        if (ij < nxy && d < nd)
            out[(int64_t)d * nxy + ij] = (T)tile[threadIdx.x][r];
    }
}
template <class T>
__global__ void k_to_cellmajor(const T *in, double *out, int64_t nxy, int nd)
{
    __shared__ double tile[32][33];
    const int64_t ij0 = (int64_t)blockIdx.x * 32;
    const int d0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int d = d0 + r;
        const int64_t ij = ij0 + threadIdx.x;
        if (ij < nxy && d < nd)
            tile[threadIdx.x][r] = (double)in[(int64_t)d * nxy + ij];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int64_t ij = ij0 + r;
        const int d = d0 + threadIdx.x;
        if (ij < nxy && d < nd)
            out[ij * nd + d] = tile[r][threadIdx.x];
    }
}
template <class T>
__global__ void k_copy_convert(const T *in, double *out, int64_t n)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        out[k] = (double)in[k];
}

int64_t blocks(int64_t n, int64_t b) { return (n + b - 1) / b; }

template <class T>
StepArgs<T> step_args(grlbm_ctx *ctx, int from)
{
    StepArgs<T> a{};
    a.g = ctx->gd;
    a.nd = ctx->st.n;
    a.ng = ctx->ng;
    a.Iin = ctx->I[from].as<T>();
    a.Iout = ctx->I[from ^ 1].as<T>();
    a.rec = static_cast<decltype(a.rec)>(ctx->rec.p);
    a.w = ctx->w.as<T>();
    a.n1 = ctx->n1.as<T>();
    a.n2 = ctx->n2.as<T>();
    a.cx = ctx->cx.as<double>();
    a.cy = ctx->cy.as<double>();
    a.ig_base = ctx->ig_base.as<int>();
    a.ig_shift = ctx->ig_shift.as<int>();
    a.ig_w = ctx->ig_w.as<T>();
    a.ia3 = ctx->ia3.as<T>();
    a.flags = ctx->flags.as<uint8_t>();
    a.u1 = ctx->cu1.as<T>();
    a.u2 = ctx->cu2.as<T>();
    a.lor = ctx->clor.as<T>();
    a.adt = ctx->cadt.as<T>();
    a.eta = ctx->ceta.as<T>();
    a.k0 = ctx->ck0.as<T>();
    a.k1 = ctx->ck1.as<T>();
    a.ka = ctx->cka.as<T>();
    a.mom = ctx->mom.as<T>();
    a.iter_sum = ctx->counters.as<unsigned long long>();
    a.iter_max = reinterpret_cast<unsigned int *>(ctx->counters.as<unsigned long long>() + 1);
    return a;
}

template <class T>
size_t step_smem(const grlbm_ctx *ctx) { return (size_t)ctx->st.n * kStepBlock * sizeof(T); }

// Enqueue one step starting from buffer `from` (no sync).
template <class T>
int enqueue_step_t(grlbm_ctx *ctx, int from)
{
    if (ctx->run.keep_source_nodes_active && ctx->nsrc > 0)
    {
        const int64_t n = ctx->nsrc * ctx->st.n;
        k_sources<T><<<(unsigned)blocks(n, 256), 256, 0, ctx->stream>>>(
            ctx->I[from].as<T>(), ctx->gd.nxy, ctx->st.n, ctx->src_nodes.as<int64_t>(), ctx->src_vals.as<T>(), ctx->nsrc);
    }
    const StepArgs<T> a = step_args<T>(ctx, from);
    const unsigned nb = (unsigned)blocks(ctx->ncell, kStepBlock);
    const size_t smem = step_smem<T>(ctx);
    if (ctx->run.streaming_type == GRLBM_CURVED_FIXED)
        k_step<T, true><<<nb, kStepBlock, smem, ctx->stream>>>(a);
    else
        k_step<T, false><<<nb, kStepBlock, smem, ctx->stream>>>(a);
    CU(cudaGetLastError());
    return GRLBM_OK;
}

int enqueue_step(grlbm_ctx *ctx, int from)
{
    return ctx->fp32 ? enqueue_step_t<float>(ctx, from) : enqueue_step_t<double>(ctx, from);
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

int set_smem_limits(grlbm_ctx *ctx)
{
    const int sm = (int)(ctx->fp32 ? step_smem<float>(ctx) : step_smem<double>(ctx));
    if (ctx->fp32)
    {
        CU(cudaFuncSetAttribute(k_step<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CU(cudaFuncSetAttribute(k_step<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    }
    else
    {
        CU(cudaFuncSetAttribute(k_step<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CU(cudaFuncSetAttribute(k_step<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    }
    return GRLBM_OK;
}

// identity Fourier coefficients of the constructor (src/Radiation.cpp:59-82)
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

int32_t grlbm_metric_array_count(void) { return kMetricArrays; }

int grlbm_create(const grlbm_grid_desc *grid, const grlbm_metric_desc *metric, const grlbm_run_desc *run,
                 int32_t device, grlbm_ctx **out)
{
    grlbm_ctx *ctx = nullptr;
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
    if (run->streaming_type != GRLBM_FLAT_FIXED && run->streaming_type != GRLBM_CURVED_FIXED)
    {
        if (run->streaming_type >= GRLBM_FLAT_FIXED && run->streaming_type <= GRLBM_GEODESIC_FIXED)
            return fail(nullptr, GRLBM_ERR_UNSUPPORTED, "streaming type %d is not built (FlatFixed and CurvedFixed are)",
                        run->streaming_type);
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "Invalid StreamingType");
    }
    if (run->precision != GRLBM_PLAIN_FP64 && run->precision != GRLBM_PRECISION_FP32)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "unknown precision %d", run->precision);
    const int maxdir = run->precision == GRLBM_PLAIN_FP64 ? 216 : kMaxDirs;
    if (run->n_dir < 4 || run->n_dir > maxdir)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "n_dir must be in [4, %d]", maxdir);
    if (run->n_fourier < 1 || run->n_fourier > kMaxFourier)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "n_fourier must be in [1, %d]", kMaxFourier);
    if (run->initial_data_type != GRLBM_MOMENTS && run->initial_data_type != GRLBM_INTENSITIES)
        return fail(nullptr, GRLBM_ERR_ARGUMENT, "unknown initial data type");

    std::unique_ptr<grlbm_ctx> owner(new (std::nothrow) grlbm_ctx);
    if (!owner)
        return fail(nullptr, GRLBM_ERR_HOST, "out of host memory");
    ctx = owner.get();
    ctx->run = *run;
    ctx->mdesc = *metric;
    ctx->fp32 = run->precision == GRLBM_PRECISION_FP32;
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
#define TRY(x)                                                                     \
    do                                                                             \
    {                                                                              \
        if ((rc = (x)) != GRLBM_OK)                                                \
        {                                                                          \
            g_create_error = ctx->err;                                             \
            return rc;                                                             \
        }                                                                          \
    } while (0)

    // stencil tables.  RotationMatrix(0) applied to c_d (src/DataTypes.hh:630-635)
    const double rc0 = approx_cos(0.0), rs0 = approx_sin(0.0);
    std::vector<double> n1(nd), n2(nd);
    for (int d = 0; d < nd; d++)
    {
        n1[d] = ctx->st.cx[d] * rc0 - ctx->st.cy[d] * rs0;
        n2[d] = ctx->st.cx[d] * rs0 + ctx->st.cy[d] * rc0;
    }
    TRY(upload_t(ctx, ctx->w, ctx->st.w));
    TRY(upload_t(ctx, ctx->n1, n1));
    TRY(upload_t(ctx, ctx->n2, n2));
    TRY(upload(ctx, ctx->cx, ctx->st.cx));
    TRY(upload(ctx, ctx->cy, ctx->st.cy));
    // cubic rows: first direction and the shift to the next row's first direction
    std::vector<int> base(ctx->ng), shift(ctx->ng);
    for (int g = 0; g < ctx->ng; g++)
    {
        base[g] = (int)ctx->st.ig_index[4 * g];
        for (int k = 1; k < 4; k++)
            if (ctx->st.ig_index[4 * g + k] != (base[g] + k) % nd)
                return fail(nullptr, GRLBM_ERR_HOST, "interpolation row %d is not 4 consecutive directions", g);
    }
    for (int g = 0; g < ctx->ng; g++)
    {
        const int nb = base[(g + 1) % ctx->ng];
        shift[g] = ((nb - base[g]) % nd + nd) % nd;
        if (shift[g] > 1)
            return fail(nullptr, GRLBM_ERR_HOST, "interpolation rows %d and %d are %d directions apart", g, g + 1, shift[g]);
    }
    TRY(upload(ctx, ctx->ig_base, base));
    TRY(upload(ctx, ctx->ig_shift, shift));
    TRY(upload_t(ctx, ctx->ig_w, ctx->st.ig_weight));

    // per-node metric data
    const MetricArrays &M = ctx->M;
    std::vector<double> rkf((size_t)nxy * kRkStride, 0.0), lfp((size_t)nxy * 12), ia3(nxy), alpha(nxy);
    std::vector<uint8_t> flags(nxy), bh(nxy);
    static const int rkmap[RF_COUNT] = {ALPHA, BETA1U, BETA2U, D1ALPHA, D2ALPHA, D1BETA1LU, D1BETA2LU,
                                        D2BETA1LU, D2BETA2LU, K11L, K12L, K22L, GAM11U, GAM12U, GAM22U,
                                        D1GAM11LLL, D1GAM12LLL, D1GAM22LLL, D2GAM11LLL, D2GAM12LLL, D2GAM22LLL,
                                        TET11, TET12, TET21, TET22, ITET11, ITET12, ITET21, ITET22};
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        for (int f = 0; f < RF_COUNT; f++)
            rkf[ij * kRkStride + f] = M.at(rkmap[f], ij);
        for (int q = 0; q < 9; q++)
            lfp[ij * 12 + q] = M.at(TET00 + q, ij);
        lfp[ij * 12 + 9] = M.at(GAM11L, ij);
        lfp[ij * 12 + 10] = M.at(GAM12L, ij);
        lfp[ij * 12 + 11] = M.at(GAM22L, ij);
        const double a = M.at(ALPHA, ij);
        alpha[ij] = a;
        ia3[ij] = 1.0 / (a * a * a);
        const bool inside = M.inside_bh(G.x((double)(ij % G.nx)), G.y((double)(ij / G.nx)));
        bh[ij] = inside;
        flags[ij] = inside ? 3 : 0;
    }
    TRY(upload(ctx, ctx->rkf, rkf));
    TRY(upload(ctx, ctx->lfp, lfp));
    TRY(upload(ctx, ctx->alpha, alpha));
    TRY(upload_t(ctx, ctx->ia3, ia3));
    TRY(upload(ctx, ctx->flags, flags));
    TRY(upload(ctx, ctx->bhmask, bh));

    // streaming stencil and Fourier bases
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

    // state buffers
    const size_t ib = (size_t)nxy * nd * tsize(ctx);
    TRY(alloc(ctx, ctx->I[0], ib));
    TRY(alloc(ctx, ctx->I[1], ib));
    TRY(alloc(ctx, ctx->mom, (size_t)6 * nxy * tsize(ctx)));
    TRY(alloc(ctx, ctx->rec, (size_t)ctx->ncell * nd * (ctx->fp32 ? sizeof(float4) : sizeof(double4))));
    TRY(alloc(ctx, ctx->counters, 8 * sizeof(unsigned long long)));
    TRY(alloc(ctx, ctx->energy_partial, kPartialBlocks * sizeof(double)));
    TRY(alloc(ctx, ctx->energy_out, sizeof(double)));
    cudaMemset(ctx->I[0].p, 0, ib);
    cudaMemset(ctx->I[1].p, 0, ib);
    cudaMemset(ctx->mom.p, 0, ctx->mom.bytes);
    cudaMemset(ctx->counters.p, 0, ctx->counters.bytes);
    cudaMemset(ctx->rec.p, 0, ctx->rec.bytes);
    // fields default to zero (the reference's buffers are value-initialised)
    std::vector<double> zeros(nxy, 0.0);
    TRY(grlbm_set_fields(ctx, zeros.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data(), zeros.data()));
    TRY(set_smem_limits(ctx));
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
    if (!ctx || !kappa0 || !kappa1 || !kappaA || !eta || !ux || !uy)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null field");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->geo.nxy;
    const MetricArrays &M = ctx->M;
    std::vector<double> u1(nxy), u2(nxy), lor(nxy), adt(nxy);
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        // TransformLFtoIF(uLF, GetTetrad(ij)) as Collide calls it (src/Radiation.cpp:652-657)
        const double a = M.at(TET11, ij) * ux[ij] + M.at(TET12, ij) * uy[ij];
        const double b = M.at(TET21, ij) * ux[ij] + M.at(TET22, ij) * uy[ij];
        u1[ij] = a;
        u2[ij] = b;
        lor[ij] = 1.0 / std::sqrt(1.0 - (a * a + b * b));
        adt[ij] = M.at(ALPHA, ij) * ctx->geo.dt;
    }
    int rc;
    if ((rc = upload_t(ctx, ctx->cu1, u1)) || (rc = upload_t(ctx, ctx->cu2, u2)) || (rc = upload_t(ctx, ctx->clor, lor)) ||
        (rc = upload_t(ctx, ctx->cadt, adt)))
        return rc;
    std::vector<double> tmp(nxy);
    const double *src[4] = {eta, kappa0, kappa1, kappaA};
    DevBuf *dst[4] = {&ctx->ceta, &ctx->ck0, &ctx->ck1, &ctx->cka};
    for (int q = 0; q < 4; q++)
    {
        std::copy(src[q], src[q] + nxy, tmp.begin());
        if ((rc = upload_t(ctx, *dst[q], tmp)))
            return rc;
    }
    invalidate_graphs(ctx);
    return GRLBM_OK;
}

int grlbm_set_initial_data(grlbm_ctx *ctx, const uint8_t *is_initial, const double *initial_I, const double *E_LF,
                           const double *Fx_LF, const double *Fy_LF, const double *Pxx_LF, const double *Pxy_LF,
                           const double *Pyy_LF)
{
    if (!ctx || !is_initial)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null argument");
    if (ctx->run.initial_data_type == GRLBM_INTENSITIES && !initial_I)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "initial_I is required for InitialDataType::Intensities");
    if (ctx->run.initial_data_type == GRLBM_MOMENTS && (!E_LF || !Fx_LF || !Fy_LF || !Pxx_LF || !Pxy_LF || !Pyy_LF))
        return fail(ctx, GRLBM_ERR_ARGUMENT, "initial moments are required for InitialDataType::Moments");
    cudaSetDevice(ctx->device);
    Sources S;
    try
    {
        S = build_sources(ctx->M, ctx->st, ctx->run.initial_data_type, is_initial, initial_I, E_LF, Fx_LF, Fy_LF,
                          Pxx_LF, Pxy_LF, Pyy_LF);
    }
    catch (const std::exception &e)
    {
        return fail(ctx, GRLBM_ERR_HOST, "source set-up failed: %s", e.what());
    }
    ctx->nsrc = (int64_t)S.nodes.size();
    int rc;
    if ((rc = upload(ctx, ctx->src_nodes, S.nodes)) || (rc = upload_t(ctx, ctx->src_vals, S.intensities)))
        return rc;
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
    const int64_t n = ctx->nsrc * ctx->st.n;
    // both buffers: halo and excised nodes are read from whichever buffer is current
    for (int b = 0; b < 2; b++)
    {
        if (ctx->fp32)
            k_sources<float><<<(unsigned)blocks(n, 256), 256, 0, ctx->stream>>>(
                ctx->I[b].as<float>(), ctx->gd.nxy, ctx->st.n, ctx->src_nodes.as<int64_t>(), ctx->src_vals.as<float>(), ctx->nsrc);
        else
            k_sources<double><<<(unsigned)blocks(n, 256), 256, 0, ctx->stream>>>(
                ctx->I[b].as<double>(), ctx->gd.nxy, ctx->st.n, ctx->src_nodes.as<int64_t>(), ctx->src_vals.as<double>(), ctx->nsrc);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_set_intensity(grlbm_ctx *ctx, const double *I)
{
    if (!ctx || !I)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null argument");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    const int nd = ctx->st.n;
    int rc = alloc(ctx, ctx->stage, (size_t)nxy * nd * sizeof(double));
    if (rc)
        return rc;
    CU(cudaMemcpyAsync(ctx->stage.p, I, ctx->stage.bytes, cudaMemcpyHostToDevice, ctx->stream));
    dim3 grid((unsigned)blocks(nxy, 32), (unsigned)blocks(nd, 32)), blk(32, 8);
    for (int b = 0; b < 2; b++)
    {
        if (ctx->fp32)
            k_to_dirmajor<float><<<grid, blk, 0, ctx->stream>>>(ctx->stage.as<double>(), ctx->I[b].as<float>(), nxy, nd);
        else
            k_to_dirmajor<double><<<grid, blk, 0, ctx->stream>>>(ctx->stage.as<double>(), ctx->I[b].as<double>(), nxy, nd);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_get_intensity(grlbm_ctx *ctx, double *I)
{
    if (!ctx || !I)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "null argument");
    cudaSetDevice(ctx->device);
    const int64_t nxy = ctx->gd.nxy;
    const int nd = ctx->st.n;
    int rc = alloc(ctx, ctx->stage, (size_t)nxy * nd * sizeof(double));
    if (rc)
        return rc;
    dim3 grid((unsigned)blocks(nxy, 32), (unsigned)blocks(nd, 32)), blk(32, 8);
    if (ctx->fp32)
        k_to_cellmajor<float><<<grid, blk, 0, ctx->stream>>>(ctx->I[ctx->cur].as<float>(), ctx->stage.as<double>(), nxy, nd);
    else
        k_to_cellmajor<double><<<grid, blk, 0, ctx->stream>>>(ctx->I[ctx->cur].as<double>(), ctx->stage.as<double>(), nxy, nd);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(I, ctx->stage.p, ctx->stage.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_update_fourier_coefficients(grlbm_ctx *ctx, double rk_tol, int32_t max_substeps)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    if (!(rk_tol > 0))
        return fail(ctx, GRLBM_ERR_ARGUMENT, "rk_tol must be positive");
    cudaSetDevice(ctx->device);
    const int nf = ctx->ss.n, nd = ctx->st.n;
    const int64_t ncell = ctx->ncell;
    unsigned long long *cnt = ctx->counters.as<unsigned long long>();
    CU(cudaMemsetAsync(cnt + 2, 0, 3 * sizeof(unsigned long long), ctx->stream));
    void *data = nullptr;
    CU(cudaMallocAsync(&data, (size_t)5 * ncell * nf * sizeof(double), ctx->stream));
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
    k_geodesic<<<(unsigned)blocks(ncell * nf, 128), 128, 0, ctx->stream>>>(ga);

    ProjectArgs pa{};
    pa.g = ctx->gd;
    pa.nf = nf;
    pa.data = ga.data;
    pa.ss_w = ctx->ss_w.as<double>();
    pa.basis = ctx->proj_basis.as<double>();
    pa.coef = ctx->coef.as<double>();
    k_fourier_project<<<(unsigned)blocks(5 * ncell * nf, 128), 128, 0, ctx->stream>>>(pa);

    DepartureArgs da{};
    da.g = ctx->gd;
    da.nf = nf;
    da.nd = nd;
    da.ng = ctx->ng;
    da.coef = ctx->coef.as<double>();
    da.eval = ctx->eval_basis.as<double>();
    da.alpha = ctx->alpha.as<double>();
    da.rot_c = approx_cos(0.0);
    da.rot_s = approx_sin(0.0);
    da.rec64 = ctx->fp32 ? nullptr : ctx->rec.as<double4>();
    da.rec32 = ctx->fp32 ? ctx->rec.as<float4>() : nullptr;
    da.clamped = reinterpret_cast<int *>(cnt + 4);
    k_departure<<<(unsigned)blocks(ncell * nd, 128), 128, 0, ctx->stream>>>(da);
    cudaEventRecord(e1, ctx->stream);
    cudaError_t le = cudaGetLastError();
    cudaFreeAsync(data, ctx->stream);
    cudaError_t se = cudaStreamSynchronize(ctx->stream);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess || se != cudaSuccess)
        return fail(ctx, GRLBM_ERR_CUDA, "table build failed: %s", cudaGetErrorString(le != cudaSuccess ? le : se));
    ctx->table_ms = ms;
    ctx->tables = true;
    unsigned long long h[5];
    CU(cudaMemcpy(h, cnt, sizeof h, cudaMemcpyDeviceToHost));
    const int nonconv = (int)(unsigned)h[3];
    if (nonconv > 0)
        return fail(ctx, GRLBM_ERR_NONCONVERGED, "%d RK45 backtraces hit the substep cap", nonconv);
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
    if (!ctx || n_steps < 0)
        return fail(ctx, GRLBM_ERR_ARGUMENT, "bad step count");
    if (ctx->run.streaming_type == GRLBM_CURVED_FIXED && !ctx->tables)
        return fail(ctx, GRLBM_ERR_STATE, "curved streaming needs grlbm_update_fourier_coefficients first");
    cudaSetDevice(ctx->device);
    int rc;
    int left = n_steps;
    while (left >= kGraphSteps)
    {
        if (!ctx->graph[ctx->cur] && (rc = build_graph(ctx, ctx->cur)))
            return rc;
        CU(cudaGraphLaunch(ctx->graph[ctx->cur], ctx->stream));
        left -= kGraphSteps; // even count: the current buffer is unchanged
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

int grlbm_sync(grlbm_ctx *ctx)
{
    if (!ctx)
        return GRLBM_ERR_ARGUMENT;
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_step(grlbm_ctx *ctx, int32_t n_steps)
{
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
    int rc = alloc(ctx, ctx->lf_out, (size_t)7 * nxy * sizeof(double));
    if (rc)
        return rc;
    if (ctx->fp32)
        k_copy_convert<float><<<(unsigned)blocks(6 * nxy, 256), 256, 0, ctx->stream>>>(ctx->mom.as<float>(), ctx->lf_out.as<double>(), 6 * nxy);
    else
        k_copy_convert<double><<<(unsigned)blocks(6 * nxy, 256), 256, 0, ctx->stream>>>(ctx->mom.as<double>(), ctx->lf_out.as<double>(), 6 * nxy);
    CU(cudaGetLastError());
    for (int q = 0; q < 6; q++)
        if (dst[q])
            CU(cudaMemcpyAsync(dst[q], ctx->lf_out.as<double>() + q * nxy, nxy * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
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
        k_moments_lf<float><<<(unsigned)blocks(nxy, 256), 256, 0, ctx->stream>>>(nxy, ctx->mom.as<float>(), ctx->lfp.as<double>(), ctx->bhmask.as<uint8_t>(), ctx->lf_out.as<double>());
    else
        k_moments_lf<double><<<(unsigned)blocks(nxy, 256), 256, 0, ctx->stream>>>(nxy, ctx->mom.as<double>(), ctx->lfp.as<double>(), ctx->bhmask.as<uint8_t>(), ctx->lf_out.as<double>());
    CU(cudaGetLastError());
    double *dst[7] = {E, Fx, Fy, Pxx, Pxy, Pyy, F};
    for (int q = 0; q < 7; q++)
        if (dst[q])
            CU(cudaMemcpyAsync(dst[q], ctx->lf_out.as<double>() + q * nxy, nxy * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_energy(grlbm_ctx *ctx, double *total)
{
    if (!ctx || !total)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (ctx->fp32)
        k_energy_partial<float><<<kPartialBlocks, 256, 0, ctx->stream>>>(ctx->gd, ctx->mom.as<float>(), ctx->energy_partial.as<double>());
    else
        k_energy_partial<double><<<kPartialBlocks, 256, 0, ctx->stream>>>(ctx->gd, ctx->mom.as<double>(), ctx->energy_partial.as<double>());
    k_energy_final<<<1, 256, 0, ctx->stream>>>(ctx->energy_partial.as<double>(), kPartialBlocks, ctx->energy_out.as<double>());
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(total, ctx->energy_out.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRLBM_OK;
}

int grlbm_get_stats(grlbm_ctx *ctx, grlbm_stats *s)
{
    if (!ctx || !s)
        return GRLBM_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    unsigned long long h[5];
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaMemcpy(h, ctx->counters.p, sizeof h, cudaMemcpyDeviceToHost));
    s->steps = ctx->steps;
    s->max_iterations = (int32_t)(unsigned)(h[1] & 0xffffffffu);
    const double denom = (double)ctx->steps * (double)(ctx->geo.nx - 2) * (double)(ctx->geo.ny - 2);
    s->average_iterations = ctx->steps ? (double)h[0] / denom : 0.0;
    s->rk_substeps = (int64_t)h[2];
    s->rk_nonconverged = (int32_t)(unsigned)h[3];
    s->table_ms = ctx->table_ms;
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
