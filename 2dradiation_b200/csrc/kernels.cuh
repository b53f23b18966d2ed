// Device kernels of the radiation step.  Layouts (all in HBM, one context):
//   intensities   I[d * nxy + ij]          direction-major, two buffers
//   records       rec[d * ncell + c]       per interior cell c and direction d
//                 {ox, oy, dd, w}: departure offset in cells from the cell,
//                 interpolation-grid coordinate of the departure angle, and
//                 s^3 alpha_c^3 (0 when the departure point is excised)
//   rk fields     rkf[ij * kRkStride + f]  node-major pack of the 21 metric
//                 arrays the geodesic right-hand side reads plus the 2x2
//                 spatial blocks of the tetrad and its inverse
// The fused step kernel assigns one thread to one interior cell and loops
// over directions; its streamed intensities live in shared memory
// Is[d * kStepBlock + thread] until the lambda iteration has converged.
#pragma once
#include <cstdint>

#include "approx_math.hpp"

namespace grlbm
{
constexpr int kRkStride = 32;
enum RkField : int
{
    RF_ALPHA, RF_B1, RF_B2, RF_DA1, RF_DA2, RF_DB11, RF_DB12, RF_DB21, RF_DB22,
    RF_K11, RF_K12, RF_K22, RF_GU11, RF_GU12, RF_GU22,
    RF_DG111, RF_DG112, RF_DG122, RF_DG211, RF_DG212, RF_DG222,
    RF_T11, RF_T12, RF_T21, RF_T22, RF_TI11, RF_TI12, RF_TI21, RF_TI22,
    RF_COUNT
};
static_assert(RF_COUNT <= kRkStride, "rk pack stride");

constexpr int kStepBlock = 128;
constexpr int kMaxDirs = 256;
constexpr int kMaxFourier = 64;

struct GridDev
{
    int64_t nx, ny, nxy, nx_, ny_, ncell;
    double dx, dy, dt, startx, starty, endx, endy;
    int kind;
    double excision2;
};

__device__ __forceinline__ bool dev_outside(const GridDev &g, double x, double y)
{
    return x > g.endx || x < g.startx || y > g.endy || y < g.starty;
}
__device__ __forceinline__ bool dev_inside_bh(const GridDev &g, double x, double y)
{
    return g.kind != 0 && x * x + y * y <= g.excision2;
}

// ---------------------------------------------------------------- geodesics
struct RkLocal
{
    double alpha, b1, b2, da1, da2, db11, db12, db21, db22, k11, k12, k22, gu11, gu12, gu22;
    double dg111, dg112, dg122, dg211, dg212, dg222;
};

// Bilinear interpolation of the packed metric fields at a coordinate, with
// the flat-space values outside the domain (src/Metric.cpp:338-348, 584-780).
__device__ __forceinline__ void rk_local(const GridDev &g, const double *__restrict__ rkf, double x, double y,
                                         RkLocal &L)
{
    if (dev_outside(g, x, y))
    {
        L = RkLocal{};
        L.alpha = 1.0;
        L.gu11 = 1.0;
        L.gu22 = 1.0;
        return;
    }
    const double fi = (x - g.startx) / g.dx, fj = (y - g.starty) / g.dy;
    // a point exactly on the far boundary keeps its corners on the grid
    const int64_t i0 = min((int64_t)floor(fi), g.nx - 2), j0 = min((int64_t)floor(fj), g.ny - 2);
    const double tx = fi - (double)i0, ty = fj - (double)j0;
    const double *p00 = rkf + (i0 + j0 * g.nx) * kRkStride;
    const double *p10 = p00 + kRkStride;
    const double *p01 = p00 + g.nx * kRkStride;
    const double *p11 = p01 + kRkStride;
    double v[RF_TI22 + 1];
#pragma unroll
    for (int f = 0; f <= RF_DG222; f++)
    {
        const double f0 = __ldg(p00 + f) * (1.0 - tx) + __ldg(p10 + f) * tx;
        const double f1 = __ldg(p01 + f) * (1.0 - tx) + __ldg(p11 + f) * tx;
        v[f] = f0 * (1.0 - ty) + f1 * ty;
    }
    L.alpha = v[RF_ALPHA];
    L.b1 = v[RF_B1];
    L.b2 = v[RF_B2];
    L.da1 = v[RF_DA1];
    L.da2 = v[RF_DA2];
    L.db11 = v[RF_DB11];
    L.db12 = v[RF_DB12];
    L.db21 = v[RF_DB21];
    L.db22 = v[RF_DB22];
    L.k11 = v[RF_K11];
    L.k12 = v[RF_K12];
    L.k22 = v[RF_K22];
    L.gu11 = v[RF_GU11];
    L.gu12 = v[RF_GU12];
    L.gu22 = v[RF_GU22];
    L.dg111 = v[RF_DG111];
    L.dg112 = v[RF_DG112];
    L.dg122 = v[RF_DG122];
    L.dg211 = v[RF_DG211];
    L.dg212 = v[RF_DG212];
    L.dg222 = v[RF_DG222];
}

// 2x2 spatial block of the (inverse) tetrad at a coordinate; identity outside.
__device__ __forceinline__ void tetrad_block(const GridDev &g, const double *__restrict__ rkf, double x, double y,
                                             int first, double &a11, double &a12, double &a21, double &a22)
{
    if (dev_outside(g, x, y))
    {
        a11 = 1.0;
        a12 = 0.0;
        a21 = 0.0;
        a22 = 1.0;
        return;
    }
    const double fi = (x - g.startx) / g.dx, fj = (y - g.starty) / g.dy;
    const int64_t i0 = min((int64_t)floor(fi), g.nx - 2), j0 = min((int64_t)floor(fj), g.ny - 2);
    const double tx = fi - (double)i0, ty = fj - (double)j0;
    const double *p00 = rkf + (i0 + j0 * g.nx) * kRkStride + first;
    const double *p10 = p00 + kRkStride;
    const double *p01 = p00 + g.nx * kRkStride;
    const double *p11 = p01 + kRkStride;
    double v[4];
#pragma unroll
    for (int f = 0; f < 4; f++)
    {
        const double f0 = __ldg(p00 + f) * (1.0 - tx) + __ldg(p10 + f) * tx;
        const double f1 = __ldg(p01 + f) * (1.0 - tx) + __ldg(p11 + f) * tx;
        v[f] = f0 * (1.0 - ty) + f1 * ty;
    }
    a11 = v[0];
    a12 = v[1];
    a21 = v[2];
    a22 = v[3];
}

// 3+1 geodesic right-hand side of Vincent, Gourgoulhon & Novak (2012) as the
// reference writes it (src/GeodesicEquationSolver.cpp:5-55).
__device__ __forceinline__ void geodesic_rhs(const RkLocal &L, double nu, double v1, double v2, double &dx1,
                                             double &dx2, double &dv1, double &dv2, double &dnu)
{
    const double v[3] = {0.0, v1, v2};
    const double da[3] = {0.0, L.da1, L.da2};
    const double K[3][3] = {{0, 0, 0}, {0, L.k11, L.k12}, {0, L.k12, L.k22}};
    const double gu[3][3] = {{0, 0, 0}, {0, L.gu11, L.gu12}, {0, L.gu12, L.gu22}};
    const double db[3][3] = {{0, 0, 0}, {0, L.db11, L.db12}, {0, L.db21, L.db22}};
    // dg[i][j][k] = d_i gamma_jk
    const double dg[3][3][3] = {{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
                                {{0, 0, 0}, {0, L.dg111, L.dg112}, {0, L.dg112, L.dg122}},
                                {{0, 0, 0}, {0, L.dg211, L.dg212}, {0, L.dg212, L.dg222}}};
    double n = 0.0;
#pragma unroll
    for (int i = 1; i < 3; i++)
    {
        n -= v[i] * da[i];
#pragma unroll
        for (int j = 1; j < 3; j++)
            n += L.alpha * K[i][j] * v[i] * v[j];
    }
    dnu = n * nu;
    dx1 = L.alpha * v1 - L.b1;
    dx2 = L.alpha * v2 - L.b2;
    double dv[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 1; k < 3; k++)
    {
#pragma unroll
        for (int i = 1; i < 3; i++)
        {
            dv[k] += v[k] * da[i] * v[i] - gu[k][i] * da[i] - v[i] * db[i][k];
#pragma unroll
            for (int j = 1; j < 3; j++)
            {
                dv[k] += 2.0 * L.alpha * gu[i][k] * K[i][j] * v[j] - L.alpha * v[k] * K[i][j] * v[i] * v[j];
#pragma unroll
                for (int l = 1; l < 3; l++)
                    dv[k] -= L.alpha * 0.5 * gu[k][l] * (dg[i][l][j] + dg[j][i][l] - dg[l][i][j]) * v[i] * v[j];
            }
        }
    }
    dv1 = dv[1];
    dv2 = dv[2];
}

struct RkState
{
    double x1, x2, v1, v2, nu;
};

__device__ __forceinline__ void rk_stage(const GridDev &g, const double *__restrict__ rkf, const RkState &s,
                                         double &kx1, double &kx2, double &kv1, double &kv2, double &kn)
{
    RkLocal L;
    rk_local(g, rkf, s.x1, s.x2, L);
    geodesic_rhs(L, s.nu, s.v1, s.v2, kx1, kx2, kv1, kv2, kn);
}

// Adaptive Runge-Kutta-Fehlberg 4(5) backwards over dt with the reference's
// tableau (including its 11/44 at stage 6), absolute velocity error control
// and step update 0.95 (tol/TE)^(1/4) (src/GeodesicEquationSolver.cpp:80-188).
// Returns nu; trials counts accepted+rejected steps; a backtrace that exceeds
// max_trials stops where it is and sets capped.
__device__ double rk45_backtrace(const GridDev &g, const double *__restrict__ rkf, double tol, double dt,
                                 double &x1, double &x2, double &v1, double &v2, int max_trials, int &trials,
                                 bool &capped)
{
    const double td = -1.0;
    double nu = 1.0, total = 0.0, h = g.dt;
    trials = 0;
    capped = false;
    while (total < dt)
    {
        if (trials >= max_trials)
        {
            capped = true;
            break;
        }
        trials++;
        h = fmin(h, dt - total);
        const double s = td * h;
        RkState y0{x1, x2, v1, v2, nu}, y;
        double k1x1, k1x2, k1v1, k1v2, k1n, k2x1, k2x2, k2v1, k2v2, k2n, k3x1, k3x2, k3v1, k3v2, k3n;
        double k4x1, k4x2, k4v1, k4v2, k4n, k5x1, k5x2, k5v1, k5v2, k5n, k6x1, k6x2, k6v1, k6v2, k6n;
        rk_stage(g, rkf, y0, k1x1, k1x2, k1v1, k1v2, k1n);
        y = {x1 + s * ((1.0 / 4.0) * k1x1), x2 + s * ((1.0 / 4.0) * k1x2), v1 + s * ((1.0 / 4.0) * k1v1),
             v2 + s * ((1.0 / 4.0) * k1v2), nu + s * ((1.0 / 4.0) * k1n)};
        rk_stage(g, rkf, y, k2x1, k2x2, k2v1, k2v2, k2n);
#define GRLBM_C2(k1, k2) ((3.0 / 32.0) * k1 + (9.0 / 32.0) * k2)
        y = {x1 + s * GRLBM_C2(k1x1, k2x1), x2 + s * GRLBM_C2(k1x2, k2x2), v1 + s * GRLBM_C2(k1v1, k2v1),
             v2 + s * GRLBM_C2(k1v2, k2v2), nu + s * GRLBM_C2(k1n, k2n)};
        rk_stage(g, rkf, y, k3x1, k3x2, k3v1, k3v2, k3n);
#define GRLBM_C3(k1, k2, k3) ((1932.0 / 2197.0) * k1 - (7200.0 / 2197.0) * k2 + (7296.0 / 2197.0) * k3)
        y = {x1 + s * GRLBM_C3(k1x1, k2x1, k3x1), x2 + s * GRLBM_C3(k1x2, k2x2, k3x2),
             v1 + s * GRLBM_C3(k1v1, k2v1, k3v1), v2 + s * GRLBM_C3(k1v2, k2v2, k3v2), nu + s * GRLBM_C3(k1n, k2n, k3n)};
        rk_stage(g, rkf, y, k4x1, k4x2, k4v1, k4v2, k4n);
#define GRLBM_C4(k1, k2, k3, k4) \
    ((439.0 / 216.0) * k1 - (8.0) * k2 + (3680.0 / 513.0) * k3 - (845.0 / 4104.0) * k4)
        y = {x1 + s * GRLBM_C4(k1x1, k2x1, k3x1, k4x1), x2 + s * GRLBM_C4(k1x2, k2x2, k3x2, k4x2),
             v1 + s * GRLBM_C4(k1v1, k2v1, k3v1, k4v1), v2 + s * GRLBM_C4(k1v2, k2v2, k3v2, k4v2),
             nu + s * GRLBM_C4(k1n, k2n, k3n, k4n)};
        rk_stage(g, rkf, y, k5x1, k5x2, k5v1, k5v2, k5n);
#define GRLBM_C5(k1, k2, k3, k4, k5)                                                                          \
    (-(8.0 / 27.0) * k1 + (2.0) * k2 - (3544.0 / 2565.0) * k3 + (1859.0 / 4104.0) * k4 - (11.0 / 44.0) * k5)
        y = {x1 + s * GRLBM_C5(k1x1, k2x1, k3x1, k4x1, k5x1), x2 + s * GRLBM_C5(k1x2, k2x2, k3x2, k4x2, k5x2),
             v1 + s * GRLBM_C5(k1v1, k2v1, k3v1, k4v1, k5v1), v2 + s * GRLBM_C5(k1v2, k2v2, k3v2, k4v2, k5v2),
             nu + s * GRLBM_C5(k1n, k2n, k3n, k4n, k5n)};
        rk_stage(g, rkf, y, k6x1, k6x2, k6v1, k6v2, k6n);
#define GRLBM_C6(k1, k3, k4, k5, k6)                                                                          \
    ((16.0 / 135.0) * k1 + (6656.0 / 12825.0) * k3 + (28561.0 / 56430.0) * k4 - (9.0 / 50.0) * k5 +           \
     (2.0 / 55.0) * k6)
#define GRLBM_TE(k1, k3, k4, k5, k6)                                                                          \
    ((1.0 / 360.0) * k1 - (128.0 / 4275.0) * k3 - (2197.0 / 75240.0) * k4 + (1.0 / 50.0) * k5 +               \
     (2.0 / 55.0) * k6)
        const double e1 = h * GRLBM_TE(k1v1, k3v1, k4v1, k5v1, k6v1);
        const double e2 = h * GRLBM_TE(k1v2, k3v2, k4v2, k5v2, k6v2);
        const double te = sqrt(e1 * e1 + e2 * e2);
        if (te > tol)
        {
            h *= 0.95 * pow(tol / te, 1.0 / 4.0);
            continue;
        }
        x1 += s * GRLBM_C6(k1x1, k3x1, k4x1, k5x1, k6x1);
        x2 += s * GRLBM_C6(k1x2, k3x2, k4x2, k5x2, k6x2);
        v1 += s * GRLBM_C6(k1v1, k3v1, k4v1, k5v1, k6v1);
        v2 += s * GRLBM_C6(k1v2, k3v2, k4v2, k5v2, k6v2);
        nu += s * GRLBM_C6(k1n, k3n, k4n, k5n, k6n);
        total += h;
        h *= 0.95 * pow(tol / (te + 1e-50), 1.0 / 4.0);
        if (dev_inside_bh(g, x1, x2) || dev_outside(g, x1, x2))
            break;
#undef GRLBM_C2
#undef GRLBM_C3
#undef GRLBM_C4
#undef GRLBM_C5
#undef GRLBM_C6
#undef GRLBM_TE
    }
    return nu;
}

struct GeodesicArgs
{
    GridDev g;
    const double *rkf;      // packed metric fields
    const double *ss_cx;    // streaming stencil directions (nf)
    const double *ss_cy;
    int nf;
    double tol;
    int max_trials;
    double *data;           // out: [5][ncell][nf]: 1/s, x, y, vIF_x, vIF_y
    unsigned long long *trials_total;
    int *nonconverged;
};

// UpdateFourierCoefficients, trajectory part (src/Radiation.cpp:204-230):
// one thread per (interior cell, streaming direction).
__global__ void __launch_bounds__(128) k_geodesic(GeodesicArgs a)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = a.g.ncell * a.nf;
    int trials = 0;
    bool capped = false;
    if (tid < total)
    {
        const int64_t c = tid / a.nf;
        const int f = (int)(tid - c * a.nf);
        const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
        const int64_t ij = i + j * a.g.nx;
        double x1 = a.g.startx + (double)i * a.g.dx, x2 = a.g.starty + (double)j * a.g.dy;
        const double alpha = __ldg(a.rkf + ij * kRkStride + RF_ALPHA);
        // Vec2ObservedByEulObs<IF,LF>(alpha (1, c), xy) (src/SpecialMath.cpp:131-136)
        const double u1 = __ldg(a.ss_cx + f) * alpha, u2 = __ldg(a.ss_cy + f) * alpha;
        RkLocal L;
        rk_local(a.g, a.rkf, x1, x2, L);
        const double w1 = u1 / L.alpha, w2 = u2 / L.alpha;
        double t11, t12, t21, t22;
        tetrad_block(a.g, a.rkf, x1, x2, RF_T11, t11, t12, t21, t22);
        double v1 = t11 * w1 + t12 * w2, v2 = t21 * w1 + t22 * w2;
        double s = 1.0;
        if (!dev_inside_bh(a.g, x1, x2))
            s *= rk45_backtrace(a.g, a.rkf, a.tol, a.g.dt, x1, x2, v1, v2, a.max_trials, trials, capped);
        else
            v1 = v2 = 0.0;
        double i11, i12, i21, i22;
        tetrad_block(a.g, a.rkf, x1, x2, RF_TI11, i11, i12, i21, i22);
        const int64_t stride = a.g.ncell * a.nf;
        const int64_t o = c * a.nf + f;
        a.data[o] = 1.0 / s;
        a.data[o + stride] = x1;
        a.data[o + 2 * stride] = x2;
        a.data[o + 3 * stride] = i11 * v1 + i12 * v2;
        a.data[o + 4 * stride] = i21 * v1 + i22 * v2;
    }
    // block-aggregated counters
    __shared__ unsigned long long s_trials;
    __shared__ int s_capped;
    if (threadIdx.x == 0)
    {
        s_trials = 0;
        s_capped = 0;
    }
    __syncthreads();
    if (trials)
        atomicAdd(&s_trials, (unsigned long long)trials);
    if (capped)
        atomicAdd(&s_capped, 1);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        if (s_trials)
            atomicAdd(a.trials_total, s_trials);
        if (s_capped)
            atomicAdd(a.nonconverged, s_capped);
    }
}

struct ProjectArgs
{
    GridDev g;
    int nf;
    const double *data;   // [5][ncell][nf]
    const double *ss_w;   // nf
    const double *basis;  // [f][k]: Basis(k, phi_f)
    double *coef;         // [5][nxy][nf] (reference layout per field)
};

// Fourier::GetCoefficients for the five fields of one interior cell
// (src/FourierHarmonics.cpp:33-45): coef_k = sum_f (data_f w_f) B_k(phi_f),
// accumulated over f in order.  One thread per (cell, field, k).
__global__ void __launch_bounds__(128) k_fourier_project(ProjectArgs a)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per_field = a.g.ncell * a.nf;
    if (tid >= 5 * per_field)
        return;
    const int field = (int)(tid / per_field);
    const int64_t r = tid - field * per_field;
    const int64_t c = r / a.nf;
    const int k = (int)(r - c * a.nf);
    const double *d = a.data + field * per_field + c * a.nf;
    double acc = 0.0;
    for (int f = 0; f < a.nf; f++)
        acc += (d[f] * __ldg(a.ss_w + f)) * __ldg(a.basis + f * a.nf + k);
    const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
    a.coef[(int64_t)field * a.g.nxy * a.nf + (i + j * a.g.nx) * a.nf + k] = acc;
}

struct DepartureArgs
{
    GridDev g;
    int nf, nd, ng;
    const double *coef;     // [5][nxy][nf]
    const double *eval;     // [k][d]: Basis(k, phi_d) at the intensity directions
    const double *alpha;    // nxy
    double rot_c, rot_s;    // RotationMatrix(0) entries
    double4 *rec64;         // [nd][ncell] or null
    float4 *rec32;          // [nd][ncell] or null
    int *clamped;           // departures moved back inside the grid
};

// Departure records from the Fourier series (what StreamCurvedFixed
// evaluates every step, src/Radiation.cpp:478-499, and the angle part of
// IntensityAt, :324-328).  One thread per (direction, interior cell).
__global__ void __launch_bounds__(128) k_departure(DepartureArgs a)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= a.g.ncell * a.nd)
        return;
    const int d = (int)(tid / a.g.ncell);
    const int64_t c = tid - (int64_t)d * a.g.ncell;
    const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
    const int64_t ij = i + j * a.g.nx;
    const int64_t fs = a.g.nxy * a.nf;
    const double *cS = a.coef + ij * a.nf;
    double s = 0.0, xt = 0.0, yt = 0.0, v1 = 0.0, v2 = 0.0;
    for (int k = 0; k < a.nf; k++)
    {
        const double b = __ldg(a.eval + k * a.nd + d);
        s += cS[k] * b;
        xt += cS[k + fs] * b;
        yt += cS[k + 2 * fs] * b;
        v1 += cS[k + 3 * fs] * b;
        v2 += cS[k + 4 * fs] * b;
    }
    double4 r;
    if (dev_inside_bh(a.g, xt, yt))
    {
        r = make_double4(0.0, 0.0, 10.0 * d + 5.0, 0.0);
    }
    else
    {
        double ox = (xt - a.g.startx) / a.g.dx - (double)i;
        double oy = (yt - a.g.starty) / a.g.dy - (double)j;
        // keep the bilinear corners on the grid (nodes 0 .. n-1)
        // (0.999: still below the next node after rounding to FP32)
        const double lox = -(double)i, hix = (double)(a.g.nx - 2 - i) + 0.999;
        const double loy = -(double)j, hiy = (double)(a.g.ny - 2 - j) + 0.999;
        if (ox < lox || ox > hix || oy < loy || oy > hiy || !(ox == ox) || !(oy == oy))
        {
            atomicAdd(a.clamped, 1);
            ox = fmin(fmax(ox, lox), hix);
            oy = fmin(fmax(oy, loy), hiy);
            if (!(ox == ox))
                ox = 0.0;
            if (!(oy == oy))
                oy = 0.0;
        }
        const double w1 = v1 * a.rot_c - v2 * a.rot_s;
        const double w2 = v1 * a.rot_s + v2 * a.rot_c;
        double dd = (double)a.ng * approx_phi(w1, w2) / (2.0 * kPi);
        dd = fmin(fmax(dd, 1e-8), (double)a.ng - 1e-8);
        const double al = a.alpha[ij];
        r = make_double4(ox, oy, dd, s * (s * s) * (al * al * al));
    }
    if (a.rec64)
        a.rec64[tid] = r;
    if (a.rec32)
        a.rec32[tid] = make_float4((float)r.x, (float)r.y, (float)r.z, (float)r.w);
}

// ------------------------------------------------------------- fused step
template <typename T>
struct StepArgs
{
    GridDev g;
    int nd, ng;
    const T *Iin;
    T *Iout;
    const typename std::conditional<sizeof(T) == 8, double4, float4>::type *rec; // curved only
    const T *w;      // nd: quadrature weights
    const T *n1;     // nd: R(0) c_d
    const T *n2;
    const double *cx; // nd: stencil directions (flat departure)
    const double *cy;
    const int *ig_base;  // ng: first direction of the cubic row
    const int *ig_shift; // ng: base(g+1) - base(g) in {0, 1}
    const T *ig_w;       // ng*4
    const T *ia3;        // nxy: 1 / alpha^3
    const uint8_t *flags;// nxy: bit0 inside BH (no collide), bit1 stream writes 0
    // collide constants (nxy each)
    const T *u1, *u2, *lor, *adt, *eta, *k0, *k1, *ka;
    T *mom;              // 6 * nxy: E, Fx, Fy, Pxx, Pxy, Pyy
    unsigned long long *iter_sum;
    unsigned int *iter_max;
};

template <typename T>
struct Acc
{
    T s, c;
    __device__ __forceinline__ void zero() { s = 0; c = 0; }
};

// Sum with compensation in FP32 (Kahan); plain sum in FP64.
template <typename T>
__device__ __forceinline__ void acc_add(Acc<T> &a, T v)
{
    if constexpr (sizeof(T) == 4)
    {
        const T y = v - a.c;
        const T t = a.s + y;
        a.c = (t - a.s) - y;
        a.s = t;
    }
    else
    {
        a.s += v;
    }
}

// One time step for the interior cells of one block: StreamFlatFixed or
// StreamCurvedFixed (src/Radiation.cpp:380-414, 454-512), ComputeMomentsIF
// (:239-269) and Collide (:641-736).  Buffer semantics of the reference's
// two swaps: the stream output of excised cells is 0 and their final state is
// the old state, so the kernel writes no intensity for them; halo nodes are
// never written.
template <typename T, bool CURVED>
__global__ void __launch_bounds__(kStepBlock) k_step(StepArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Is = reinterpret_cast<T *>(smem_raw);
    const int t = threadIdx.x;
    const int64_t c = (int64_t)blockIdx.x * kStepBlock + t;
    const bool active = c < a.g.ncell;
    const int64_t cc = active ? c : 0;
    const int64_t i = 1 + cc % a.g.nx_, j = 1 + cc / a.g.nx_;
    const int64_t ij = i + j * a.g.nx;
    const int64_t nxy = a.g.nxy;
    const uint8_t fl = active ? a.flags[ij] : (uint8_t)3;
    const bool zero_stream = CURVED && (fl & 2);

    Acc<T> E, Fx, Fy, Pxx, Pxy, Pyy;
    E.zero(); Fx.zero(); Fy.zero(); Pxx.zero(); Pxy.zero(); Pyy.zero();

    for (int d = 0; d < a.nd; d++)
    {
        T val = 0;
        if (!zero_stream)
        {
            if constexpr (CURVED)
            {
                const auto r = a.rec[(int64_t)d * a.g.ncell + cc];
                if (r.w != (T)0)
                {
                    const T fli = floor(r.x), flj = floor(r.y);
                    const T fx = r.x - fli, fy = r.y - flj;
                    // corners stay on the grid whatever the record holds
                    const int64_t i0 = min(max(i + (int64_t)fli, (int64_t)0), a.g.nx - 2);
                    const int64_t j0 = min(max(j + (int64_t)flj, (int64_t)0), a.g.ny - 2);
                    const int64_t c00 = i0 + j0 * a.g.nx;
                    int g0 = (int)floor(r.z);
                    g0 = max(0, min(g0, a.ng - 1));
                    const T tt = r.z - (T)g0;
                    const int g1 = (g0 + 1 == a.ng) ? 0 : g0 + 1;
                    const int base = __ldg(a.ig_base + g0);
                    const int shift = __ldg(a.ig_shift + g0);
                    T w[5];
                    const T u = (T)1 - tt;
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        w[k] = u * __ldg(a.ig_w + 4 * g0 + k);
                    w[4] = 0;
                    // second row, aligned by its shift
                    if (shift == 0)
                    {
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            w[k] += tt * __ldg(a.ig_w + 4 * g1 + k);
                    }
                    else
                    {
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            w[k + 1] += tt * __ldg(a.ig_w + 4 * g1 + k);
                    }
                    const int ntap = 4 + shift;
                    const T *plane[5];
#pragma unroll
                    for (int k = 0; k < 5; k++)
                    {
                        int dk = base + k;
                        dk = dk >= a.nd ? dk - a.nd : dk;
                        plane[k] = a.Iin + (int64_t)dk * nxy;
                    }
                    const int64_t corner[4] = {c00, c00 + a.g.nx, c00 + 1, c00 + 1 + a.g.nx}; // 00 01 10 11
                    T cv[4];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                    {
                        T v = 0;
#pragma unroll
                        for (int k = 0; k < 5; k++)
                            if (k < ntap)
                                v += w[k] * __ldg(plane[k] + corner[q]);
                        v = v > (T)0 ? v : (T)0;
                        cv[q] = v * __ldg(a.ia3 + corner[q]);
                    }
                    const T f0 = cv[0] * ((T)1 - fx) + cv[2] * fx;
                    const T f1 = cv[1] * ((T)1 - fx) + cv[3] * fx;
                    val = r.w * (f0 * ((T)1 - fy) + f1 * fy);
                }
            }
            else
            {
                const double xt = (a.g.startx + (double)i * a.g.dx) - __ldg(a.cx + d) * a.g.dt;
                const double yt = (a.g.starty + (double)j * a.g.dy) - __ldg(a.cy + d) * a.g.dt;
                const double it = (xt - a.g.startx) / a.g.dx, jt = (yt - a.g.starty) / a.g.dy;
                const double fli = floor(it), flj = floor(jt);
                const T fx = (T)(it - fli), fy = (T)(jt - flj);
                const T *plane = a.Iin + (int64_t)d * nxy;
                const int64_t i0 = min(max((int64_t)fli, (int64_t)0), a.g.nx - 2);
                const int64_t j0 = min(max((int64_t)flj, (int64_t)0), a.g.ny - 2);
                const int64_t c00 = i0 + j0 * a.g.nx;
                const T f00 = __ldg(plane + c00), f01 = __ldg(plane + c00 + a.g.nx);
                const T f10 = __ldg(plane + c00 + 1), f11 = __ldg(plane + c00 + 1 + a.g.nx);
                const T f0 = f00 * ((T)1 - fx) + f10 * fx;
                const T f1 = f01 * ((T)1 - fx) + f11 * fx;
                val = f0 * ((T)1 - fy) + f1 * fy;
            }
        }
        Is[d * kStepBlock + t] = val;
        const T cw = __ldg(a.w + d) * val;
        const T m1 = __ldg(a.n1 + d), m2 = __ldg(a.n2 + d);
        acc_add(E, cw);
        acc_add(Fx, cw * m1);
        acc_add(Fy, cw * m2);
        acc_add(Pxx, cw * m1 * m1);
        acc_add(Pxy, cw * m1 * m2);
        acc_add(Pyy, cw * m2 * m2);
    }

    int cycles = 0;
    if (active && !(fl & 1))
    {
        const T u1 = a.u1[ij], u2 = a.u2[ij], lor = a.lor[ij], adt = a.adt[ij];
        const T eta = a.eta[ij], k0 = a.k0[ij], k1 = a.k1[ij], ka = a.ka[ij];
        const bool rest = (u1 == (T)0) && (u2 == (T)0);
        const T rden = (T)1 / ((T)1 + adt * (ka + k0));
        T diff = 1;
        T fE = 0, fFx = 0, fFy = 0;
        while (fabs(diff) > (T)1e-4 && cycles < 100)
        {
            cycles++;
            const T pE = E.s, pFx = Fx.s, pFy = Fy.s, pPxx = Pxx.s, pPxy = Pxy.s, pPyy = Pyy.s;
            const T uF = u1 * pFx + u2 * pFy;
            const T uxP = u1 * pPxx + u2 * pPxy;
            const T uyP = u1 * pPxy + u2 * pPyy;
            const T uuP = u1 * uxP + u2 * uyP;
            fE = lor * lor * (pE - (T)2 * uF + uuP);
            const T q = u1 * lor / ((T)1 + lor) * (((T)2 * lor + (T)1) * uF - lor * uuP);
            const T q2 = u2 * lor / ((T)1 + lor) * (((T)2 * lor + (T)1) * uF - lor * uuP);
            fFx = lor * lor * (pFx - lor * pE * u1 - uxP + q);
            fFy = lor * lor * (pFy - lor * pE * u2 - uyP + q2);
            const T base = k0 * fE;
            E.zero(); Fx.zero(); Fy.zero(); Pxx.zero(); Pxy.zero(); Pyy.zero();
            for (int d = 0; d < a.nd; d++)
            {
                const T m1 = __ldg(a.n1 + d), m2 = __ldg(a.n2 + d);
                T v;
                if (rest)
                {
                    const T nF = m1 * fFx + m2 * fFy;
                    const T M = base + (T)3 * k1 * nF;
                    v = (Is[d * kStepBlock + t] + adt * (eta + M)) * rden;
                }
                else
                {
                    const T un = u1 * m1 + u2 * m2;
                    const T A = lor * ((T)1 - un);
                    const T sc = ((T)1 - (lor * un) / (lor + (T)1)) * lor;
                    const T nF = ((m1 - sc * u1) / A) * fFx + ((m2 - sc * u2) / A) * fFy;
                    const T M = base + (T)3 * k1 * nF;
                    v = (Is[d * kStepBlock + t] + adt * (eta + M) / (A * A)) / ((T)1 + adt * (ka + k0) * A);
                }
                const T cw = __ldg(a.w + d) * v;
                acc_add(E, cw);
                acc_add(Fx, cw * m1);
                acc_add(Fy, cw * m2);
                acc_add(Pxx, cw * m1 * m1);
                acc_add(Pxy, cw * m1 * m2);
                acc_add(Pyy, cw * m2 * m2);
            }
            const T a1 = (pE - E.s) / E.s, a2 = (pFx - Fx.s) / Fx.s, a3 = (pFy - Fy.s) / Fy.s;
            const T a4 = (pPxx - Pxx.s) / Pxx.s, a5 = (pPxy - Pxy.s) / Pxy.s, a6 = (pPyy - Pyy.s) / Pyy.s;
            diff = sqrt(a1 * a1 + a2 * a2 + a3 * a3 + a4 * a4 + a5 * a5 + a6 * a6);
        }
        // final state: the last iterate, recomputed from the same inputs
        const T base = k0 * fE;
        for (int d = 0; d < a.nd; d++)
        {
            const T m1 = __ldg(a.n1 + d), m2 = __ldg(a.n2 + d);
            T v;
            if (rest)
            {
                const T nF = m1 * fFx + m2 * fFy;
                const T M = base + (T)3 * k1 * nF;
                v = (Is[d * kStepBlock + t] + adt * (eta + M)) * rden;
            }
            else
            {
                const T un = u1 * m1 + u2 * m2;
                const T A = lor * ((T)1 - un);
                const T sc = ((T)1 - (lor * un) / (lor + (T)1)) * lor;
                const T nF = ((m1 - sc * u1) / A) * fFx + ((m2 - sc * u2) / A) * fFy;
                const T M = base + (T)3 * k1 * nF;
                v = (Is[d * kStepBlock + t] + adt * (eta + M) / (A * A)) / ((T)1 + adt * (ka + k0) * A);
            }
            a.Iout[(int64_t)d * nxy + ij] = v;
        }
    }
    if (active)
    {
        a.mom[ij] = E.s;
        a.mom[ij + nxy] = Fx.s;
        a.mom[ij + 2 * nxy] = Fy.s;
        a.mom[ij + 3 * nxy] = Pxx.s;
        a.mom[ij + 4 * nxy] = Pxy.s;
        a.mom[ij + 5 * nxy] = Pyy.s;
    }
    // lambda-iteration statistics: block sum and max, one atomic each
    __shared__ unsigned int s_sum, s_max;
    if (t == 0)
    {
        s_sum = 0;
        s_max = 0;
    }
    __syncthreads();
    if (cycles)
    {
        atomicAdd(&s_sum, (unsigned int)cycles);
        atomicMax(&s_max, (unsigned int)cycles);
    }
    __syncthreads();
    if (t == 0 && s_sum)
    {
        atomicAdd(a.iter_sum, (unsigned long long)s_sum);
        atomicMax(a.iter_max, s_max);
    }
}

// LoadInitialData for fixed streaming: the precomputed source intensities of
// the flagged nodes (src/Radiation.cpp:138-181).
template <typename T>
__global__ void k_sources(T *I, int64_t nxy, int nd, const int64_t *nodes, const T *vals, int64_t nsrc)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nsrc * nd)
        return;
    const int64_t s = tid / nd;
    const int d = (int)(tid - s * nd);
    I[(int64_t)d * nxy + nodes[s]] = vals[tid];
}

// Radiation::ComputeMomentsLF (src/Radiation.cpp:270-301) for every node:
// T_LF^{ab} = e^a_A e^b_B T_IF^{AB}; zero inside the excision; F_LF is the
// gamma-norm of the lab-frame flux.
template <typename T>
__global__ void k_moments_lf(int64_t nxy, const T *mom, const double *lfp /* [nxy][12] */,
                             const uint8_t *bh, double *out /* 7 * nxy */)
{
    const int64_t ij = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= nxy)
        return;
    double o[7] = {0, 0, 0, 0, 0, 0, 0};
    if (!bh[ij])
    {
        const double E = mom[ij], Fx = mom[ij + nxy], Fy = mom[ij + 2 * nxy];
        const double Pxx = mom[ij + 3 * nxy], Pxy = mom[ij + 4 * nxy], Pyy = mom[ij + 5 * nxy];
        const double Tm[9] = {E, Fx, Fy, Fx, Pxx, Pxy, Fy, Pxy, Pyy};
        const double *e = lfp + ij * 12;
        double L[9];
#pragma unroll
        for (int a_ = 0; a_ < 3; a_++)
#pragma unroll
            for (int b = 0; b < 3; b++)
            {
                double s = 0.0;
#pragma unroll
                for (int A = 0; A < 3; A++)
#pragma unroll
                    for (int B = 0; B < 3; B++)
                        s += Tm[3 * A + B] * e[3 * a_ + A] * e[3 * b + B];
                L[3 * a_ + b] = s;
            }
        o[0] = L[0];
        o[1] = L[1];
        o[2] = L[2];
        o[3] = L[4];
        o[4] = L[5];
        o[5] = L[8];
        const double g11 = e[9], g12 = e[10], g22 = e[11];
        const double n2 = g11 * o[1] * o[1] + g12 * o[1] * o[2] + g12 * o[2] * o[1] + g22 * o[2] * o[2];
        o[6] = sqrt(fabs(n2));
    }
#pragma unroll
    for (int q = 0; q < 7; q++)
        out[ij + q * nxy] = o[q];
}

// Global energy, first pass: fixed-order partial sums of E over the interior
// cells, one per block (blockDim 256).
template <typename T>
__global__ void __launch_bounds__(256) k_energy_partial(GridDev g, const T *E, double *partial)
{
    __shared__ double s[256];
    const int t = threadIdx.x;
    double acc = 0.0;
    for (int64_t c = (int64_t)blockIdx.x * 256 + t; c < g.ncell; c += (int64_t)gridDim.x * 256)
    {
        const int64_t i = 1 + c % g.nx_, j = 1 + c / g.nx_;
        acc += (double)E[i + j * g.nx];
    }
    s[t] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if (t < w)
            s[t] += s[t + w];
        __syncthreads();
    }
    if (t == 0)
        partial[blockIdx.x] = s[0];
}

// Second pass: one block folds the partials in a fixed order.
__global__ void __launch_bounds__(256) k_energy_final(const double *partial, int n, double *out)
{
    __shared__ double s[256];
    const int t = threadIdx.x;
    double acc = 0.0;
    for (int k = t; k < n; k += 256)
        acc += partial[k];
    s[t] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if (t < w)
            s[t] += s[t + w];
        __syncthreads();
    }
    if (t == 0)
        *out = s[0];
}
} // namespace grlbm
