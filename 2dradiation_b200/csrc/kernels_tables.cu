// Geodesic tables (Radiation::UpdateFourierCoefficients,
// src/Radiation.cpp:191-237) and the per-(cell, direction) departure records
// derived from them.  FP64 throughout; built with -fmad=false so that each
// expression rounds exactly as the reference's CPU build does.
#include "approx_math.hpp"
#include "device_common.cuh"

namespace grlbm
{
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
    // the fields in pairs (16-byte loads; the pair after RF_DG222 is the pad)
    double v[RF_DG222 + 2];
#pragma unroll
    for (int f = 0; f <= RF_DG222; f += 2)
    {
        const double2 a00 = __ldg(reinterpret_cast<const double2 *>(p00 + f));
        const double2 a10 = __ldg(reinterpret_cast<const double2 *>(p10 + f));
        const double2 a01 = __ldg(reinterpret_cast<const double2 *>(p01 + f));
        const double2 a11 = __ldg(reinterpret_cast<const double2 *>(p11 + f));
        double f0 = a00.x * (1.0 - tx) + a10.x * tx;
        double f1 = a01.x * (1.0 - tx) + a11.x * tx;
        v[f] = f0 * (1.0 - ty) + f1 * ty;
        f0 = a00.y * (1.0 - tx) + a10.y * tx;
        f1 = a01.y * (1.0 - tx) + a11.y * tx;
        v[f + 1] = f0 * (1.0 - ty) + f1 * ty;
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
    for (int f = 0; f < 4; f += 2) // in pairs: `first` is even
    {
        const double2 a00 = __ldg(reinterpret_cast<const double2 *>(p00 + f));
        const double2 a10 = __ldg(reinterpret_cast<const double2 *>(p10 + f));
        const double2 a01 = __ldg(reinterpret_cast<const double2 *>(p01 + f));
        const double2 a11 = __ldg(reinterpret_cast<const double2 *>(p11 + f));
        double f0 = a00.x * (1.0 - tx) + a10.x * tx;
        double f1 = a01.x * (1.0 - tx) + a11.x * tx;
        v[f] = f0 * (1.0 - ty) + f1 * ty;
        f0 = a00.y * (1.0 - tx) + a10.y * tx;
        f1 = a01.y * (1.0 - tx) + a11.y * tx;
        v[f + 1] = f0 * (1.0 - ty) + f1 * ty;
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

// UpdateFourierCoefficients, trajectory part (src/Radiation.cpp:204-230):
// one thread per (interior cell, streaming direction).
// Sized for 4 resident blocks per SM (128 registers; the few spills cost
// less than the occupancy gained: 17.0 ms per 400^2 x 16 build against 19.2
// ms at 172 registers and 2 blocks, with the same coefficients).
__global__ void __launch_bounds__(128, 4) k_geodesic(GeodesicArgs a)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = a.cn * a.nf;
    int trials = 0;
    bool capped = false;
    if (tid < total)
    {
        const int64_t lc = tid / a.nf; // the cell within the built range
        const int f = (int)(tid - lc * a.nf);
        const int64_t c = a.c0 + lc;
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
        const int64_t stride = a.cn * a.nf;
        const int64_t o = lc * a.nf + f;
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

// Fourier::GetCoefficients for the five fields of one interior cell
// (src/FourierHarmonics.cpp:33-45): coef_k = sum_f (data_f w_f) B_k(phi_f),
// accumulated over f in order.  One thread per (cell, field) and kProjectK
// consecutive k, which share each product data_f w_f (the load-bound
// one-k-per-thread form issued three loads per multiply-add).
constexpr int kProjectK = 4;
__global__ void __launch_bounds__(128) k_fourier_project(ProjectArgs a)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int groups = (a.nf + kProjectK - 1) / kProjectK;
    const int64_t per_field = a.cn * groups;
    if (tid >= 5 * per_field)
        return;
    const int field = (int)(tid / per_field);
    const int64_t r = tid - field * per_field;
    const int64_t lc = r / groups; // the cell within the built range
    const int k0 = (int)(r - lc * groups) * kProjectK;
    const int64_t c = a.c0 + lc;
    const double *d = a.data + ((int64_t)field * a.cn + lc) * a.nf;
    double acc[kProjectK];
#pragma unroll
    for (int u = 0; u < kProjectK; u++)
        acc[u] = 0.0;
    for (int f = 0; f < a.nf; f++)
    {
        const double dw = d[f] * __ldg(a.ss_w + f);
        const double *b = a.basis + f * a.nf + k0;
#pragma unroll
        for (int u = 0; u < kProjectK; u++)
            if (k0 + u < a.nf)
                acc[u] += dw * __ldg(b + u);
    }
    const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
    double *out = a.coef + (int64_t)field * a.g.nxy * a.nf + (i + j * a.g.nx) * a.nf + k0;
#pragma unroll
    for (int u = 0; u < kProjectK; u++)
        if (k0 + u < a.nf)
            out[u] = acc[u];
}

// Departure records from the Fourier series: what StreamCurvedFixed
// evaluates every step (src/Radiation.cpp:478-499) and the angle part of
// IntensityAt (:324-328).  One thread per (interior cell, direction): plain
// records are written direction-major ([d * ncell + c], threads over cells
// fastest), precision records cell-major ([c * nd + d], threads over
// directions fastest).
__global__ void __launch_bounds__(128) k_departure(DepartureArgs a)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= a.cn * a.nd)
        return;
    int d;
    int64_t c, ri; // the cell, and its record's index
    if (a.rec32 || a.recf)
    {
        c = a.c0 + tid / a.nd;
        d = (int)(tid % a.nd);
        ri = c * a.nd + d;
    }
    else
    {
        d = (int)(tid / a.cn);
        c = a.c0 + (tid - (int64_t)d * a.cn);
        ri = (int64_t)d * a.g.ncell + c;
    }
    const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
    const int64_t ij = i + j * a.g.nx;
    const int64_t fs = a.g.nxy * a.nf;
    const double *cS = a.coef + ij * a.nf;
    // Fourier::GetValue (src/FourierHarmonics.cpp:56-61), summed in k order
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
    double4 r64;
    float4 r32;
    double4 sf; // the FP64 side record {i_dep - i, j_dep - j, angle coordinate, s^3 alpha_c^3}
    double dd; // angle coordinate of the departure direction
    if (dev_inside_bh(a.g, xt, yt))
    {
        r64 = make_double4((double)i, (double)j, -1.0, 0.0);
        dd = 10.0 * d + 5.0;
        r32 = make_float4(0.f, 0.f, (float)dd, 0.f);
        sf = make_double4(0.0, 0.0, dd, 0.0);
    }
    else
    {
        const double it = (xt - a.g.startx) / a.g.dx;
        const double jt = (yt - a.g.starty) / a.g.dy;
        if (!(it >= 0.0 && it < (double)(a.g.nx - 1) && jt >= 0.0 && jt < (double)(a.g.ny - 1)))
            atomicAdd(a.clamped, 1);
        if (jt == jt)
        {
            // node rows the bilinear gather reads, relative to the cell (a slab's ghost depth)
            const double jf = floor(jt) - (double)j;
            const double ext = fmax(fabs(jf), fabs(jf + 1.0));
            atomicMax(a.row_extent, ext < 1e9 ? (int)ext : 1000000000);
        }
        // RotationMatrix(0).Inverse() * v (src/DataTypes.hh:625-635)
        const double w1 = v1 * a.rot_c - v2 * a.rot_s;
        const double w2 = v1 * a.rot_s + v2 * a.rot_c;
        // InterpolationGrid::d (src/Stencil.cpp:35-38)
        dd = (double)a.ng * approx_phi(w1, w2) / (2.0 * kPi);
        dd = dd < 1e-8 ? 1e-8 : (dd > (double)a.ng - 1e-8 ? (double)a.ng - 1e-8 : dd);
        const double s3 = s * (s * s);
        r64 = make_double4(it, jt, dd, s3);
        // FP32 side record: offsets kept on the grid, alpha_c^3 folded in
        double ox = it - (double)i, oy = jt - (double)j;
        const double lox = -(double)i, hix = (double)(a.g.nx - 2 - i) + 0.999;
        const double loy = -(double)j, hiy = (double)(a.g.ny - 2 - j) + 0.999;
        ox = ox < lox ? lox : (ox > hix ? hix : ox);
        oy = oy < loy ? loy : (oy > hiy ? hiy : oy);
        if (!(ox == ox))
            ox = 0.0;
        if (!(oy == oy))
            oy = 0.0;
        const double al = a.alpha[ij];
        const double s3a3 = s3 * (al * al * al);
        r32 = make_float4((float)ox, (float)oy, (float)dd, (float)s3a3);
        sf = make_double4(ox, oy, dd, s3a3);
    }
    if (a.rec32)
    {
        // packed record (packed32): row type, window start and blend; the
        // corner in the fractions' sign bits, far in the scale's
        const double fxd = floor((double)r32.x), fyd = floor((double)r32.y);
        const bool near = (fxd == -1.0 || fxd == 0.0) && (fyd == -1.0 || fyd == 0.0);
        double ddc = dd == dd ? dd : 0.0;
        int g = (int)floor(ddc);
        g = g < 0 ? 0 : (g > a.ng - 1 ? a.ng - 1 : g);
        double t = ddc - (double)g;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        const int rt = g % a.q, m = g / a.q;
        const unsigned start = (unsigned)((a.row_base[rt] + a.p * m) % a.nd);
        unsigned tq = (unsigned)(t * (double)(1u << packed32::kTBits) + 0.5);
        tq = tq > (1u << packed32::kTBits) - 1u ? (1u << packed32::kTBits) - 1u : tq;
        const unsigned word = tq | ((unsigned)rt << packed32::kTypeShift) | (start << packed32::kStartShift);
        const float fx = near ? (float)((double)r32.x - fxd) : 0.f, fy = near ? (float)((double)r32.y - fyd) : 0.f;
        const unsigned ux = __float_as_uint(fx) | (near && fxd == 0.0 ? 0x80000000u : 0u);
        const unsigned uy = __float_as_uint(fy) | (near && fyd == 0.0 ? 0x80000000u : 0u);
        const unsigned uw = __float_as_uint(r32.w) | (near ? 0u : 0x80000000u);
        a.rec32[ri] = make_uint4(word, ux, uy, uw);
        if (!near && a.far)
            atomicAdd(a.far, 1ull);
        a.side32[ri] = r32;
    }
    if (a.recf)
    {
        // packed64 record: the fractions, blend and window of the FP64 side
        // record, with the corner, row type, window start and far flag in the
        // spare bits of 1 + f
        const double fxd = floor(sf.x), fyd = floor(sf.y);
        const bool near = (fxd == -1.0 || fxd == 0.0) && (fyd == -1.0 || fyd == 0.0);
        double ddc = dd == dd ? dd : 0.0;
        int g = (int)floor(ddc);
        g = g < 0 ? 0 : (g > a.ng - 1 ? a.ng - 1 : g);
        double t = ddc - (double)g;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        const int rt = g % a.q, m = g / a.q;
        const unsigned start = (unsigned)((a.row_base[rt] + a.p * m) % a.nd);
        // 1 + f in [1, 2): a value that rounds up to 2 is kept just below it
        auto biased = [](double f, unsigned payload) {
            double v = 1.0 + f;
            if (!(v < 2.0))
                v = 1.9999999999999998;
            const unsigned long long b = (unsigned long long)__double_as_longlong(v);
            const unsigned hi = ((unsigned)(b >> 32) & packed64::kMantHi) | payload;
            return __hiloint2double((int)hi, (int)(unsigned)b);
        };
        const double fx = near ? sf.x - fxd : 0.0, fy = near ? sf.y - fyd : 0.0;
        const unsigned cx = near && fxd == 0.0 ? 0x80000000u : 0u, cy = near && fyd == 0.0 ? 0x80000000u : 0u;
        double4 rf;
        rf.x = biased(fx, cx | ((unsigned)rt << packed64::kExpShift));
        rf.y = biased(fy, cy);
        rf.z = biased(t, start << packed64::kExpShift);
        rf.w = near ? sf.w : __hiloint2double((int)((unsigned)__double2hiint(sf.w) | 0x80000000u), __double2loint(sf.w));
        a.recf[ri] = rf;
        if (!near && a.far)
            atomicAdd(a.far, 1ull);
        a.sidef[ri] = sf;
    }
    if (a.rec64)
        a.rec64[ri] = r64;
}

// (alpha_ij / alpha_n)^3 for the 3x3 neighbours n of each interior node, as
// IntegerPow<3>(alpha / metric.GetAlpha(corner)) (src/Radiation.cpp:502-505).
__global__ void k_alpha_cube(GridDev g, const double *alpha, double *acube)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.ncell)
        return;
    const int64_t i = 1 + c % g.nx_, j = 1 + c / g.nx_;
    const int64_t ij = i + j * g.nx;
    const double al = alpha[ij];
    for (int dj = -1; dj <= 1; dj++)
        for (int di = -1; di <= 1; di++)
        {
            const double r = al / alpha[ij + di + dj * g.nx];
            acube[ij * 9 + 3 * (dj + 1) + (di + 1)] = r * (r * r);
        }
}

static inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

void launch_geodesic(const GeodesicArgs &a, cudaStream_t s)
{
    k_geodesic<<<nblk(a.cn * a.nf, 128), 128, 0, s>>>(a);
}
void launch_project(const ProjectArgs &a, cudaStream_t s)
{
    k_fourier_project<<<nblk(5 * a.cn * ((a.nf + kProjectK - 1) / kProjectK), 128), 128, 0, s>>>(a);
}
void launch_departure(const DepartureArgs &a, cudaStream_t s)
{
    k_departure<<<nblk(a.cn * a.nd, 128), 128, 0, s>>>(a);
}
void launch_alpha_cube(const GridDev &g, const double *alpha, double *acube, cudaStream_t s)
{
    k_alpha_cube<<<nblk(g.ncell, 128), 128, 0, s>>>(g, alpha, acube);
}
} // namespace grlbm
