/* grlbm_oracle.c -- CPU restatement of Tom-Olsen/2dRadiation's radiation step.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg load it (through oracle/oracle.py).  The
 * product library neither links nor calls anything in this directory.
 *
 * It restates, in plain C with IEEE FP64 arithmetic (built with
 * -ffp-contract=off, no fast-math), every function on the reference's
 * GR lattice-Boltzmann step:
 *   set-up   : polynomial trig (src/Utility.hh:128-471), Stencil and its cubic
 *              interpolation grid (src/Stencil.cpp:4-200), flux->sigma look-up
 *              tables (src/Stencil.cpp:378-455, src/DataTypes.hh:637-701),
 *              Grid (src/Grid.cpp:4-107), metric arrays of the three
 *              spacetimes (src/Metric.cpp:126-336, src/Spacetimes.cpp);
 *   tables   : RK45 geodesic backtrace + Fourier projection
 *              (src/Radiation.cpp:191-237, src/GeodesicEquationSolver.cpp:5-188,
 *              src/FourierHarmonics.cpp:5-61);
 *   step     : LoadInitialData (src/Radiation.cpp:103-182), StreamFlatFixed
 *              (:380-414), StreamCurvedFixed (:454-512) with IntensityAt
 *              (:322-343), ComputeMomentsIF (:239-269), Collide (:641-736),
 *              ComputeMomentsLF (:270-301), in the order of the time loop
 *              (:745-832).
 * Every expression keeps the reference's association order, so that with the
 * same compiler semantics it reproduces the reference bit for bit; this is
 * checked against the reference itself (oracle/_ref, strict build) by
 * tests/test_oracle_golden.py and against committed golden vectors.
 *
 * Parity is pinned to the reference compiled with a project-written stand-in
 * for its un-vendored Eigen submodule (oracle/eigen_standin); the 3x3 inverse
 * below (inv3) follows that stand-in.  Parity against real Eigen is not pinned.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "ref_api.h"

#define PI 3.14159265358979323846
#define PI_2 1.57079632679489661923

/* ------------------------------------------------------------------ trig */
/* MyAtan<9> (src/Utility.hh:179-188) */
static double my_atan9(double z)
{
    const double a1 = 0.9998660, a3 = -0.3302995, a5 = 0.1801410, a7 = -0.0851330, a9 = 0.0208351;
    double zz = z * z;
    return z * (a1 + zz * (a3 + zz * (a5 + zz * (a7 + zz * a9))));
}
/* MyAtan2<9> (src/Utility.hh:220-254); branch choice compares |x|,|y| as floats */
static double my_atan2(double y, double x)
{
    if (x != 0.0)
    {
        if (fabsf((float)x) > fabsf((float)y))
        {
            const double z = y / x;
            if (x > 0.0)
                return my_atan9(z);
            else if (y >= 0.0)
                return my_atan9(z) + PI;
            else
                return my_atan9(z) - PI;
        }
        else
        {
            const double z = x / y;
            if (y > 0.0)
                return -my_atan9(z) + PI_2;
            else
                return -my_atan9(z) - PI_2;
        }
    }
    else
    {
        if (y > 0.0)
            return PI_2;
        else if (y < 0.0)
            return -PI_2;
    }
    return 0.0;
}
/* Tensor2::Phi (src/DataTypes.hh:166-170) */
static double phi_of(double x, double y)
{
    double phi = my_atan2(y, x);
    return (phi < 0) ? phi + 2.0 * PI : phi;
}
/* MySin<9> (src/Utility.hh:272-323); inputs outside [-pi/2, 5pi/2] abort in
 * the reference (ExitOnError); here they return NAN. */
static double my_sin(double x)
{
    if (-PI_2 <= x && x <= PI_2)
    {
    }
    else if (PI_2 <= x && x <= 3.0 * PI_2)
        x = -(x - PI);
    else if (3.0 * PI_2 <= x && x <= 5.0 * PI_2)
        x = x - 2.0 * PI;
    else
        return NAN;
    x *= 2.0 / PI;
    const double a1 = 1.57079631847, a3 = -0.64596371106, a5 = 0.07968967928, a7 = -0.00467376557,
                 a9 = 0.00015148419;
    double xx = x * x;
    return x * (a1 + xx * (a3 + xx * (a5 + xx * (a7 + xx * a9))));
}
/* MyCos<9>(float) (src/Utility.hh:340-349): float argument and result */
static float my_cos_f(float x)
{
    const float pi = (float)PI;
    const float pi_2 = (float)PI_2;
    if (x >= pi)
        return (float)(-my_sin((double)(x - pi_2)));
    else
        return (float)my_sin((double)(x + pi_2));
}
/* MyCos(double) (src/Utility.hh:353-360) */
static double my_cos(double x) { return (double)my_cos_f((float)x); }
/* MyAsin<4> (src/Utility.hh:366-395).  At its definition the unqualified
 * `abs(x)` (src/Utility.hh:374) binds to the C library's int abs(int): the
 * argument is truncated to an integer, so |x| < 1 becomes 0.  Reproduced. */
static double my_asin4(double x)
{
    double sign = (double)((0.0 < x) - (x < 0.0));
    x = (double)abs((int)x);
    const double a0 = 1.57078786, a1 = -0.21412453, a2 = 0.08466649, a3 = -0.03575663, a4 = 0.00864884;
    double polynome = a0 + x * (a1 + x * (a2 + x * (a3 + x * a4)));
    return sign * (PI_2 - sqrt(1.0 - x) * polynome);
}
/* MyAcos<4>(float) (src/Utility.hh:453-471) */
static double my_acos(double xd)
{
    float x = (float)xd;
    float r;
    if (x >= 0)
        r = (float)(PI_2 - my_asin4((double)x));
    else
        r = (float)(PI_2 + my_asin4((double)(-x)));
    return (double)r;
}
/* RotationMatrix(0) * v (src/DataTypes.hh:620-635): the cosine of the zero
 * rotation is the float polynomial value, not 1. */
static double rot0_cos(void) { return my_cos(0.0); }
static double rot0_sin(void) { return my_sin(0.0); }

/* ------------------------------------------------------------ 3x3 inverse */
/* adjugate / determinant in the fixed order of oracle/eigen_standin */
static void inv3(const double *m, double *r)
{
    const double c00 = m[4] * m[8] - m[5] * m[7];
    const double c01 = m[5] * m[6] - m[3] * m[8];
    const double c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    const double inv = 1.0 / det;
    r[0] = c00 * inv;
    r[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
    r[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    r[3] = c01 * inv;
    r[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    r[6] = c02 * inv;
    r[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
}

/* ------------------------------------------------------------------ grid */
typedef struct
{
    int64_t nx, ny, nxy;
    double dx, dy, dt, startx, starty, endx, endy;
} Grid;

/* Grid(nx_, ny_, start, end, halo=1) + SetCFL (src/Grid.cpp:4-37) */
static Grid grid_make(const grlbm_ref_params *p)
{
    Grid g;
    const int halo = 1;
    g.nx = p->nx_ + 2 * halo;
    g.ny = p->ny_ + 2 * halo;
    g.nxy = g.nx * g.ny;
    g.dx = (p->endx - p->startx) / ((double)g.nx - 1.0 - 2.0 * halo);
    g.dy = (p->endy - p->starty) / ((double)g.ny - 1.0 - 2.0 * halo);
    g.startx = p->startx - g.dx;
    g.starty = p->starty - g.dy;
    g.endx = p->endx + g.dx;
    g.endy = p->endy + g.dy;
    g.dt = p->cfl * (g.dx < g.dy ? g.dx : g.dy);
    return g;
}
static double gx(const Grid *g, double i) { return g->startx + i * g->dx; }
static double gy(const Grid *g, double j) { return g->starty + j * g->dy; }
static double gi(const Grid *g, double x) { return (x - g->startx) / g->dx; }
static double gj(const Grid *g, double y) { return (y - g->starty) / g->dy; }
/* Grid::OutsideDomain(Coord) (src/Grid.cpp:98-102) */
static int outside(const Grid *g, double x, double y)
{
    return x > g->endx || x < g->startx || y > g->endy || y < g->starty;
}

/* --------------------------------------------------------------- stencil */
typedef struct
{
    int n;
    double *w, *phi, *cx, *cy;
    /* cubic interpolation grid (nGrid = 10 n) */
    int ng;
    int64_t *idx; /* 4 per row */
    double *wt;   /* 4 per row */
    /* flux -> sigma / normalization look-up tables */
    int nlut;
    double *lut_in, *lut_sigma, *lut_norm;
} Stencil;

/* Stencil(nOrder, nGhost=0) directions (src/Stencil.cpp:188-200) */
static void stencil_dirs(Stencil *s, int n)
{
    s->n = n;
    s->w = malloc(sizeof(double) * n);
    s->phi = malloc(sizeof(double) * n);
    s->cx = malloc(sizeof(double) * n);
    s->cy = malloc(sizeof(double) * n);
    for (int d = 0; d < n; d++)
    {
        s->w[d] = 1.0 / (double)n;
        s->phi[d] = 2.0 * PI * (d + 0.5) / (double)n;
        s->cx[d] = my_cos(s->phi[d]);
        s->cy[d] = my_sin(s->phi[d]);
    }
}

/* InterpolationGrid::NeighbourIndexesCubic / LagrangeWeightsCubic
 * (src/Stencil.cpp:109-162) */
static void interp_row(const Stencil *s, double phi, int64_t *idx, double *wt)
{
    int index = -1;
    double minDist = 10;
    for (int d = 0; d < s->n; d++)
    {
        double delta = fabs(phi - s->phi[d]);
        double alt = 2.0 * PI - delta;
        double dist = delta < alt ? delta : alt;
        if (dist < minDist)
        {
            minDist = dist;
            index = d;
        }
    }
    double phiMin = fmod(s->phi[index] + PI - phi, 2.0 * PI);
    const int64_t n = s->n;
    if (phiMin < PI)
    {
        idx[0] = (index - 1 + n) % n;
        idx[1] = (index + 0 + n) % n;
        idx[2] = (index + 1 + n) % n;
        idx[3] = (index + 2 + n) % n;
    }
    else
    {
        idx[0] = (index - 2 + n) % n;
        idx[1] = (index - 1 + n) % n;
        idx[2] = (index + 0 + n) % n;
        idx[3] = (index + 1 + n) % n;
    }
    for (int i = 0; i < 4; i++)
    {
        double weight = 1;
        double phi_i = fmod(s->phi[idx[i]] + PI - phi + 2.0 * PI, 2.0 * PI);
        for (int j = 0; j < 4; j++)
        {
            double phi_j = fmod(s->phi[idx[j]] + PI - phi + 2.0 * PI, 2.0 * PI);
            if (i != j)
                weight *= (PI - phi_j) / (phi_i - phi_j);
        }
        wt[i] = weight;
    }
}

/* LookUpTable<double>::Add (src/DataTypes.hh:644-670) on parallel arrays */
static void lut_add(Stencil *s, int *cap, double in, double sigma, double norm)
{
    int n = s->nlut;
    int pos;
    if (n == 0 || in < s->lut_in[0])
        pos = 0;
    else if (in > s->lut_in[n - 1])
        pos = n;
    else
    {
        int lo = 0, hi = n; /* lower_bound */
        while (lo < hi)
        {
            int mid = (lo + hi) / 2;
            if (s->lut_in[mid] < in)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo == n || in < s->lut_in[lo])
            pos = lo;
        else
            return;
    }
    if (n + 1 > *cap)
    {
        *cap = *cap ? 2 * *cap : 64;
        s->lut_in = realloc(s->lut_in, sizeof(double) * *cap);
        s->lut_sigma = realloc(s->lut_sigma, sizeof(double) * *cap);
        s->lut_norm = realloc(s->lut_norm, sizeof(double) * *cap);
    }
    memmove(s->lut_in + pos + 1, s->lut_in + pos, sizeof(double) * (n - pos));
    memmove(s->lut_sigma + pos + 1, s->lut_sigma + pos, sizeof(double) * (n - pos));
    memmove(s->lut_norm + pos + 1, s->lut_norm + pos, sizeof(double) * (n - pos));
    s->lut_in[pos] = in;
    s->lut_sigma[pos] = sigma;
    s->lut_norm[pos] = norm;
    s->nlut = n + 1;
}
/* LookUpTable<double>::Evaluate (src/DataTypes.hh:672-701) */
static double lut_eval(const double *in, const double *out, int size, double x)
{
    if (x <= in[0] || size == 1)
        return out[0];
    if (x >= in[size - 1])
        return out[size - 1];
    int lo = 0, hi = size;
    while (lo < hi)
    {
        int mid = (lo + hi) / 2;
        if (in[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    int i0 = lo - 1, i1 = lo;
    if (in[i0] == x)
        return out[i0];
    double t = (x - in[i0]) / (in[i1] - in[i0]);
    return out[i0] + t * (out[i1] - out[i0]);
}

/* Stencil::PopulateLookUpTable (src/Stencil.cpp:378-455); the reference loop
 * is unbounded, this one stops after 10^6 passes. */
static void stencil_lut(Stencil *s)
{
    const double deltaPhi = PI / 8.0 + 1e-8;
    const double maxInterpolationError = 0.01;
    double E = 1.0, Fx = 1, Fy = 0;
    double *I = malloc(sizeof(double) * s->n);
    double sigma = 0, currentF = 0, refinement = 1;
    int cap = 0;
    for (long pass = 0; pass < 1000000; pass++)
    {
        double normalization = 0;
        for (int d = 0; d < s->n; d++)
            normalization += s->w[d] * exp(sigma * (Fx * s->cx[d] + Fy * s->cy[d]));
        normalization = log(normalization);
        double cE = 0, cFx = 0, cFy = 0;
        for (int d = 0; d < s->n; d++)
        {
            I[d] = E * exp(sigma * (Fx * s->cx[d] + Fy * s->cy[d]) - normalization);
            double c = s->w[d] * I[d];
            cE += c;
            cFx += c * s->cx[d];
            cFy += c * s->cy[d];
        }
        currentF = sqrt(cFx * cFx + cFy * cFy);
        double averageError = 0;
        int count = 0;
        for (int g = 0; g < s->ng; g++)
        {
            double gphi = 2.0 * PI * g / (double)s->ng;
            double gcx = my_cos(gphi), gcy = my_sin(gphi);
            if (my_acos(Fx * gcx + Fy * gcy) > deltaPhi / 2.0)
                continue;
            double analyticValue = E * exp(sigma * (Fx * gcx + Fy * gcy) - normalization);
            double interp = 0;
            for (int p = 0; p < 4; p++)
                interp += s->wt[4 * g + p] * I[s->idx[4 * g + p]];
            double error = fabs((analyticValue - interp) / analyticValue);
            averageError += error;
            count++;
        }
        averageError /= count;
        if (averageError > maxInterpolationError)
        {
            sigma -= pow(10, -refinement);
            refinement++;
            sigma += pow(10, -refinement);
            if (refinement >= 8)
                break;
        }
        else
        {
            lut_add(s, &cap, currentF, sigma, normalization);
            /* the normalization table is filled by the same Add() calls with
             * the same inputs, so it shares the input column */
            sigma += pow(10, -refinement);
        }
    }
    free(I);
}

static void stencil_make(Stencil *s, int n, int intensity)
{
    memset(s, 0, sizeof(*s));
    stencil_dirs(s, n);
    s->ng = intensity ? 10 * n : 3;
    s->idx = malloc(sizeof(int64_t) * 4 * s->ng);
    s->wt = malloc(sizeof(double) * 4 * s->ng);
    for (int g = 0; g < s->ng; g++)
    {
        double phi = 2.0 * PI * g / (double)s->ng;
        interp_row(s, phi, s->idx + 4 * g, s->wt + 4 * g);
    }
    if (intensity)
        stencil_lut(s);
}
static void stencil_free(Stencil *s)
{
    free(s->w);
    free(s->phi);
    free(s->cx);
    free(s->cy);
    free(s->idx);
    free(s->wt);
    free(s->lut_in);
    free(s->lut_sigma);
    free(s->lut_norm);
}

/* ---------------------------------------------------------------- metric */
enum
{
    G00L, G00U, G01L, G01U, G02L, G02U, G11L, G11U, G12L, G12U, G22L, G22U,
    D0G00L, D1G00L, D2G00L, D0G01L, D1G01L, D2G01L, D0G02L, D1G02L, D2G02L,
    D0G11L, D1G11L, D2G11L, D0G12L, D1G12L, D2G12L, D0G22L, D1G22L, D2G22L,
    D0G00U, D1G00U, D2G00U, D0G01U, D1G01U, D2G01U, D0G02U, D1G02U, D2G02U,
    D0G11U, D1G11U, D2G11U, D0G12U, D1G12U, D2G12U, D0G22U, D1G22U, D2G22U,
    ALPHA, BETA1U, BETA1L, BETA2U, BETA2L, GAM11L, GAM11U, GAM12L, GAM12U, GAM22L, GAM22U,
    D1ALPHA, D2ALPHA, D1BETA1LU, D1BETA2LU, D2BETA1LU, D2BETA2LU,
    D1BETA1LL, D1BETA2LL, D2BETA1LL, D2BETA2LL,
    D1GAM11LLL, D2GAM11LLL, D1GAM12LLL, D2GAM12LLL, D1GAM22LLL, D2GAM22LLL,
    D1GAM11LUU, D2GAM11LUU, D1GAM12LUU, D2GAM12LUU, D1GAM22LUU, D2GAM22LUU,
    K11, K12, K22,
    T00, T01, T02, T10, T11, T12, T20, T21, T22,
    TI00, TI01, TI02, TI10, TI11, TI12, TI20, TI21, TI22,
    NMETRIC
};
_Static_assert(NMETRIC == GRLBM_N_METRIC_ARRAYS, "metric array count");

typedef struct
{
    int kind;
    double m, a, excision2;
    Grid g;
    double *arr; /* NMETRIC * nxy */
} Metric;

#define MA(M, k, ij) ((M)->arr[(size_t)(k) * (M)->g.nxy + (ij)])

/* MetricFunction of Minkowski / SchwarzSchild / KerrSchild
 * (src/Spacetimes.cpp:21-24, 48-64, 87-112); row-major 3x3 */
static void metric_function(const Metric *M, double x, double y, double *g)
{
    for (int k = 0; k < 9; k++)
        g[k] = 0.0;
    g[0] = -1;
    g[4] = 1;
    g[8] = 1;
    if (M->kind == 1)
    {
        double rs = 2.0 * M->m;
        double r2 = x * x + y * y;
        double r = sqrt(r2);
        if (r > 2.0 * M->m)
        {
            g[0] = -1.0 + rs / r;
            g[4] = x * x / (r2 - rs * r) + y * y / r2;
            g[8] = x * x / r2 + y * y / (r2 - rs * r);
            g[5] = g[7] = rs * x * y / (r2 * (r - rs));
        }
    }
    else if (M->kind == 2)
    {
        double a2 = M->a * M->a;
        double R2 = x * x + y * y;
        if (R2 > a2)
        {
            double r2 = R2 - a2;
            double r = sqrt(r2);
            double rho2 = r2 + a2;
            double H = M->m / r;
            double l[3] = {1, (r * x + M->a * y) / rho2, (r * y - M->a * x) / rho2};
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                {
                    if (i == 0 && j == 0)
                        g[3 * i + j] = -1.0 + 2.0 * H * l[i] * l[j];
                    else
                        g[3 * i + j] = (double)(i == j) + 2.0 * H * l[i] * l[j];
                }
        }
    }
}
/* InsideBH (src/Spacetimes.cpp:16-19, 38-42, 78-81) */
static int inside_bh(const Metric *M, double x, double y)
{
    if (M->kind == 0)
        return 0;
    return x * x + y * y <= M->excision2;
}

/* Metric::MetricDeriv<k> / InverseMetricDeriv<k> (src/Metric.cpp:189-219) */
static void metric_deriv(const Metric *M, int k, double x, double y, int inverse, double *out)
{
    const double dk = 1e-8;
    double gm2[9], gm1[9], gp1[9], gp2[9], t[9];
    double ex = (k == 1), ey = (k == 2);
    metric_function(M, x - 2 * dk * ex, y - 2 * dk * ey, gm2);
    metric_function(M, x - 1 * dk * ex, y - 1 * dk * ey, gm1);
    metric_function(M, x + 1 * dk * ex, y + 1 * dk * ey, gp1);
    metric_function(M, x + 2 * dk * ex, y + 2 * dk * ey, gp2);
    if (inverse)
    {
        inv3(gm2, t);
        memcpy(gm2, t, sizeof t);
        inv3(gm1, t);
        memcpy(gm1, t, sizeof t);
        inv3(gp1, t);
        memcpy(gp1, t, sizeof t);
        inv3(gp2, t);
        memcpy(gp2, t, sizeof t);
    }
    for (int q = 0; q < 9; q++)
        out[q] = (1.0 / 12.0 * gm2[q] - 1 / 12.0 * gp2[q] - 2.0 / 3.0 * gm1[q] + 2.0 / 3.0 * gp1[q]) / dk;
}

static void metric_build(Metric *M, const grlbm_ref_params *p, const Grid *g)
{
    M->kind = p->metric_kind;
    M->m = p->m;
    M->a = p->a;
    double rex = p->excision > 0 ? p->excision : 2.1;
    M->excision2 = rex * rex * M->m * M->m;
    M->g = *g;
    const int64_t nx = g->nx, ny = g->ny, nxy = g->nxy;
    M->arr = calloc((size_t)NMETRIC * nxy, sizeof(double));
    /* InitializeMetricOnGrid (src/Metric.cpp:126-150) */
#pragma omp parallel for collapse(2)
    for (int64_t j = 0; j < ny; j++)
        for (int64_t i = 0; i < nx; i++)
        {
            double gl[9], gu[9];
            metric_function(M, gx(g, (double)i), gy(g, (double)j), gl);
            inv3(gl, gu);
            int64_t ij = i + j * nx;
            MA(M, G00L, ij) = gl[0];
            MA(M, G00U, ij) = gu[0];
            MA(M, G01L, ij) = gl[1];
            MA(M, G01U, ij) = gu[1];
            MA(M, G02L, ij) = gl[2];
            MA(M, G02U, ij) = gu[2];
            MA(M, G11L, ij) = gl[4];
            MA(M, G11U, ij) = gu[4];
            MA(M, G12L, ij) = gl[5];
            MA(M, G12U, ij) = gu[5];
            MA(M, G22L, ij) = gl[8];
            MA(M, G22U, ij) = gu[8];
        }
    /* InitializeMetricDerivativesOnGrid (src/Metric.cpp:221-274) */
#pragma omp parallel for collapse(2)
    for (int64_t j = 0; j < ny; j++)
        for (int64_t i = 0; i < nx; i++)
        {
            double x = gx(g, (double)i), y = gy(g, (double)j);
            double dxl[9], dyl[9], dxu[9], dyu[9];
            metric_deriv(M, 1, x, y, 0, dxl);
            metric_deriv(M, 2, x, y, 0, dyl);
            metric_deriv(M, 1, x, y, 1, dxu);
            metric_deriv(M, 2, x, y, 1, dyu);
            int64_t ij = i + j * nx;
            static const int comp[6] = {0, 1, 2, 4, 5, 8}; /* 00 01 02 11 12 22 */
            for (int c = 0; c < 6; c++)
            {
                MA(M, D0G00L + 3 * c, ij) = 0.0;
                MA(M, D1G00L + 3 * c, ij) = dxl[comp[c]];
                MA(M, D2G00L + 3 * c, ij) = dyl[comp[c]];
                MA(M, D0G00U + 3 * c, ij) = 0.0;
                MA(M, D1G00U + 3 * c, ij) = dxu[comp[c]];
                MA(M, D2G00U + 3 * c, ij) = dyu[comp[c]];
            }
        }
    /* InitializeAdmComponentsOnGrid (src/Metric.cpp:276-336) */
#pragma omp parallel for
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        double g00u = MA(M, G00U, ij), g01u = MA(M, G01U, ij), g02u = MA(M, G02U, ij);
        double alpha = 1.0 / sqrt(-g00u);
        double b1 = alpha * alpha * g01u;
        double b2 = alpha * alpha * g02u;
        MA(M, ALPHA, ij) = alpha;
        MA(M, BETA1U, ij) = b1;
        MA(M, BETA2U, ij) = b2;
        MA(M, BETA1L, ij) = MA(M, G01L, ij);
        MA(M, BETA2L, ij) = MA(M, G02L, ij);
        MA(M, GAM11L, ij) = MA(M, G11L, ij);
        MA(M, GAM11U, ij) = MA(M, G11U, ij) + b1 * b1 / (alpha * alpha);
        MA(M, GAM12L, ij) = MA(M, G12L, ij);
        MA(M, GAM12U, ij) = MA(M, G12U, ij) + b1 * b2 / (alpha * alpha);
        MA(M, GAM22L, ij) = MA(M, G22L, ij);
        MA(M, GAM22U, ij) = MA(M, G22U, ij) + b2 * b2 / (alpha * alpha);
        double d1a = MA(M, D1G00U, ij) / (2.0 * pow(-g00u, 3.0 / 2.0));
        double d2a = MA(M, D2G00U, ij) / (2.0 * pow(-g00u, 3.0 / 2.0));
        MA(M, D1ALPHA, ij) = d1a;
        MA(M, D2ALPHA, ij) = d2a;
        double d1b1 = alpha * alpha * MA(M, D1G01U, ij) + 2.0 * g01u * alpha * d1a;
        double d2b1 = alpha * alpha * MA(M, D2G01U, ij) + 2.0 * g01u * alpha * d2a;
        double d1b2 = alpha * alpha * MA(M, D1G02U, ij) + 2.0 * g02u * alpha * d1a;
        double d2b2 = alpha * alpha * MA(M, D2G02U, ij) + 2.0 * g02u * alpha * d2a;
        MA(M, D1BETA1LU, ij) = d1b1;
        MA(M, D2BETA1LU, ij) = d2b1;
        MA(M, D1BETA2LU, ij) = d1b2;
        MA(M, D2BETA2LU, ij) = d2b2;
        MA(M, D1BETA1LL, ij) = MA(M, D1G01L, ij);
        MA(M, D1BETA2LL, ij) = MA(M, D1G02L, ij);
        MA(M, D2BETA1LL, ij) = MA(M, D2G01L, ij);
        MA(M, D2BETA2LL, ij) = MA(M, D2G02L, ij);
        MA(M, D1GAM11LLL, ij) = MA(M, D1G11L, ij);
        MA(M, D2GAM11LLL, ij) = MA(M, D2G11L, ij);
        MA(M, D1GAM12LLL, ij) = MA(M, D1G12L, ij);
        MA(M, D2GAM12LLL, ij) = MA(M, D2G12L, ij);
        MA(M, D1GAM22LLL, ij) = MA(M, D1G22L, ij);
        MA(M, D2GAM22LLL, ij) = MA(M, D2G22L, ij);
        double a3 = pow(alpha, 3);
        MA(M, D1GAM11LUU, ij) = MA(M, D1G11U, ij) + (d1b1 * b1 + b1 * d1b1) / (alpha * alpha) - 2.0 * b1 * b1 * d1a / a3;
        MA(M, D1GAM12LUU, ij) = MA(M, D1G12U, ij) + (d1b1 * b2 + b1 * d1b2) / (alpha * alpha) - 2.0 * b1 * b2 * d1a / a3;
        MA(M, D1GAM22LUU, ij) = MA(M, D1G22U, ij) + (d1b2 * b2 + b2 * d1b2) / (alpha * alpha) - 2.0 * b2 * b2 * d1a / a3;
        MA(M, D2GAM11LUU, ij) = MA(M, D2G11U, ij) + (d2b1 * b1 + b1 * d2b1) / (alpha * alpha) - 2.0 * b1 * b1 * d2a / a3;
        MA(M, D2GAM12LUU, ij) = MA(M, D2G12U, ij) + (d2b1 * b2 + b1 * d2b2) / (alpha * alpha) - 2.0 * b1 * b2 * d2a / a3;
        MA(M, D2GAM22LUU, ij) = MA(M, D2G22U, ij) + (d2b2 * b2 + b2 * d2b2) / (alpha * alpha) - 2.0 * b2 * b2 * d2a / a3;
        /* K_ab = (sum_c 2 gamma_ac d_b beta^c + d_c gamma_ab beta^c) / (2 alpha) */
        double beta[3] = {0, b1, b2};
        double gam[3][3] = {{0}, {0, MA(M, GAM11L, ij), MA(M, GAM12L, ij)}, {0, MA(M, GAM12L, ij), MA(M, GAM22L, ij)}};
        double dbeta[3][3] = {{0}, {0, d1b1, d1b2}, {0, d2b1, d2b2}}; /* [b][c] = d_b beta^c */
        double dgam[3][3][3];                                         /* [c][a][b] = d_c gamma_ab */
        dgam[1][1][1] = MA(M, D1GAM11LLL, ij);
        dgam[1][1][2] = dgam[1][2][1] = MA(M, D1GAM12LLL, ij);
        dgam[1][2][2] = MA(M, D1GAM22LLL, ij);
        dgam[2][1][1] = MA(M, D2GAM11LLL, ij);
        dgam[2][1][2] = dgam[2][2][1] = MA(M, D2GAM12LLL, ij);
        dgam[2][2][2] = MA(M, D2GAM22LLL, ij);
        double K[3][3];
        for (int a = 1; a < 3; a++)
            for (int b = 1; b < 3; b++)
            {
                K[a][b] = -0.0;
                for (int c = 1; c < 3; c++)
                    K[a][b] += 2.0 * gam[a][c] * dbeta[b][c] + dgam[c][a][b] * beta[c];
                K[a][b] /= 2.0 * alpha;
            }
        MA(M, K11, ij) = K[1][1];
        MA(M, K12, ij) = K[1][2];
        MA(M, K22, ij) = K[2][2];
    }
    /* InitializeBoostedTetradOnGrid (src/Metric.cpp:152-187) */
    for (int64_t ij = 0; ij < nxy; ij++)
    {
        double g22 = MA(M, GAM22L, ij);
        double gi11 = MA(M, GAM11U, ij), gi12 = MA(M, GAM12U, ij);
        double a = 1.0 / sqrt(gi11);
        double b = a * a * gi12;
        double m11 = 1 / a, m21 = b / a, m22 = 1;
        double g2 = m22 * g22 * m22;
        double alpha = MA(M, ALPHA, ij);
        double n0 = 1.0 / alpha, n1 = -MA(M, BETA1U, ij) / alpha, n2 = -MA(M, BETA2U, ij) / alpha;
        double t[9] = {n0, 0, 0, n1, m11, 0, n2, m21, 1 / sqrt(g2)};
        double ti[9];
        inv3(t, ti);
        for (int q = 0; q < 9; q++)
        {
            MA(M, T00 + q, ij) = t[q];
            MA(M, TI00 + q, ij) = ti[q];
        }
    }
}

/* Metric::InterpolateArrayTo_ij (src/Metric.cpp:338-348) */
static double interp_arr(const Metric *M, int k, double fi, double fj)
{
    int64_t i0 = (int64_t)floor(fi), j0 = (int64_t)floor(fj);
    int64_t i1 = i0 + 1, j1 = j0 + 1;
    double x = fi - (double)i0, y = fj - (double)j0;
    const int64_t nx = M->g.nx;
    double f00 = MA(M, k, i0 + j0 * nx), f01 = MA(M, k, i0 + j1 * nx);
    double f10 = MA(M, k, i1 + j0 * nx), f11 = MA(M, k, i1 + j1 * nx);
    double f0 = f00 * (1.0 - x) + f10 * x;
    double f1 = f01 * (1.0 - x) + f11 * x;
    return f0 * (1.0 - y) + f1 * y;
}

/* The metric quantities the geodesic right-hand side reads at a point
 * (Metric::Get*(Coord), src/Metric.cpp:584-780, with their flat defaults
 * outside the domain). */
typedef struct
{
    double alpha, beta1, beta2, da1, da2;
    double db[3][3];     /* [i][k] = d_i beta^k */
    double K[3][3];      /* K_ij */
    double gu[3][3];     /* gamma^ij */
    double dg[3][3][3];  /* [i][j][k] = d_i gamma_jk */
} Local;

static void local_at(const Metric *M, double x, double y, Local *L)
{
    memset(L, 0, sizeof(*L));
    if (outside(&M->g, x, y))
    {
        L->alpha = 1.0;
        L->gu[1][1] = 1;
        L->gu[2][2] = 1;
        return;
    }
    double fi = gi(&M->g, x), fj = gj(&M->g, y);
    L->alpha = interp_arr(M, ALPHA, fi, fj);
    L->beta1 = interp_arr(M, BETA1U, fi, fj);
    L->beta2 = interp_arr(M, BETA2U, fi, fj);
    L->da1 = interp_arr(M, D1ALPHA, fi, fj);
    L->da2 = interp_arr(M, D2ALPHA, fi, fj);
    L->db[1][1] = interp_arr(M, D1BETA1LU, fi, fj);
    L->db[1][2] = interp_arr(M, D1BETA2LU, fi, fj);
    L->db[2][1] = interp_arr(M, D2BETA1LU, fi, fj);
    L->db[2][2] = interp_arr(M, D2BETA2LU, fi, fj);
    L->K[1][1] = interp_arr(M, K11, fi, fj);
    L->K[2][2] = interp_arr(M, K22, fi, fj);
    L->K[1][2] = L->K[2][1] = interp_arr(M, K12, fi, fj);
    L->gu[1][1] = interp_arr(M, GAM11U, fi, fj);
    L->gu[2][2] = interp_arr(M, GAM22U, fi, fj);
    L->gu[1][2] = L->gu[2][1] = interp_arr(M, GAM12U, fi, fj);
    L->dg[1][1][1] = interp_arr(M, D1GAM11LLL, fi, fj);
    L->dg[1][2][2] = interp_arr(M, D1GAM22LLL, fi, fj);
    L->dg[1][1][2] = L->dg[1][2][1] = interp_arr(M, D1GAM12LLL, fi, fj);
    L->dg[2][1][1] = interp_arr(M, D2GAM11LLL, fi, fj);
    L->dg[2][2][2] = interp_arr(M, D2GAM22LLL, fi, fj);
    L->dg[2][1][2] = L->dg[2][2][1] = interp_arr(M, D2GAM12LLL, fi, fj);
}

/* GetTetrad(Coord) / GetTetradInverse(Coord) (src/Metric.cpp:547-577) */
static void tetrad_at(const Metric *M, double x, double y, int inverse, double *t)
{
    if (outside(&M->g, x, y))
    {
        for (int q = 0; q < 9; q++)
            t[q] = (q % 4 == 0) ? 1 : 0;
        return;
    }
    double fi = gi(&M->g, x), fj = gj(&M->g, y);
    for (int q = 0; q < 9; q++)
        t[q] = interp_arr(M, (inverse ? TI00 : T00) + q, fi, fj);
}
/* GetAlpha(Coord) (src/Metric.cpp:584-593) */
static double alpha_at(const Metric *M, double x, double y)
{
    if (outside(&M->g, x, y))
        return 1.0;
    return interp_arr(M, ALPHA, gi(&M->g, x), gj(&M->g, y));
}

/* ------------------------------------------------------ geodesic solver */
/* Dnu, Dx, Dv (src/GeodesicEquationSolver.cpp:5-55) */
static void geodesic_rhs(const Local *L, double nu, const double *v /* [3], 1-based */, double *dx, double *dv,
                         double *dnu)
{
    double da[3] = {0, L->da1, L->da2};
    double bu[3] = {0, L->beta1, L->beta2};
    double n = 0;
    for (int i = 1; i < 3; i++)
    {
        n -= v[i] * da[i];
        for (int j = 1; j < 3; j++)
            n += L->alpha * L->K[i][j] * v[i] * v[j];
    }
    n *= nu;
    *dnu = n;
    for (int k = 1; k < 3; k++)
        dx[k] = L->alpha * v[k] - bu[k];
    for (int k = 1; k < 3; k++)
    {
        dv[k] = 0.0;
        for (int i = 1; i < 3; i++)
        {
            dv[k] += v[k] * da[i] * v[i] - L->gu[k][i] * da[i] - v[i] * L->db[i][k];
            for (int j = 1; j < 3; j++)
            {
                dv[k] += 2.0 * L->alpha * L->gu[i][k] * L->K[i][j] * v[j] - L->alpha * v[k] * L->K[i][j] * v[i] * v[j];
                for (int l = 1; l < 3; l++)
                    dv[k] -= L->alpha * 0.5 * L->gu[k][l] * (L->dg[i][l][j] + L->dg[j][i][l] - L->dg[l][i][j]) * v[i] * v[j];
            }
        }
    }
}

static void stage(const Metric *M, const double *x, const double *v, double nu, double *kx, double *kv, double *knu)
{
    Local L;
    local_at(M, x[1], x[2], &L);
    geodesic_rhs(&L, nu, v, kx, kv, knu);
}

/* RK45_GeodesicEquation<-1> (src/GeodesicEquationSolver.cpp:80-188) */
static double rk45_backward(const Metric *M, double maxTE, double dt, double *x, double *v)
{
    const double td = -1;
    double k1x[3], k2x[3], k3x[3], k4x[3], k5x[3], k6x[3];
    double k1v[3], k2v[3], k3v[3], k4v[3], k5v[3], k6v[3];
    double k1n, k2n, k3n, k4n, k5n, k6n;
    double xt[3] = {0}, vt[3] = {0}, nt;
    double ddx[3], ddv[3], dnu;
    double nu = 1;
    double totalTime = 0;
    double ddt = M->g.dt;
    long guard = 0;
    while (totalTime < dt)
    {
        if (++guard > 10000000)
            return NAN;
        ddt = ddt < dt - totalTime ? ddt : dt - totalTime;
        stage(M, x, v, nu, k1x, k1v, &k1n);
        for (int d = 1; d < 3; d++)
        {
            xt[d] = x[d] + td * ddt * ((1.0 / 4.0) * k1x[d]);
            vt[d] = v[d] + td * ddt * ((1.0 / 4.0) * k1v[d]);
        }
        nt = nu + td * ddt * ((1.0 / 4.0) * k1n);
        stage(M, xt, vt, nt, k2x, k2v, &k2n);
        for (int d = 1; d < 3; d++)
        {
            xt[d] = x[d] + td * ddt * ((3.0 / 32.0) * k1x[d] + (9.0 / 32.0) * k2x[d]);
            vt[d] = v[d] + td * ddt * ((3.0 / 32.0) * k1v[d] + (9.0 / 32.0) * k2v[d]);
        }
        nt = nu + td * ddt * ((3.0 / 32.0) * k1n + (9.0 / 32.0) * k2n);
        stage(M, xt, vt, nt, k3x, k3v, &k3n);
        for (int d = 1; d < 3; d++)
        {
            xt[d] = x[d] + td * ddt * ((1932.0 / 2197.0) * k1x[d] - (7200.0 / 2197.0) * k2x[d] + (7296.0 / 2197.0) * k3x[d]);
            vt[d] = v[d] + td * ddt * ((1932.0 / 2197.0) * k1v[d] - (7200.0 / 2197.0) * k2v[d] + (7296.0 / 2197.0) * k3v[d]);
        }
        nt = nu + td * ddt * ((1932.0 / 2197.0) * k1n - (7200.0 / 2197.0) * k2n + (7296.0 / 2197.0) * k3n);
        stage(M, xt, vt, nt, k4x, k4v, &k4n);
        for (int d = 1; d < 3; d++)
        {
            xt[d] = x[d] + td * ddt * ((439.0 / 216.0) * k1x[d] - (8.0) * k2x[d] + (3680.0 / 513.0) * k3x[d] - (845.0 / 4104.0) * k4x[d]);
            vt[d] = v[d] + td * ddt * ((439.0 / 216.0) * k1v[d] - (8.0) * k2v[d] + (3680.0 / 513.0) * k3v[d] - (845.0 / 4104.0) * k4v[d]);
        }
        nt = nu + td * ddt * ((439.0 / 216.0) * k1n - (8.0) * k2n + (3680.0 / 513.0) * k3n - (845.0 / 4104.0) * k4n);
        stage(M, xt, vt, nt, k5x, k5v, &k5n);
        for (int d = 1; d < 3; d++)
        {
            xt[d] = x[d] + td * ddt * (-(8.0 / 27.0) * k1x[d] + (2.0) * k2x[d] - (3544.0 / 2565.0) * k3x[d] + (1859.0 / 4104.0) * k4x[d] - (11.0 / 44.0) * k5x[d]);
            vt[d] = v[d] + td * ddt * (-(8.0 / 27.0) * k1v[d] + (2.0) * k2v[d] - (3544.0 / 2565.0) * k3v[d] + (1859.0 / 4104.0) * k4v[d] - (11.0 / 44.0) * k5v[d]);
        }
        nt = nu + td * ddt * (-(8.0 / 27.0) * k1n + (2.0) * k2n - (3544.0 / 2565.0) * k3n + (1859.0 / 4104.0) * k4n - (11.0 / 44.0) * k5n);
        stage(M, xt, vt, nt, k6x, k6v, &k6n);
        for (int d = 1; d < 3; d++)
        {
            ddx[d] = (16.0 / 135.0) * k1x[d] + (6656.0 / 12825.0) * k3x[d] + (28561.0 / 56430.0) * k4x[d] - (9.0 / 50.0) * k5x[d] + (2.0 / 55.0) * k6x[d];
            ddv[d] = (16.0 / 135.0) * k1v[d] + (6656.0 / 12825.0) * k3v[d] + (28561.0 / 56430.0) * k4v[d] - (9.0 / 50.0) * k5v[d] + (2.0 / 55.0) * k6v[d];
        }
        dnu = (16.0 / 135.0) * k1n + (6656.0 / 12825.0) * k3n + (28561.0 / 56430.0) * k4n - (9.0 / 50.0) * k5n + (2.0 / 55.0) * k6n;
        double TE = 0;
        for (int d = 1; d < 3; d++)
        {
            double e = ddt * ((1.0 / 360.0) * k1v[d] - (128.0 / 4275.0) * k3v[d] - (2197.0 / 75240.0) * k4v[d] + (1.0 / 50.0) * k5v[d] + (2.0 / 55.0) * k6v[d]);
            TE += e * e;
        }
        TE = sqrt(TE);
        if (TE > maxTE)
        {
            ddt *= 0.95 * pow(maxTE / TE, 1.0 / 4.0);
            continue;
        }
        for (int d = 1; d < 3; d++)
        {
            x[d] += td * ddt * ddx[d];
            v[d] += td * ddt * ddv[d];
        }
        nu += td * ddt * dnu;
        totalTime += ddt;
        ddt *= 0.95 * pow(maxTE / (TE + 1e-50), 1.0 / 4.0);
        if (inside_bh(M, x[1], x[2]) || outside(&M->g, x[1], x[2]))
            break;
    }
    return nu;
}

/* ---------------------------------------------------------------- fourier */
/* Fourier::Basis (src/FourierHarmonics.cpp:5-14) */
static double fbasis(int k, double phi)
{
    const double sqrt2 = 1.41421356237309504880;
    if (k == 0)
        return 1.0;
    else if (k % 2 != 0)
        return sqrt2 * cos(phi * (k + 1.0) / 2.0);
    else
        return sqrt2 * sin(phi * k / 2.0);
}
/* Fourier::GetCoefficients (src/FourierHarmonics.cpp:33-45) */
static void fcoef(const Stencil *s, const double *data, double *coef)
{
    for (int i = 0; i < s->n; i++)
        coef[i] = 0;
    for (int d = 0; d < s->n; d++)
    {
        double phi = s->phi[d];
        double c = data[d] * s->w[d];
        for (int i = 0; i < s->n; i++)
            coef[i] += c * fbasis(i, phi);
    }
}
/* Fourier::GetValue (src/FourierHarmonics.cpp:56-61) */
static double fvalue(double phi, const double *coef, int n)
{
    double result = 0;
    for (int i = 0; i < n; i++)
        result += coef[i] * fbasis(i, phi);
    return result;
}

/* ------------------------------------------------------------- radiation */
typedef struct
{
    const grlbm_ref_params *p;
    Grid g;
    Metric M;
    Stencil st, ss;
    int nd, nf;
    double c0, s0; /* RotationMatrix(0) entries */
    double *nxd, *nyd; /* R(0) C(d) */
    double *I, *Inew;
    double *E, *Fx, *Fy, *Pxx, *Pxy, *Pyy;
    double *cS, *cX, *cY, *cCx, *cCy;
    int *iters;
    int maxIter;
    double sumIter;
} Rad;

/* Radiation::UpdateFourierCoefficients (src/Radiation.cpp:191-237) */
static void update_fourier(Rad *R)
{
    const Grid *g = &R->g;
    const int nf = R->nf;
    const double maxTE = R->p->rk_tol;
#pragma omp parallel for collapse(2) schedule(dynamic, 50)
    for (int64_t j = 1; j < g->ny - 1; j++)
        for (int64_t i = 1; i < g->nx - 1; i++)
        {
            int64_t ij = i + j * g->nx;
            double dS[64], dX[64], dY[64], dCx[64], dCy[64];
            double x0 = gx(g, (double)i), y0 = gy(g, (double)j);
            double alpha = MA(&R->M, ALPHA, ij);
            for (int d = 0; d < nf; d++)
            {
                double s = 1;
                double x[3] = {0, x0, y0};
                double c1 = R->ss.cx[d], c2 = R->ss.cy[d];
                double u0 = alpha, u1 = c1 * alpha, u2 = c2 * alpha;
                (void)u0;
                /* Vec2ObservedByEulObs<IF,LF> (src/SpecialMath.cpp:131-136) */
                double a = alpha_at(&R->M, x[1], x[2]);
                double vv1 = u1 / a, vv2 = u2 / a;
                double t[9];
                tetrad_at(&R->M, x[1], x[2], 0, t);
                double v[3] = {0, t[4] * vv1 + t[5] * vv2, t[7] * vv1 + t[8] * vv2};
                if (!inside_bh(&R->M, x[1], x[2]))
                    s *= rk45_backward(&R->M, maxTE, g->dt, x, v);
                else
                    v[1] = v[2] = 0.0;
                double ti[9];
                tetrad_at(&R->M, x[1], x[2], 1, ti);
                double vIF1 = ti[4] * v[1] + ti[5] * v[2];
                double vIF2 = ti[7] * v[1] + ti[8] * v[2];
                dS[d] = 1.0 / s;
                dX[d] = x[1];
                dY[d] = x[2];
                dCx[d] = vIF1;
                dCy[d] = vIF2;
            }
            fcoef(&R->ss, dS, R->cS + ij * nf);
            fcoef(&R->ss, dX, R->cX + ij * nf);
            fcoef(&R->ss, dY, R->cY + ij * nf);
            fcoef(&R->ss, dCx, R->cCx + ij * nf);
            fcoef(&R->ss, dCy, R->cCy + ij * nf);
        }
}

/* identity coefficients of the constructor (src/Radiation.cpp:59-82) */
static void identity_fourier(Rad *R)
{
    const int nf = R->nf;
    for (int64_t ij = 0; ij < R->g.nxy; ij++)
    {
        double dS[64], dX[64], dY[64], dCx[64], dCy[64];
        int64_t i = ij % R->g.nx, j = ij / R->g.nx;
        for (int d = 0; d < nf; d++)
        {
            dS[d] = 1.0;
            dX[d] = gx(&R->g, (double)i);
            dY[d] = gy(&R->g, (double)j);
            dCx[d] = R->st.cx[d]; /* the reference reads the intensity stencil here */
            dCy[d] = R->st.cy[d];
        }
        fcoef(&R->ss, dS, R->cS + ij * nf);
        fcoef(&R->ss, dX, R->cX + ij * nf);
        fcoef(&R->ss, dY, R->cY + ij * nf);
        fcoef(&R->ss, dCx, R->cCx + ij * nf);
        fcoef(&R->ss, dCy, R->cCy + ij * nf);
    }
}

/* Radiation::InitialDataLFtoIF + LoadInitialData (src/Radiation.cpp:103-182)
 * for fixed (non-rotated) streaming */
static void load_initial(Rad *R, const grlbm_ref_inputs *in)
{
    const int nd = R->nd;
    for (int64_t ij = 0; ij < R->g.nxy; ij++)
    {
        if (!in->is_initial[ij])
            continue;
        if (R->p->initial_data_type == 1)
        {
            for (int d = 0; d < nd; d++)
                R->I[ij * nd + d] = in->initial_I[ij * nd + d];
            continue;
        }
        double TL[9] = {in->initial_E_LF[ij], in->initial_Fx_LF[ij], in->initial_Fy_LF[ij],
                        in->initial_Fx_LF[ij], in->initial_Pxx_LF[ij], in->initial_Pxy_LF[ij],
                        in->initial_Fy_LF[ij], in->initial_Pxy_LF[ij], in->initial_Pyy_LF[ij]};
        double t[9], ti[9], TI[9];
        for (int q = 0; q < 9; q++)
            t[q] = MA(&R->M, T00 + q, ij);
        inv3(t, ti);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
            {
                TI[3 * a + b] = 0.0;
                for (int A = 0; A < 3; A++)
                    for (int B = 0; B < 3; B++)
                        TI[3 * a + b] += TL[3 * A + B] * ti[3 * a + A] * ti[3 * b + B];
            }
        double E = TI[0];
        double Fx = TL[1]; /* the reference takes the flux from the LF tensor */
        double Fy = TL[2];
        double F = sqrt(Fx * Fx + Fy * Fy);
        if (F > E)
        {
            Fx *= E / F;
            Fy *= E / F;
        }
        double Fn = sqrt(Fx * Fx + Fy * Fy);
        double rel = Fn / E;
        double dir1 = Fx / Fn, dir2 = Fy / Fn;
        if (Fn < 1e-16)
        {
            dir1 = 1;
            dir2 = 0;
        }
        double sigma = lut_eval(R->st.lut_in, R->st.lut_sigma, R->st.nlut, rel);
        double norm = lut_eval(R->st.lut_in, R->st.lut_norm, R->st.nlut, rel);
        for (int d = 0; d < nd; d++)
            R->I[ij * nd + d] = E * exp(sigma * (dir1 * R->st.cx[d] + dir2 * R->st.cy[d]) - norm);
    }
}

/* Radiation::StreamFlatFixed (src/Radiation.cpp:380-414) */
static void stream_flat(Rad *R)
{
    const Grid *g = &R->g;
    const int nd = R->nd;
    const int64_t nx = g->nx;
#pragma omp parallel for collapse(2) schedule(dynamic, 50)
    for (int64_t j = 1; j < g->ny - 1; j++)
        for (int64_t i = 1; i < g->nx - 1; i++)
        {
            int64_t ij = i + j * nx;
            for (int d = 0; d < nd; d++)
            {
                double x = gx(g, (double)i), y = gy(g, (double)j);
                x -= R->st.cx[d] * g->dt;
                y -= R->st.cy[d] * g->dt;
                double it = gi(g, x), jt = gj(g, y);
                int64_t i0 = (int64_t)floor(it), j0 = (int64_t)floor(jt);
                int64_t i1 = i0 + 1, j1 = j0 + 1;
                double fx = it - (double)i0, fy = jt - (double)j0;
                double f00 = R->I[(i0 + j0 * nx) * nd + d], f01 = R->I[(i0 + j1 * nx) * nd + d];
                double f10 = R->I[(i1 + j0 * nx) * nd + d], f11 = R->I[(i1 + j1 * nx) * nd + d];
                double f0 = f00 * (1.0 - fx) + f10 * fx;
                double f1 = f01 * (1.0 - fx) + f11 * fx;
                R->Inew[ij * nd + d] = f0 * (1.0 - fy) + f1 * fy;
            }
        }
    double *t = R->I;
    R->I = R->Inew;
    R->Inew = t;
}

/* Radiation::IntensityAt with rotationAngle 0 (src/Radiation.cpp:322-343) */
static double intensity_at(const Rad *R, int64_t ij, double v1, double v2)
{
    double w1 = v1 * R->c0 - v2 * R->s0;
    double w2 = v1 * R->s0 + v2 * R->c0;
    double angle = phi_of(w1, w2);
    const int ng = R->st.ng;
    double dd = (double)ng * angle / (2.0 * PI);
    if (dd < 1e-8)
        dd = 1e-8;
    if (dd > ng - 1e-8)
        dd = ng - 1e-8;
    int64_t d0 = ((int64_t)floor(dd)) % ng;
    int64_t d1 = (d0 + 1) % ng;
    const int nd = R->nd;
    double v0 = 0, vv1 = 0;
    for (int k = 0; k < 4; k++)
    {
        v0 += R->st.wt[4 * d0 + k] * R->I[ij * nd + R->st.idx[4 * d0 + k]];
        vv1 += R->st.wt[4 * d1 + k] * R->I[ij * nd + R->st.idx[4 * d1 + k]];
    }
    double x = dd - (double)d0;
    double r = v0 * (1.0 - x) + vv1 * x;
    return r > 0.0 ? r : 0.0;
}

/* Radiation::StreamCurvedFixed (src/Radiation.cpp:454-512) */
static void stream_curved(Rad *R)
{
    const Grid *g = &R->g;
    const int nd = R->nd, nf = R->nf;
    const int64_t nx = g->nx;
#pragma omp parallel for collapse(2) schedule(dynamic, 50)
    for (int64_t j = 1; j < g->ny - 1; j++)
        for (int64_t i = 1; i < g->nx - 1; i++)
        {
            int64_t ij = i + j * nx;
            if (inside_bh(&R->M, gx(g, (double)i), gy(g, (double)j)))
            {
                for (int d = 0; d < nd; d++)
                    R->Inew[ij * nd + d] = 0;
                continue;
            }
            double alpha = MA(&R->M, ALPHA, ij);
            for (int d = 0; d < nd; d++)
            {
                double angle = R->st.phi[d];
                double s = fvalue(angle, R->cS + ij * nf, nf);
                double xt = fvalue(angle, R->cX + ij * nf, nf);
                double yt = fvalue(angle, R->cY + ij * nf, nf);
                double v1 = fvalue(angle, R->cCx + ij * nf, nf);
                double v2 = fvalue(angle, R->cCy + ij * nf, nf);
                if (inside_bh(&R->M, xt, yt))
                {
                    R->Inew[ij * nd + d] = 0;
                    continue;
                }
                double it = gi(g, xt), jt = gj(g, yt);
                int64_t i0 = (int64_t)floor(it), j0 = (int64_t)floor(jt);
                int64_t i1 = i0 + 1, j1 = j0 + 1;
                int64_t c00 = i0 + j0 * nx, c01 = i0 + j1 * nx, c10 = i1 + j0 * nx, c11 = i1 + j1 * nx;
                double r;
                r = alpha / MA(&R->M, ALPHA, c00);
                double I00 = r * (r * r) * intensity_at(R, c00, v1, v2);
                r = alpha / MA(&R->M, ALPHA, c01);
                double I01 = r * (r * r) * intensity_at(R, c01, v1, v2);
                r = alpha / MA(&R->M, ALPHA, c10);
                double I10 = r * (r * r) * intensity_at(R, c10, v1, v2);
                r = alpha / MA(&R->M, ALPHA, c11);
                double I11 = r * (r * r) * intensity_at(R, c11, v1, v2);
                double fx = it - (double)i0, fy = jt - (double)j0;
                double f0 = I00 * (1.0 - fx) + I10 * fx;
                double f1 = I01 * (1.0 - fx) + I11 * fx;
                R->Inew[ij * nd + d] = s * (s * s) * (f0 * (1.0 - fy) + f1 * fy);
            }
        }
    double *t = R->I;
    R->I = R->Inew;
    R->Inew = t;
}

/* Radiation::ComputeMomentsIF (src/Radiation.cpp:239-269) */
static void moments_if(Rad *R)
{
    const int nd = R->nd;
#pragma omp parallel for
    for (int64_t ij = 0; ij < R->g.nxy; ij++)
    {
        double E = 0, Fx = 0, Fy = 0, Pxx = 0, Pxy = 0, Pyy = 0;
        for (int d = 0; d < nd; d++)
        {
            if (R->st.w[d] == 0.0)
                continue;
            double c = R->st.w[d] * R->I[ij * nd + d];
            double n1 = R->nxd[d], n2 = R->nyd[d];
            E += c;
            Fx += c * n1;
            Fy += c * n2;
            Pxx += c * n1 * n1;
            Pxy += c * n1 * n2;
            Pyy += c * n2 * n2;
        }
        R->E[ij] = E;
        R->Fx[ij] = Fx;
        R->Fy[ij] = Fy;
        R->Pxx[ij] = Pxx;
        R->Pxy[ij] = Pxy;
        R->Pyy[ij] = Pyy;
    }
}

/* Radiation::Collide (src/Radiation.cpp:641-736) */
static void collide(Rad *R, const grlbm_ref_inputs *in)
{
    const Grid *g = &R->g;
    const int nd = R->nd;
    const int64_t nx = g->nx;
#pragma omp parallel for collapse(2) schedule(dynamic, 50)
    for (int64_t j = 1; j < g->ny - 1; j++)
        for (int64_t i = 1; i < g->nx - 1; i++)
        {
            if (inside_bh(&R->M, gx(g, (double)i), gy(g, (double)j)))
                continue;
            int64_t ij = i + j * nx;
            double uL1 = in->ux[ij], uL2 = in->uy[ij];
            /* TransformLFtoIF(uLF, GetTetrad(ij)): the reference passes the tetrad */
            double u1 = MA(&R->M, T11, ij) * uL1 + MA(&R->M, T12, ij) * uL2;
            double u2 = MA(&R->M, T21, ij) * uL1 + MA(&R->M, T22, ij) * uL2;
            double alpha = MA(&R->M, ALPHA, ij);
            double uu = u1 * u1 + u2 * u2;
            double lorentz = 1.0 / sqrt(1.0 - uu);
            double k0 = in->kappa0[ij], k1 = in->kappa1[ij], ka = in->kappaA[ij], eta = in->eta[ij];
            int cycles = 0;
            double diff = 1;
            while (fabs(diff) > 1e-4 && cycles < 100)
            {
                cycles++;
                double pE = R->E[ij], pFx = R->Fx[ij], pFy = R->Fy[ij];
                double pPxx = R->Pxx[ij], pPxy = R->Pxy[ij], pPyy = R->Pyy[ij];
                double uF = u1 * pFx + u2 * pFy;
                double uxP = u1 * pPxx + u2 * pPxy;
                double uyP = u1 * pPxy + u2 * pPyy;
                double uuP = u1 * uxP + u2 * uyP;
                double fE = lorentz * lorentz * (pE - 2.0 * uF + uuP);
                double fFx = lorentz * lorentz * (pFx - lorentz * pE * u1 - uxP + u1 * lorentz / (1.0 + lorentz) * ((2.0 * lorentz + 1.0) * uF - lorentz * uuP));
                double fFy = lorentz * lorentz * (pFy - lorentz * pE * u2 - uyP + u2 * lorentz / (1.0 + lorentz) * ((2.0 * lorentz + 1.0) * uF - lorentz * uuP));
                double E = 0, Fx = 0, Fy = 0, Pxx = 0, Pxy = 0, Pyy = 0;
                for (int d = 0; d < nd; d++)
                {
                    double n1 = R->nxd[d], n2 = R->nyd[d];
                    double un = u1 * n1 + u2 * n2;
                    double A = lorentz * (1.0 - un);
                    double sc = (1 - (lorentz * un) / (lorentz + 1)) * lorentz;
                    double nF1 = (n1 - sc * u1) / A;
                    double nF2 = (n2 - sc * u2) / A;
                    double nF = nF1 * fFx + nF2 * fFy;
                    double M = k0 * fE + 3.0 * k1 * nF;
                    double v = (R->I[ij * nd + d] + alpha * g->dt * (eta + M) / (A * A)) /
                               (1.0 + alpha * g->dt * (ka + k0) * A);
                    R->Inew[ij * nd + d] = v;
                    double c = R->st.w[d] * v;
                    E += c;
                    Fx += c * n1;
                    Fy += c * n2;
                    Pxx += c * n1 * n1;
                    Pxy += c * n1 * n2;
                    Pyy += c * n2 * n2;
                }
                R->E[ij] = E;
                R->Fx[ij] = Fx;
                R->Fy[ij] = Fy;
                R->Pxx[ij] = Pxx;
                R->Pxy[ij] = Pxy;
                R->Pyy[ij] = Pyy;
                double a1 = (pE - E) / E, a2 = (pFx - Fx) / Fx, a3 = (pFy - Fy) / Fy;
                double a4 = (pPxx - Pxx) / Pxx, a5 = (pPxy - Pxy) / Pxy, a6 = (pPyy - Pyy) / Pyy;
                diff = sqrt(a1 * a1 + a2 * a2 + a3 * a3 + a4 * a4 + a5 * a5 + a6 * a6);
            }
            R->iters[ij] = cycles;
        }
    int mx = 0;
    for (int64_t ij = 0; ij < g->nxy; ij++)
    {
        if (R->iters[ij] > mx)
            mx = R->iters[ij];
        R->sumIter += R->iters[ij];
        R->iters[ij] = 0;
    }
    if (mx > R->maxIter)
        R->maxIter = mx;
    double *t = R->I;
    R->I = R->Inew;
    R->Inew = t;
}

/* Radiation::ComputeMomentsLF (src/Radiation.cpp:270-301) */
static void moments_lf(Rad *R, grlbm_ref_outputs *out)
{
    const Grid *g = &R->g;
    for (int64_t j = 0; j < g->ny; j++)
        for (int64_t i = 0; i < g->nx; i++)
        {
            int64_t ij = i + j * g->nx;
            double o[7] = {0, 0, 0, 0, 0, 0, 0};
            if (!inside_bh(&R->M, gx(g, (double)i), gy(g, (double)j)))
            {
                double T[9] = {R->E[ij], R->Fx[ij], R->Fy[ij], R->Fx[ij], R->Pxx[ij], R->Pxy[ij],
                               R->Fy[ij], R->Pxy[ij], R->Pyy[ij]};
                double e[9], L[9];
                for (int q = 0; q < 9; q++)
                    e[q] = MA(&R->M, T00 + q, ij);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                    {
                        L[3 * a + b] = 0.0;
                        for (int A = 0; A < 3; A++)
                            for (int B = 0; B < 3; B++)
                                L[3 * a + b] += T[3 * A + B] * e[3 * a + A] * e[3 * b + B];
                    }
                o[0] = L[0];
                o[1] = L[1];
                o[2] = L[2];
                o[3] = L[4];
                o[4] = L[5];
                o[5] = L[8];
                double v[3] = {0, o[1], o[2]};
                double gam[3][3] = {{0}, {0, MA(&R->M, GAM11L, ij), MA(&R->M, GAM12L, ij)},
                                    {0, MA(&R->M, GAM12L, ij), MA(&R->M, GAM22L, ij)}};
                double n2 = 0;
                for (int a = 1; a < 3; a++)
                    for (int b = 1; b < 3; b++)
                        n2 += gam[a][b] * v[a] * v[b];
                o[6] = sqrt(fabs(n2));
            }
            double *dst[7] = {out->E_LF, out->Fx_LF, out->Fy_LF, out->Pxx_LF, out->Pxy_LF, out->Pyy_LF, out->F_LF};
            for (int q = 0; q < 7; q++)
                if (dst[q])
                    dst[q][ij] = o[q];
        }
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void put(double *dst, const double *src, size_t n)
{
    if (dst)
        memcpy(dst, src, n * sizeof(double));
}

int oracle_run(const grlbm_ref_params *p, const grlbm_ref_inputs *in, grlbm_ref_outputs *out)
{
    if (p->streaming_type != 0 && p->streaming_type != 2)
        return -2;
    if (p->n_fourier > 64 || p->n_fourier < 1 || p->n_dir < 4)
        return -3;
#ifdef _OPENMP
    if (p->n_threads > 0)
        omp_set_num_threads(p->n_threads);
#endif
    Rad R;
    memset(&R, 0, sizeof R);
    R.p = p;
    R.g = grid_make(p);
    metric_build(&R.M, p, &R.g);
    const size_t nxy = R.g.nxy;
    if (out->metric_arrays)
        memcpy(out->metric_arrays, R.M.arr, sizeof(double) * NMETRIC * nxy);
    if (in->metric_override)
        memcpy(R.M.arr, in->metric_override, sizeof(double) * NMETRIC * nxy);
    stencil_make(&R.st, p->n_dir, 1);
    stencil_make(&R.ss, p->n_fourier, 0);
    R.nd = p->n_dir;
    R.nf = p->n_fourier;
    R.c0 = rot0_cos();
    R.s0 = rot0_sin();
    R.nxd = malloc(sizeof(double) * R.nd);
    R.nyd = malloc(sizeof(double) * R.nd);
    for (int d = 0; d < R.nd; d++)
    {
        double cx = R.st.cx[d], cy = R.st.cy[d];
        R.nxd[d] = cx * R.c0 - cy * R.s0;
        R.nyd[d] = cx * R.s0 + cy * R.c0;
    }
    R.I = calloc(nxy * R.nd, sizeof(double));
    R.Inew = calloc(nxy * R.nd, sizeof(double));
    R.E = calloc(nxy, sizeof(double));
    R.Fx = calloc(nxy, sizeof(double));
    R.Fy = calloc(nxy, sizeof(double));
    R.Pxx = calloc(nxy, sizeof(double));
    R.Pxy = calloc(nxy, sizeof(double));
    R.Pyy = calloc(nxy, sizeof(double));
    R.cS = calloc(nxy * R.nf, sizeof(double));
    R.cX = calloc(nxy * R.nf, sizeof(double));
    R.cY = calloc(nxy * R.nf, sizeof(double));
    R.cCx = calloc(nxy * R.nf, sizeof(double));
    R.cCy = calloc(nxy * R.nf, sizeof(double));
    R.iters = calloc(nxy, sizeof(int));
    identity_fourier(&R);

    /* src/Radiation.cpp:745-746, 784-832 */
    load_initial(&R, in);
    double t0 = now_s();
    update_fourier(&R);
    out->table_time_s = now_s() - t0;
    t0 = now_s();
    for (int n = 0; n < p->n_steps; n++)
    {
        double ts = now_s();
        if (p->keep_source_nodes_active)
            load_initial(&R, in);
        if (p->streaming_type == 0)
            stream_flat(&R);
        else
            stream_curved(&R);
        moments_if(&R);
        collide(&R, in);
        if (out->step_times)
            out->step_times[n] = now_s() - ts;
    }
    out->computation_time_s = now_s() - t0;
    out->max_iterations = R.maxIter;
    out->average_iterations = R.sumIter / ((double)p->n_steps * (R.g.nx - 2) * (R.g.ny - 2));

    put(out->E, R.E, nxy);
    put(out->Fx, R.Fx, nxy);
    put(out->Fy, R.Fy, nxy);
    put(out->Pxx, R.Pxx, nxy);
    put(out->Pxy, R.Pxy, nxy);
    put(out->Pyy, R.Pyy, nxy);
    put(out->I, R.I, nxy * R.nd);
    put(out->coefS, R.cS, nxy * R.nf);
    put(out->coefX, R.cX, nxy * R.nf);
    put(out->coefY, R.cY, nxy * R.nf);
    put(out->coefCx, R.cCx, nxy * R.nf);
    put(out->coefCy, R.cCy, nxy * R.nf);
    moments_lf(&R, out);
    put(out->st_w, R.st.w, R.nd);
    put(out->st_phi, R.st.phi, R.nd);
    put(out->st_cx, R.st.cx, R.nd);
    put(out->st_cy, R.st.cy, R.nd);
    if (out->ig_index)
        memcpy(out->ig_index, R.st.idx, sizeof(int64_t) * 4 * R.st.ng);
    put(out->ig_weight, R.st.wt, 4 * (size_t)R.st.ng);
    put(out->ss_phi, R.ss.phi, R.nf);
    put(out->ss_w, R.ss.w, R.nf);

    free(R.nxd);
    free(R.nyd);
    free(R.I);
    free(R.Inew);
    free(R.E);
    free(R.Fx);
    free(R.Fy);
    free(R.Pxx);
    free(R.Pxy);
    free(R.Pyy);
    free(R.cS);
    free(R.cX);
    free(R.cY);
    free(R.cCx);
    free(R.cCy);
    free(R.iters);
    free(R.M.arr);
    stencil_free(&R.st);
    stencil_free(&R.ss);
    return 0;
}
