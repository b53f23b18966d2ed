// Fast FP64 step of the fixed streaming types (StreamFlatFixed and
// StreamCurvedFixed with IntensityAt, then ComputeMomentsIF and Collide;
// src/Radiation.cpp:380-414, 454-512, 322-343, 239-269, 641-736) on a
// cell-major FP64 state.  Same scheme as the FP32 precision step
// (kernels_step32.cu) with every value in FP64 and contracted FMAs: it agrees
// with the reference to rounding wherever the lambda iteration stops at the
// reference's cycle (always without scattering, kappa0 = kappa1 = 0, where
// the first cycle's intensities are final).
//
// State: J[(i + j nx) dp + d] (J = I / alpha^3 for curved streaming, I for
// flat), directions fastest, directions 0..3 repeated after the last one
// (dp = nd + 4 rounded up to 2 doubles): every 5-direction angular window of a
// node is one contiguous run.  In shared memory a node's run is padded to dps
// doubles, a multiple of 16 (the TMA box is wider than dp; the rest is zero
// fill), so that lanes reading neighbouring nodes at the same direction
// offset hit disjoint banks.
//
// Work split: every warp takes tiles of tx x ty <= 16 cells from a counter,
// stages the tile's (tx + 2) x (ty + 2) node patch with one TMA tensor copy,
// and runs three phases:
//   1. stream every cell, lanes over the directions, into the warp's buffer
//      of streamed values (then the next tile's copy is issued);
//   2. moments and the lambda iteration, two lanes per cell -- the iteration
//      is affine in the previous moments, so it runs on the six moments;
//   3. store the cells' new state, coalesced along the directions.
//
// Curved departures come from 32-byte packed records (packed64); flat ones
// are computed per cell with the reference's roundings (each product and sum
// rounded once: the _rn intrinsics are never contracted), so that they are
// the reference's bit for bit.  Departures outside the cell's 3x3
// neighbourhood gather from global memory (cold code).
#include <cudaTypedefs.h>

#include <algorithm>

#include "device_common.cuh"
#include "step_common.cuh"

// resident blocks per SM the step is compiled for: three at one pass (at
// most 168 registers; 12-18% faster than two blocks at 16 and 32 directions
// with curved streaming, 72 bytes of spills included), two at more passes
#ifndef GRLBM_STEP64_MIN_BLOCKS
#define GRLBM_STEP64_MIN_BLOCKS 2
#endif
#ifndef GRLBM_STEP64_MIN_BLOCKS_1
#define GRLBM_STEP64_MIN_BLOCKS_1 3
#endif

namespace grlbm
{
namespace
{
constexpr int kWarps = kStep64Warps;
constexpr int kUnitCells = kStep32UnitCells;
constexpr int kThreads = 32 * kWarps;
// shared layout: the warps' mbarriers, then (16-byte aligned) the row-type
// table, the direction coefficients, the moment sums, then the warps' buffers
constexpr int kTablesOffset = 64;
static_assert(8 * kWarps <= kTablesOffset, "mbarriers before the tables");
static_assert(kUnitCells == 16, "phase 2 pairs lane c and lane c + 16");

__device__ __forceinline__ unsigned hi_word(double x) { return (unsigned)__double2hiint(x); }

// a 32-byte record read once (streaming), or through the read-only path
__device__ __forceinline__ double4 ld_once(const double4 *p)
{
    const double2 lo = __ldcs(reinterpret_cast<const double2 *>(p)), hi = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ double4 ld_ro(const double4 *p)
{
    const double2 lo = __ldg(reinterpret_cast<const double2 *>(p)), hi = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// v in [1, 2) with its exponent field and sign replaced by a payload: the
// fraction v - 1 (exact)
__device__ __forceinline__ double unbias(double v)
{
    return __hiloint2double((int)((hi_word(v) & packed64::kMantHi) | packed64::kOne), __double2loint(v)) - 1.0;
}

// direction coefficients of the affine collide map for a moving fluid
__device__ __forceinline__ void collide_coeffs64(double n1, double n2, double u1, double u2, double lor, double adt,
                                                 double kak0, double &g, double &h, double &q1, double &q2)
{
    const double un = u1 * n1 + u2 * n2;
    const double A = lor * (1.0 - un);
    const double sc = (1.0 - (lor * un) / (lor + 1.0)) * lor;
    q1 = (n1 - sc * u1) / A;
    q2 = (n2 - sc * u2) / A;
    g = 1.0 / (1.0 + adt * kak0 * A);
    h = adt / (A * A) * g;
}

// The 5-tap angular window at one corner, clamped at zero.
__device__ __forceinline__ double window5(const double *p, double w0, double w1, double w2, double w3, double w4)
{
    return fmax(fma(w4, p[4], fma(w3, p[3], fma(w2, p[2], fma(w1, p[1], w0 * p[0])))), 0.0);
}

// One curved stream value from global memory, for a departure outside the
// cell's 3x3 neighbourhood: the side record {i_dep - i, j_dep - j, angle
// coordinate, s^3 alpha_c^3}, corners clamped to the grid as the reference's
// gather would index them (cold code, kept out of line).
__device__ __noinline__ double stream_far64(const double *__restrict__ Iin, double4 r, int dp, int nx, int ny, int nd,
                                            int ng, const double *rowtab, int q, int p, double inv_q, int i, int j)
{
    const double fli = floor(r.x), flj = floor(r.y);
    const double fx = r.x - fli, fy = r.y - flj;
    const int i0 = min(max(i + (int)fli, 0), nx - 2);
    const int j0 = min(max(j + (int)flj, 0), ny - 2);
    const double z = r.z == r.z ? r.z : 0.0;
    const double g = fmin(fmax(floor(z), 0.0), (double)(ng - 1));
    const double t = fmin(fmax(z - g, 0.0), 1.0);
    const double m = floor((g + 0.5) * inv_q);
    const int rt = min(max((int)(g - m * (double)q), 0), q - 1);
    const double *row = rowtab + rt * 12;
    const int s = (int)(m * (double)p + row[10]) % nd;
    const double w[5] = {fma(t, row[4], row[0]), fma(t, row[5], row[1]), fma(t, row[6], row[2]),
                         fma(t, row[7], row[3]), fma(t, row[9], row[8])};
    const double *b = Iin + ((size_t)i0 + (size_t)j0 * (size_t)nx) * (size_t)dp + (size_t)s;
    const size_t off[4] = {0, (size_t)dp, (size_t)nx * dp, (size_t)nx * dp + dp}; // 00 10 01 11
    double c[4];
#pragma unroll
    for (int k = 0; k < 4; k++)
    {
        const double *x = b + off[k];
        double v = w[0] * __ldg(x);
#pragma unroll
        for (int u = 1; u < 5; u++)
            v = fma(w[u], __ldg(x + u), v);
        c[k] = fmax(v, 0.0);
    }
    const double f0 = fma(fx, c[1] - c[0], c[0]);
    const double f1 = fma(fx, c[3] - c[2], c[2]);
    return r.w * fma(fy, f1 - f0, f0);
}

// One flat stream value from global memory (a departure more than a cell
// away: CFL above 1), from the departure's grid coordinates, corners clamped.
__device__ __noinline__ double stream_flat_far64(const double *__restrict__ Iin, double it, double jt, int dp, int nx,
                                                 int ny, int d)
{
    const int i0 = min(max((int)floor(it), 0), nx - 2);
    const int j0 = min(max((int)floor(jt), 0), ny - 2);
    const double fx = it - (double)i0, fy = jt - (double)j0;
    const double *b = Iin + ((size_t)i0 + (size_t)j0 * (size_t)nx) * (size_t)dp + (size_t)d;
    const double c00 = __ldg(b), c10 = __ldg(b + dp), c01 = __ldg(b + (size_t)nx * dp),
                 c11 = __ldg(b + (size_t)nx * dp + dp);
    const double f0 = fma(fx, c10 - c00, c00);
    const double f1 = fma(fx, c11 - c01, c01);
    return fma(fy, f1 - f0, f0);
}

// Stage the patch of `tile` into the warp's buffer: one tensor copy,
// completing on the warp's mbarrier.
__device__ __forceinline__ void stage_tile(const Step64Args &a, int tile, double *patch, unsigned bar)
{
    if ((threadIdx.x & 31) == 0)
    {
        const int bx = tile % a.tiles_x, by = tile / a.tiles_x;
        // the lanes' reads of the buffer are done (__syncwarp before the call)
        fence_proxy_async_smem();
        mbar_arrive_expect(bar, (unsigned)((a.tx + 2) * (a.ty + 2) * a.dps) * 8u);
        tma_load_4d(smem_addr(patch), &a.in_map, 0, 0, bx * a.tx, (int)a.g.jlo - 1 + by * a.ty, bar);
    }
}

// A tile's cells as phase 1 and phase 2 need them (lane c < 16 and its
// partner c + 16: cell c), and every lane its directions' records of cell 0;
// loaded for the next tile while the current one is finished.
template <int P>
struct UnitCells
{
    int x0, y0, txv, ncells;
    int cij, ccell, cpo, cfl;
    double u1, u2, lor, adt, eta, k0, k3, kak0, scale;
    double4 rec0[P];
};

template <bool CURVED, int P>
__device__ __forceinline__ void load_unit(const Step64Args &a, int tile, UnitCells<P> &U)
{
    const int lane = threadIdx.x & 31;
    const int tx = a.tx, px = tx + 2, nd = a.nd;
    const int bx = tile % a.tiles_x, by = tile / a.tiles_x;
    U.x0 = bx * tx;
    U.y0 = (int)a.g.jlo - 1 + by * a.ty;
    U.txv = min(tx, (int)a.g.nx_ - U.x0);
    U.ncells = U.txv * min(a.ty, (int)a.g.jhi - 1 - U.y0);
    const int c = lane & (kUnitCells - 1);
    const bool cact = c < U.ncells;
    const int ccx = cact ? c % U.txv : 0, ccy = cact ? c / U.txv : 0;
    U.cij = (1 + U.x0 + ccx) + (1 + U.y0 + ccy) * (int)a.g.nx;
    U.ccell = (U.x0 + ccx) + (U.y0 + ccy) * (int)a.g.nx_;
    U.cpo = (ccy * px + ccx) * a.dps;
    U.cfl = cact ? (int)a.flags[U.cij] : 3;
    U.u1 = __ldg(a.u1 + U.cij), U.u2 = __ldg(a.u2 + U.cij), U.lor = __ldg(a.lor + U.cij);
    U.adt = __ldg(a.adt + U.cij), U.eta = __ldg(a.eta + U.cij), U.k0 = __ldg(a.k0 + U.cij);
    U.k3 = __ldg(a.k3 + U.cij), U.kak0 = __ldg(a.ka + U.cij) + U.k0;
    U.scale = CURVED ? __ldg(a.ia3 + U.cij) : 1.0;
    if (CURVED)
    {
        const int cell0 = __shfl_sync(0xffffffffu, U.ccell, 0);
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            U.rec0[p] = d < nd ? ld_once(a.rec + (size_t)cell0 * (size_t)nd + (size_t)d) : make_double4(0, 0, 0, 0);
        }
#pragma unroll
        for (int k = 1; k < 4; k++)
        {
            const int cell = __shfl_sync(0xffffffffu, U.ccell, k);
#pragma unroll
            for (int p = 0; p < P; p++)
            {
                const int d = lane + 32 * p;
                if (k < U.ncells && d < nd)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.rec + (size_t)cell * (size_t)nd + (size_t)d));
            }
        }
    }
}

// One tile of one step by one warp, its patch staged (see the file comment).
// S: [cell][direction], row stride a.ss.  next() stages the next tile.
template <bool CURVED, int P, class Next>
__device__ __forceinline__ void step_unit64(const Step64Args &a, const DirTable64 &dt, const double *rowtab,
                                            const double *dirc, const double2 (&LN)[P], const UnitCells<P> &U,
                                            const double *patch, double *S, step::IterStats &st, Next next)
{
    const int lane = threadIdx.x & 31;
    const int px = a.tx + 2, dp = a.dp, dps = a.dps, nd = a.nd, ss = a.ss;
    const int nxn = (int)a.g.nx, nx_ = (int)a.g.nx_;
    const size_t nxy = (size_t)a.g.nxy;
    const int ncells = U.ncells;
    const int pdp = px * dps; // patch offset of the next node row
    const int c = lane & (kUnitCells - 1), h = lane >> 4;
    const bool cact = c < ncells;
    const int cij = U.cij, ccell = U.ccell, cpo = U.cpo, cfl = U.cfl;
    const double u1 = U.u1, u2 = U.u2, lor = U.lor, adt = U.adt, eta = U.eta, k0 = U.k0, k3 = U.k3, kak0 = U.kak0;
    const double scale = U.scale;

    // ---- phase 1: stream every cell, lanes over the directions ----
    double4 rc[P], rn[P];
    auto load_recs = [&](double4(&r)[P], int cell) {
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            r[p] = d < nd ? ld_once(a.rec + (size_t)cell * (size_t)nd + (size_t)d) : make_double4(0, 0, 0, 0);
        }
    };
    auto prefetch_recs = [&](int cell) {
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            if (d < nd)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(a.rec + (size_t)cell * (size_t)nd + (size_t)d));
        }
    };
    if (CURVED)
    {
#pragma unroll
        for (int p = 0; p < P; p++)
            rc[p] = U.rec0[p];
    }
    for (int k = 0; k < ncells; k++)
    {
        const int cell1 = __shfl_sync(0xffffffffu, ccell, (k + 1) & 15);
        const int cell4 = __shfl_sync(0xffffffffu, ccell, (k + 4) & 15);
        const int ijk = __shfl_sync(0xffffffffu, cij, k);
        const int pok = __shfl_sync(0xffffffffu, cpo, k);
        const int flk = __shfl_sync(0xffffffffu, cfl, k);
        if (CURVED)
        {
            if (k + 1 < ncells)
                load_recs(rn, cell1);
            if (k + 4 < ncells)
                prefetch_recs(cell4);
        }
        const double *cellp = patch + pok; // node (i - 1, j - 1) of cell k
        double *Sk = S + k * ss;
        double v[P], fit[P], fjt[P]; // fit, fjt: a flat departure's grid coordinates
        bool far[P];
#pragma unroll
        for (int p = 0; p < P; p++)
            v[p] = fit[p] = fjt[p] = 0.0, far[p] = false;
        const int i = ijk % nxn, j = ijk / nxn;
        if (!(CURVED && (flk & 2))) // a cell inside the excision streams zeros
        {
            // the flat departure's grid coordinates, rounded as the reference's
            // xy(i, j) - c dt, then grid.i() / grid.j() (src/Radiation.cpp:394-402)
            double xi = 0.0, yj = 0.0;
            if (!CURVED)
            {
                xi = __dadd_rn(a.g.startx, __dmul_rn((double)i, a.g.dx));
                yj = __dadd_rn(a.g.starty, __dmul_rn((double)j, a.g.dy));
            }
#pragma unroll
            for (int p = 0; p < P; p++)
            {
                if (CURVED)
                {
                    const double4 r = rc[p];
                    const unsigned hx = hi_word(r.x), hy = hi_word(r.y), hz = hi_word(r.z), hw = hi_word(r.w);
                    far[p] = (hw >> 31) != 0;
                    const double fx = unbias(r.x), fy = unbias(r.y), t = unbias(r.z);
                    const double *row = rowtab + ((hx >> packed64::kExpShift) & 31u) * 12;
                    const double w0 = fma(t, row[4], row[0]), w1 = fma(t, row[5], row[1]);
                    const double w2 = fma(t, row[6], row[2]), w3 = fma(t, row[7], row[3]);
                    const double w4 = fma(t, row[9], row[8]);
                    const int s = (int)((hz >> packed64::kExpShift) & 255u);
                    const double *p00 = cellp + (int)(hx >> 31) * dps + (int)(hy >> 31) * pdp + s;
                    const double c00 = window5(p00, w0, w1, w2, w3, w4);
                    const double c10 = window5(p00 + dps, w0, w1, w2, w3, w4);
                    const double c01 = window5(p00 + pdp, w0, w1, w2, w3, w4);
                    const double c11 = window5(p00 + pdp + dps, w0, w1, w2, w3, w4);
                    const double f0 = fma(fx, c10 - c00, c00);
                    const double f1 = fma(fx, c11 - c01, c01);
                    v[p] = __hiloint2double((int)(hw & 0x7fffffffu), __double2loint(r.w)) * fma(fy, f1 - f0, f0);
                }
                else
                {
                    const int d = min(lane + 32 * p, nd - 1);
                    const double it = __ddiv_rn(__dsub_rn(__dsub_rn(xi, dt.cxdt[d]), a.g.startx), a.g.dx);
                    const double jt = __ddiv_rn(__dsub_rn(__dsub_rn(yj, dt.cydt[d]), a.g.starty), a.g.dy);
                    const int i0 = min(max((int)floor(it), 0), nxn - 2);
                    const int j0 = min(max((int)floor(jt), 0), (int)a.g.ny - 2);
                    const int ci = i0 - (i - 1), cj = j0 - (j - 1);
                    far[p] = !((unsigned)ci <= 1u && (unsigned)cj <= 1u);
                    const double *b = cellp + (far[p] ? 0 : ci * dps + cj * pdp) + d;
                    const double fx = it - (double)i0, fy = jt - (double)j0;
                    const double c00 = b[0], c10 = b[dps], c01 = b[pdp], c11 = b[pdp + dps];
                    const double f0 = fma(fx, c10 - c00, c00);
                    const double f1 = fma(fx, c11 - c01, c01);
                    v[p] = fma(fy, f1 - f0, f0);
                    fit[p] = it;
                    fjt[p] = jt;
                }
            }
            // departures outside the 3x3 neighbourhood (rare): from global memory
            bool any = false;
#pragma unroll
            for (int p = 0; p < P; p++)
                any |= far[p];
            if (__any_sync(0xffffffffu, any))
            {
                const int cell = (i - 1) + (j - 1) * nx_;
#pragma unroll
                for (int p = 0; p < P; p++)
                {
                    const int d = lane + 32 * p;
                    if (far[p] && d < nd)
                        v[p] = CURVED ? stream_far64(a.Iin, ld_ro(a.side + (size_t)cell * (size_t)nd + (size_t)d), dp,
                                                     nxn, (int)a.g.ny, nd, a.ng, rowtab, dt.q, dt.p, dt.inv_q, i, j)
                                      : stream_flat_far64(a.Iin, fit[p], fjt[p], dp, nxn, (int)a.g.ny, d);
                }
            }
        }
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            if (d < nd)
                Sk[d] = v[p];
        }
        if (CURVED)
        {
#pragma unroll
            for (int p = 0; p < P; p++)
                rc[p] = rn[p];
        }
    }
    __syncwarp();
    next(); // the patch buffer is free: the next tile's copy lands during phases 2 and 3

    // ---- phase 2: moments and collide, two lanes per cell ----
    // phase 3's map of the streamed values of this lane's cell: og S + oa +
    // ob1 n1 + ob2 n2 (identity where phase 2 has written the values already)
    double og = 1.0, oa = 0.0, ob1 = 0.0, ob2 = 0.0;
    if (cact)
    {
        const unsigned pair = 0x10001u << c; // the two lanes of this cell
        double *Sc = S + c * ss;
        double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int d = h; d < nd; d += 2)
        {
            const double v = Sc[d];
            const double *cf = dirc + 8 * d;
#pragma unroll
            for (int q = 0; q < 6; q++)
                m[q] = fma(cf[q], v, m[q]);
        }
        // a + b == b + a: both lanes hold the same moments
#pragma unroll
        for (int q = 0; q < 6; q++)
            m[q] += __shfl_xor_sync(pair, m[q], 16);
        const bool collides = !(cfl & 1);
        if (collides)
        {
            int cycles = 0;
            const bool rest = (u1 == 0.0) && (u2 == 0.0);
            // m_new[q] = A[q] + (eta + k0 fE) B[q] + k3 (fFx C[q] + fFy D[q])
            double A6[6], B6[6], C6[6], D6[6];
            double g0 = 0.0, h0 = 0.0;
            if (rest)
            {
                g0 = 1.0 / (1.0 + adt * kak0);
                h0 = adt * g0;
#pragma unroll
                for (int q = 0; q < 6; q++)
                {
                    A6[q] = g0 * m[q];
                    B6[q] = h0 * dt.wmom[q];
                    C6[q] = h0 * dt.wmom[6 + q];
                    D6[q] = h0 * dt.wmom[12 + q];
                }
            }
            else
            {
#pragma unroll
                for (int q = 0; q < 6; q++)
                    A6[q] = B6[q] = C6[q] = D6[q] = 0.0;
                for (int d = h; d < nd; d += 2)
                {
                    const double *cf = dirc + 8 * d;
                    const double n1 = cf[6], n2 = cf[7], w = cf[0];
                    double g, hh, q1, q2;
                    collide_coeffs64(n1, n2, u1, u2, lor, adt, kak0, g, hh, q1, q2);
                    const double mu[6] = {1.0, n1, n2, n1 * n1, n1 * n2, n2 * n2};
                    const double gs = w * g * Sc[d], wh = w * hh;
#pragma unroll
                    for (int q = 0; q < 6; q++)
                    {
                        A6[q] = fma(gs, mu[q], A6[q]);
                        B6[q] = fma(wh, mu[q], B6[q]);
                        C6[q] = fma(wh * q1, mu[q], C6[q]);
                        D6[q] = fma(wh * q2, mu[q], D6[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < 6; q++)
                {
                    A6[q] += __shfl_xor_sync(pair, A6[q], 16);
                    B6[q] += __shfl_xor_sync(pair, B6[q], 16);
                    C6[q] += __shfl_xor_sync(pair, C6[q], 16);
                    D6[q] += __shfl_xor_sync(pair, D6[q], 16);
                }
            }
            double diff = 1.0;
            double fE = 0.0, fFx = 0.0, fFy = 0.0;
            while (fabs(diff) > 1e-4 && cycles < 100)
            {
                cycles++;
                const double pE = m[0], pFx = m[1], pFy = m[2], pPxx = m[3], pPxy = m[4], pPyy = m[5];
                const double uF = u1 * pFx + u2 * pFy;
                const double uxP = u1 * pPxx + u2 * pPxy;
                const double uyP = u1 * pPxy + u2 * pPyy;
                const double uuP = u1 * uxP + u2 * uyP;
                fE = lor * lor * (pE - 2.0 * uF + uuP);
                const double rr = lor / (1.0 + lor) * ((2.0 * lor + 1.0) * uF - lor * uuP);
                fFx = lor * lor * (pFx - lor * pE * u1 - uxP + u1 * rr);
                fFy = lor * lor * (pFy - lor * pE * u2 - uyP + u2 * rr);
                const double ee = eta + k0 * fE;
                const double prev[6] = {pE, pFx, pFy, pPxx, pPxy, pPyy};
                double s2 = 0.0;
#pragma unroll
                for (int q = 0; q < 6; q++)
                {
                    m[q] = A6[q] + ee * B6[q] + k3 * (fFx * C6[q] + fFy * D6[q]);
                    // the reference's relative change (0 / 0 is NaN and ends the iteration)
                    const double x = (prev[q] - m[q]) / m[q];
                    s2 += x * x;
                }
                diff = sqrt(s2);
            }
            // the intensities of the last iterate (its moments m are the stored
            // ones): at rest the affine map phase 3 applies; a moving fluid's here
            const double ee = eta + k0 * fE;
            if (rest)
            {
                og = g0 * scale;
                oa = h0 * ee * scale;
                ob1 = h0 * k3 * fFx * scale;
                ob2 = h0 * k3 * fFy * scale;
            }
            else
            {
                for (int d = h; d < nd; d += 2)
                {
                    const double *cf = dirc + 8 * d;
                    const double n1 = cf[6], n2 = cf[7];
                    double g, hh, q1, q2;
                    collide_coeffs64(n1, n2, u1, u2, lor, adt, kak0, g, hh, q1, q2);
                    Sc[d] = (g * Sc[d] + hh * (ee + k3 * (q1 * fFx + q2 * fFy))) * scale;
                }
            }
            if (h == 0)
            {
                st.sum += (unsigned)cycles;
                st.max = max(st.max, (unsigned)cycles);
            }
        }
        else
            og = scale;
#pragma unroll
        for (int q = 0; q < 3; q++)
            a.mom[(size_t)cij + (size_t)(3 * h + q) * nxy] = h ? m[3 + q] : m[q];
    }
    __syncwarp();

    // ---- phase 3: the cells' new state, coalesced along the directions
    // (and the mirrored directions 0..3 after the last one) ----
    for (int k = 0; k < ncells; k++)
    {
        const int ij = __shfl_sync(0xffffffffu, cij, k);
        const double g = __shfl_sync(0xffffffffu, og, k), ca = __shfl_sync(0xffffffffu, oa, k);
        const double cb1 = __shfl_sync(0xffffffffu, ob1, k), cb2 = __shfl_sync(0xffffffffu, ob2, k);
        double *o = a.Iout + (size_t)ij * (size_t)dp;
        const double *Sk = S + k * ss;
        double first = 0.0;
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            const double val = fma(g, Sk[min(d, nd - 1)], fma(cb1, LN[p].x, fma(cb2, LN[p].y, ca)));
            if (d < nd)
                o[d] = val;
            if (p == 0)
                first = val;
        }
        if (lane < kStateMirror)
            o[nd + lane] = first;
    }
    __syncwarp(); // S is rewritten by the next tile's phase 1
}

// shared layout: mbarriers, rows (q x 12), direction coefficients (nd x 8)
__device__ __forceinline__ int step64_header(int nd, int q) { return kTablesOffset + (q * 12 + nd * 8) * 8; }

template <bool CURVED, int P>
__global__ void __launch_bounds__(kThreads, P == 1 ? GRLBM_STEP64_MIN_BLOCKS_1 : GRLBM_STEP64_MIN_BLOCKS)
    k_step_fast64(const __grid_constant__ Step64Args a, const DirTable64 *__restrict__ dtp, int warp_stride)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const DirTable64 &dt = *dtp;
    const int q = CURVED ? a.q : 0;
    double *rowtab = reinterpret_cast<double *>(smem + kTablesOffset);
    double *dirc = rowtab + q * 12;
    const unsigned bar = smem_addr(smem) + 8u * (unsigned)(threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0)
        mbar_init(bar, 1);
    for (int k = threadIdx.x; k < q * 12; k += kThreads)
        rowtab[k] = dt.rowtab[k];
    for (int k = threadIdx.x; k < 8 * a.nd; k += kThreads)
        dirc[k] = dt.dirc[k];
    __syncthreads();
    double *patch = step::warp_buffers<double>(smem, step64_header(a.nd, q), warp_stride);
    double *S = patch + a.patch_elems;
    const int lane = threadIdx.x & 31;
    double2 LN[P];
#pragma unroll
    for (int p = 0; p < P; p++)
    {
        const double *cf = dirc + 8 * min(lane + 32 * p, a.nd - 1);
        LN[p] = make_double2(cf[6], cf[7]);
    }
    step::IterStats st{0ull, 0u};
    unsigned parity = 0;
    int tile = step::take_tile(a.tiles);
    UnitCells<P> U;
    if (tile < a.ntiles)
    {
        stage_tile(a, tile, patch, bar);
        load_unit<CURVED, P>(a, tile, U);
    }
    while (tile < a.ntiles)
    {
        if (!step::wait_tile(bar, parity, a.fault))
            break;
        int next = a.ntiles;
        UnitCells<P> N;
        step_unit64<CURVED, P>(a, dt, rowtab, dirc, LN, U, patch, S, st, [&]() {
            next = step::take_tile(a.tiles);
            if (next < a.ntiles)
            {
                stage_tile(a, next, patch, bar);
                load_unit<CURVED, P>(a, next, N);
            }
        });
        U = N;
        tile = next;
    }
    step::flush_stats(st, a.iter_sum, a.iter_max);
    step::retire_warp(a.tiles, kWarps);
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

constexpr int kPassSet[] = {1, 2, 3, 4, 6, 8};
} // namespace

int step64_passes(int nd)
{
    const int need = (nd + 31) / 32;
    for (int p : kPassSet)
        if (p >= need)
            return p;
    return -1;
}

// row stride of the streamed values: >= nd and 1 mod 16 doubles, so that the
// 16 cells of a half-warp in phase 2 read disjoint banks
int step64_s_stride(int nd) { return nd + ((1 - nd) % 16 + 16) % 16; }

int step64_patch_node_elems(int dp)
{
    const int padded = (dp + 15) / 16 * 16;
    return padded <= 256 ? padded : dp;
}

static int step64_patch_elems(int tx, int ty, int dp) { return ((tx + 2) * (ty + 2) * step64_patch_node_elems(dp) + 15) / 16 * 16; }

int step64_warp_stride(int tx, int ty, int dp, int nd)
{
    return ((step64_patch_elems(tx, ty, dp) + kUnitCells * step64_s_stride(nd)) * 8 + 127) / 128 * 128;
}

size_t step64_smem(int tx, int ty, int dp, int nd, int q)
{
    return (size_t)kTablesOffset + (size_t)(q * 12 + nd * 8) * 8 + 128 +
           (size_t)kWarps * (size_t)step64_warp_stride(tx, ty, dp, nd);
}

cudaError_t prepare_step64()
{
    cudaError_t e = cudaSuccess;
#define GRLBM_PREP(P)                                                                                      \
    if (e == cudaSuccess)                                                                                  \
        e = cudaFuncSetAttribute(k_step_fast64<true, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                 kStep32MaxSmem);                                                          \
    if (e == cudaSuccess)                                                                                  \
        e = cudaFuncSetAttribute(k_step_fast64<false, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                 kStep32MaxSmem);
    GRLBM_PREP(1)
    GRLBM_PREP(2)
    GRLBM_PREP(3)
    GRLBM_PREP(4)
    GRLBM_PREP(6)
    GRLBM_PREP(8)
#undef GRLBM_PREP
    return e;
}

cudaError_t step64_occupancy(int P, bool curved, size_t smem, int *blocks)
{
    const void *f = nullptr;
#define GRLBM_PICK(PP)                                                                                     \
    if (P == PP)                                                                                           \
        f = curved ? (const void *)k_step_fast64<true, PP> : (const void *)k_step_fast64<false, PP>;
    GRLBM_PICK(1)
    GRLBM_PICK(2)
    GRLBM_PICK(3)
    GRLBM_PICK(4)
    GRLBM_PICK(6)
    GRLBM_PICK(8)
#undef GRLBM_PICK
    if (!f)
        return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, f, kThreads, smem);
}

void launch_step64(const Step64Args &a, const DirTable64 *dt, bool curved, int P, int blocks, cudaStream_t s)
{
    if (a.ntiles <= 0)
        return;
    // the flat kernel reads no row types
    const size_t smem = step64_smem(a.tx, a.ty, a.dp, a.nd, curved ? a.q : 0);
    const int stride = step64_warp_stride(a.tx, a.ty, a.dp, a.nd);
    const unsigned grid = (unsigned)std::max(1, std::min(blocks, (int)nblk(a.ntiles, kWarps)));
#define GRLBM_LAUNCH(PP)                                                                                   \
    if (P == PP)                                                                                           \
    {                                                                                                      \
        if (curved)                                                                                        \
            k_step_fast64<true, PP><<<grid, kThreads, smem, s>>>(a, dt, stride);                           \
        else                                                                                               \
            k_step_fast64<false, PP><<<grid, kThreads, smem, s>>>(a, dt, stride);                          \
        return;                                                                                            \
    }
    GRLBM_LAUNCH(1)
    GRLBM_LAUNCH(2)
    GRLBM_LAUNCH(3)
    GRLBM_LAUNCH(4)
    GRLBM_LAUNCH(6)
    GRLBM_LAUNCH(8)
#undef GRLBM_LAUNCH
}

// The cell-major FP64 state as a 4D tensor {c0, dp / c0, nx, ny} read in
// boxes {box0, dp / c0, tx + 2, ty + 2}: one box is a tile's whole patch,
// landing in shared memory as [node row][node][direction].  When dp is at
// most 256, c0 = dp and the box's first extent is the padded node run
// (step64_patch_node_elems: its doubles past dp are the copy's zero fill);
// else c0 is the largest even divisor of dp up to 256 and the run is not
// padded.
cudaError_t encode_state_map64(CUtensorMap *map, const double *state, int64_t nx, int64_t ny, int dp, int tx, int ty)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode)
    {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e =
            cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
        if (e != cudaSuccess)
            return e;
        if (q != cudaDriverEntryPointSuccess || !fn)
            return cudaErrorNotSupported;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if (dp % 2 != 0 || reinterpret_cast<uintptr_t>(state) % 16 != 0 || tx < 1 || ty < 1 || tx + 2 > 256 ||
        ty + 2 > 256)
        return cudaErrorInvalidValue;
    int c0 = 0, box0 = 0;
    if (dp <= 256)
        c0 = dp, box0 = step64_patch_node_elems(dp);
    else
    {
        for (int c = 2; c <= 256 && c <= dp; c += 2)
            if (dp % c == 0)
                c0 = c;
        box0 = c0;
    }
    if (c0 == 0 || dp / c0 > 256 || (box0 != c0 && dp / c0 != 1))
        return cudaErrorInvalidValue;
    const cuuint64_t dims[4] = {(cuuint64_t)c0, (cuuint64_t)(dp / c0), (cuuint64_t)nx, (cuuint64_t)ny};
    const cuuint64_t strides[3] = {(cuuint64_t)c0 * sizeof(double), (cuuint64_t)dp * sizeof(double),
                                   (cuuint64_t)nx * (cuuint64_t)dp * sizeof(double)};
    const cuuint32_t box[4] = {(cuuint32_t)box0, (cuuint32_t)(dp / c0), (cuuint32_t)(tx + 2), (cuuint32_t)(ty + 2)};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double *>(state), dims, strides,
                              box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
} // namespace grlbm
