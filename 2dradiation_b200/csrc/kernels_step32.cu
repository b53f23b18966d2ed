// Precision-form step of the fixed streaming types (StreamFlatFixed and
// StreamCurvedFixed with IntensityAt, then ComputeMomentsIF and Collide;
// src/Radiation.cpp:380-414, 454-512, 322-343, 239-269, 641-736) on the
// cell-major FP32 state.
//
// State: J[(i + j nx) dp + d], directions fastest, with directions 0..3
// repeated after the last one (dp = nd + 4 rounded up to 4 floats), so that
// every 5-direction angular window of a node is one contiguous run.  For
// curved streaming J = I / alpha^3: the reference multiplies each corner's
// angular interpolation by (alpha_c / alpha_n)^3 after clamping it at zero
// (src/Radiation.cpp:502-505, 342); alpha_n^-3 > 0 commutes with the clamp,
// so gathering J needs no alpha at the corners.
//
// In shared memory a node's run is padded to dps floats, a multiple of 32
// (the TMA box is wider than the node's dp floats; the rest is zero fill):
// lanes whose departures fall in different corner columns or rows then read
// disjoint banks.  (Half-warp mode pads to 16 mod 32 instead; see
// step32_patch_node_floats.)
//
// Work split: every warp works alone.  It takes tiles of tx x ty <= 16 cells
// from a counter and stages the tile's (tx + 2) x (ty + 2) node patch of the
// whole state (all directions) into its own shared-memory buffer with one TMA
// tensor copy.  Phase 1 streams the tile's cells one after another with the
// lanes over the directions (direction d = lane + 32 p on pass p), into the
// warp's buffer of streamed values; the next tile's copy is then issued into
// the free patch buffer, to land while phase 2 takes the moments and collides
// with two lanes per cell (each summing every other direction), and phase 3
// writes the cells' new state, coalesced along the directions.
//
// Per (cell, direction) the lane reads its 16-byte packed departure record
// (window row type, window start, blend t, corner fractions with the corner in
// their sign bits, s^3 alpha_c^3 with the far flag in its sign bit), takes the
// window's weights W0 + t D from the row-type table, gathers the 5-tap window
// at the 4 bilinear corners from the patch (contiguous runs), clamps each at
// zero and interpolates.  Departures outside the cell's 3x3 neighbourhood read
// a side record and gather from global memory (cold code).
//
// Moments: each of a cell's two lanes sums its directions in FP32 chunks of 8
// folded into Kahan accumulators; the two lanes' compensated sums are
// combined by an exact two-sum, so both hold the same moments.
//
// Collide: the lambda iteration of src/Radiation.cpp:661-722 is affine in
// the previous moments -- I_d = g_d S_d + h_d (eta + kappa0 E_ff + 3 kappa1
// nFF_d . F_ff) -- so each iteration runs on the six moments (the same scalar
// work on every lane); the last iterate's moments, the affine map's moments of
// exactly the written intensities, are the stored ones.
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>

#include "device_common.cuh"
#include "step_common.cuh"

// resident blocks per SM the single-problem kernel is compiled for: three
// at one pass (at most 112 registers; 16 and 32 directions step 8-12% faster
// than at two blocks), two at more passes (at three their registers spill)
#ifndef GRLBM_STEP32_MIN_BLOCKS
#define GRLBM_STEP32_MIN_BLOCKS 2
#endif
#ifndef GRLBM_STEP32_MIN_BLOCKS_1
#define GRLBM_STEP32_MIN_BLOCKS_1 3
#endif

namespace grlbm
{
namespace
{
constexpr int kWarps = kStep32Warps;
constexpr int kUnitCells = kStep32UnitCells;
constexpr int kThreads = 32 * kWarps;
// shared layout: the warps' mbarriers, the row-type table and the direction
// coefficients (single-problem kernel), then the warps' buffers from the next
// 128-byte boundary
constexpr int kBarBytes = 8 * kWarps;
constexpr int kRowtabOffset = 64;
static_assert(kBarBytes <= kRowtabOffset, "mbarriers before the row-type table");
static_assert(kUnitCells == 16, "phase 2 pairs lane c and lane c + 16");

// direction coefficients of the affine collide map for a moving fluid
__device__ __forceinline__ void collide_coeffs32(float n1, float n2, float u1, float u2, float lor, float adt,
                                                 float kak0, float &g, float &h, float &q1, float &q2)
{
    const float un = u1 * n1 + u2 * n2;
    const float A = lor * (1.f - un);
    const float sc = (1.f - (lor * un) / (lor + 1.f)) * lor;
    q1 = (n1 - sc * u1) / A;
    q2 = (n2 - sc * u2) / A;
    g = 1.f / (1.f + adt * kak0 * A);
    h = adt / (A * A) * g;
}

// One curved stream value from global memory, for a departure outside the
// cell's 3x3 neighbourhood: the side record {i_dep - i, j_dep - j, angle
// coordinate, s^3 alpha_c^3}, corners clamped to the grid as the reference's
// gather would index them (cold code, kept out of line).
__device__ __noinline__ float stream_far32(const float *__restrict__ Iin, float4 r, int dp, int nx, int ny, int nd,
                                           int ng, const float *rowtab, int q, int p, float inv_q, int i, int j)
{
    const float fli = floorf(r.x), flj = floorf(r.y);
    const float fx = r.x - fli, fy = r.y - flj;
    const int i0 = min(max(i + (int)fli, 0), nx - 2);
    const int j0 = min(max(j + (int)flj, 0), ny - 2);
    const float z = r.z == r.z ? r.z : 0.f;
    const float g = fminf(fmaxf(floorf(z), 0.f), (float)(ng - 1));
    const float t = fminf(fmaxf(z - g, 0.f), 1.f);
    const float m = floorf((g + 0.5f) * inv_q);
    const int rt = min(max((int)fmaf(-m, (float)q, g), 0), q - 1);
    const float *row = rowtab + rt * 12;
    const int s = (int)fmaf(m, (float)p, row[10]) % nd;
    const float w[5] = {fmaf(t, row[4], row[0]), fmaf(t, row[5], row[1]), fmaf(t, row[6], row[2]),
                        fmaf(t, row[7], row[3]), fmaf(t, row[9], row[8])};
    const float *b = Iin + ((unsigned)i0 + (unsigned)j0 * (unsigned)nx) * (unsigned)dp + (unsigned)s;
    const unsigned off[4] = {0u, (unsigned)dp, (unsigned)(nx * dp), (unsigned)(nx * dp + dp)}; // 00 10 01 11
    float c[4];
#pragma unroll
    for (int k = 0; k < 4; k++)
    {
        const float *x = b + off[k];
        float v = w[0] * __ldg(x);
#pragma unroll
        for (int u = 1; u < 5; u++)
            v = fmaf(w[u], __ldg(x + u), v);
        c[k] = fmaxf(v, 0.f);
    }
    const float f0 = fmaf(fx, c[1] - c[0], c[0]);
    const float f1 = fmaf(fx, c[3] - c[2], c[2]);
    return r.w * fmaf(fy, f1 - f0, f0);
}

// One flat stream value from global memory (a departure more than a cell
// away: CFL above 1), corners clamped to the grid.
__device__ __noinline__ float stream_flat_far32(const float *__restrict__ Iin, float ox, float oy, int dp, int nx,
                                                int ny, int d, int i, int j)
{
    const float fli = floorf(ox), flj = floorf(oy);
    const float fx = ox - fli, fy = oy - flj;
    const int i0 = min(max(i + (int)fli, 0), nx - 2);
    const int j0 = min(max(j + (int)flj, 0), ny - 2);
    const float *b = Iin + ((unsigned)i0 + (unsigned)j0 * (unsigned)nx) * (unsigned)dp + (unsigned)d;
    const float c00 = __ldg(b), c10 = __ldg(b + dp), c01 = __ldg(b + nx * dp), c11 = __ldg(b + nx * dp + dp);
    const float f0 = fmaf(fx, c10 - c00, c00);
    const float f1 = fmaf(fx, c11 - c01, c01);
    return fmaf(fy, f1 - f0, f0);
}

// The 5-tap angular window at one corner, clamped at zero.
__device__ __forceinline__ float window5(const float *p, float w0, float w1, float w2, float w3, float w4)
{
    return fmaxf(fmaf(w4, p[4], fmaf(w3, p[3], fmaf(w2, p[2], fmaf(w1, p[1], w0 * p[0])))), 0.f);
}

// The direction of a lane's first pass: the lane, or in half-warp mode (H:
// at most 16 directions, the two half-warps on two cells) the lane within its
// half-warp.
template <bool H>
__device__ __forceinline__ int lane_dir()
{
    return H ? (int)(threadIdx.x & 15) : (int)(threadIdx.x & 31);
}

// A lane's per-direction constants of flat streaming for its P passes (of PM
// stored): the departure's corner offset in the patch, its fractions and
// whether it lies within the 3x3 neighbourhood (else the far gather).
template <int PM>
struct LaneFlat
{
    float ox[PM], oy[PM], fx[PM], fy[PM];
    int off[PM];
    bool near[PM];
};

template <int P, bool H, int PM>
__device__ __forceinline__ void load_lane_flat(LaneFlat<PM> &L, const DirTable &dt, int nd, int dps, int px)
{
    const int dl = lane_dir<H>();
#pragma unroll
    for (int p = 0; p < P; p++)
    {
        const int dd = min(dl + 32 * p, nd - 1);
        const float ox = dt.ox[dd], oy = dt.oy[dd];
        const float fli = floorf(ox), flj = floorf(oy);
        L.ox[p] = ox;
        L.oy[p] = oy;
        L.fx[p] = ox - fli;
        L.fy[p] = oy - flj;
        L.near[p] = (fli == -1.f || fli == 0.f) && (flj == -1.f || flj == 0.f);
        L.off[p] = L.near[p] ? ((int)fli + 1 + ((int)flj + 1) * px) * dps + dd : 0;
    }
}

// A lane's rotated directions (n1, n2) for its P passes (phase 3's map).
template <int P, bool H, int PM>
__device__ __forceinline__ void load_lane_dirs(float2 (&LN)[PM], const float4 *dirc, int nd)
{
    const int dl = lane_dir<H>();
#pragma unroll
    for (int p = 0; p < P; p++)
    {
        const float4 c1 = dirc[2 * min(dl + 32 * p, nd - 1) + 1];
        LN[p] = make_float2(c1.z, c1.w);
    }
}

// Stage the patch of `tile` (node origin x0 = bx tx, y0 = jlo - 1 + by ty)
// into the warp's buffer: one tensor copy, completing on the warp's mbarrier.
__device__ __forceinline__ void stage_tile(const Step32Args &a, int tile, float *patch, unsigned bar)
{
    if ((threadIdx.x & 31) == 0)
    {
        const int bx = tile % a.tiles_x, by = tile / a.tiles_x;
        // the lanes' reads of the buffer are done (__syncwarp before the call)
        fence_proxy_async_smem();
        mbar_arrive_expect(bar, (unsigned)((a.tx + 2) * (a.ty + 2) * a.dps) * 4u);
        tma_load_4d(smem_addr(patch), &a.in_map, 0, 0, bx * a.tx, (int)a.g.jlo - 1 + by * a.ty, bar);
    }
}

// A tile's cells as phase 1 and phase 2 need them: lane c (< 16, and its
// partner c + 16) holds cell c's node index, interior cell index, patch
// offset, flags and fields; and every lane its directions' records of its
// first cell (cell 0, or in half-warp mode cell 0 or 1 by half-warp).
// Loaded for the next tile while the current one is finished, so that none
// of these loads stalls the streaming.  rec0 has room for PM passes.
template <int PM>
struct UnitCells
{
    int x0, y0, txv, ncells;
    int cij, ccell, cpo, cfl;
    float u1, u2, lor, adt, eta, k0, k3, kak0, scale;
    uint4 rec0[PM];
};

template <bool CURVED, int P, bool H, int PM>
__device__ __forceinline__ void load_unit(const Step32Args &a, int tile, UnitCells<PM> &U)
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
    // (fields exist at every node: loaded without waiting for the flags)
    U.u1 = __ldg(a.u1 + U.cij), U.u2 = __ldg(a.u2 + U.cij), U.lor = __ldg(a.lor + U.cij);
    U.adt = __ldg(a.adt + U.cij), U.eta = __ldg(a.eta + U.cij), U.k0 = __ldg(a.k0 + U.cij);
    U.k3 = __ldg(a.k3 + U.cij), U.kak0 = __ldg(a.ka + U.cij) + U.k0;
    U.scale = CURVED ? __ldg(a.ia3 + U.cij) : 1.f;
    if (CURVED)
    {
        constexpr int kStep = H ? 2 : 1;
        const int dl = lane_dir<H>(), hk = H ? (lane >> 4) : 0;
        const int cell0 = __shfl_sync(0xffffffffu, U.ccell, hk);
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = dl + 32 * p;
            U.rec0[p] = d < nd && hk < U.ncells ? __ldcs(a.rec + (unsigned)cell0 * (unsigned)nd + (unsigned)d)
                                                : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int m = 1; m < 4; m++)
        {
            const int k = m * kStep + hk;
            const int cell = __shfl_sync(0xffffffffu, U.ccell, k & 15);
#pragma unroll
            for (int p = 0; p < P; p++)
            {
                const int d = dl + 32 * p;
                if (k < U.ncells && d < nd)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.rec + (unsigned)cell * (unsigned)nd + (unsigned)d));
            }
        }
    }
}

// One tile of one step by one warp, its patch staged: phase 1 streams every
// cell with the lanes over the directions into the warp's buffer S
// ([cell][direction], row stride a.ss), then calls next() (which stages the
// next tile into the patch buffer); phase 2 takes the moments and collides
// with two lanes per cell (lane = cell + 16 h, h the parity of the
// directions it sums), writing the collided values back into S; phase 3
// stores the cells' new state, coalesced along the directions.  In
// half-warp mode (H, at most 16 directions) phases 1 and 3 take two cells at
// a time, one per half-warp.  P passes of the PM the lane arrays hold.
template <bool CURVED, int P, bool H, int PM, class DT, class Next>
__device__ __forceinline__ void step_unit32(const Step32Args &a, const DT &dt, const float *rowtab,
                                            const float4 *dirc, const LaneFlat<PM> &LF, const float2 (&LN)[PM],
                                            const UnitCells<PM> &U, const float *patch, float *S,
                                            step::IterStats &st, Next next)
{
    static_assert(!H || P == 1, "half-warp mode streams at most 16 directions");
    constexpr int kStep = H ? 2 : 1; // cells per iteration of phases 1 and 3
    const int lane = threadIdx.x & 31;
    const int dl = lane_dir<H>(), hk = H ? (lane >> 4) : 0;
    const int tx = a.tx, px = tx + 2, dp = a.dp, dps = a.dps, nd = a.nd, ss = a.ss;
    (void)tx;
    const int nxn = (int)a.g.nx, nx_ = (int)a.g.nx_;
    const unsigned nxy = (unsigned)a.g.nxy;
    const int ncells = U.ncells;
    const int pdp = px * dps; // patch offset of the next node row
    const int c = lane & (kUnitCells - 1), h = lane >> 4;
    const bool cact = c < ncells;
    const int cij = U.cij, ccell = U.ccell, cpo = U.cpo, cfl = U.cfl;
    const float u1 = U.u1, u2 = U.u2, lor = U.lor, adt = U.adt, eta = U.eta, k0 = U.k0, k3 = U.k3, kak0 = U.kak0;
    const float scale = U.scale;

    // ---- phase 1: stream every cell, lanes over the directions ----
    // The cell loop reads the cells' tables from lanes 0..15 by shuffle.  A
    // lane's next cell's records are loaded while its current cell streams,
    // and those three cells on are prefetched into L2 (the first cell's came
    // with the tile's tables).
    uint4 rc[PM], rn[PM];
    auto load_recs = [&](uint4(&r)[PM], int cell) {
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = dl + 32 * p;
            r[p] = d < nd ? __ldcs(a.rec + (unsigned)cell * (unsigned)nd + (unsigned)d) : make_uint4(0u, 0u, 0u, 0u);
        }
    };
    auto prefetch_recs = [&](int cell) {
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = dl + 32 * p;
            if (d < nd)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(a.rec + (unsigned)cell * (unsigned)nd + (unsigned)d));
        }
    };
    if (CURVED)
    {
#pragma unroll
        for (int p = 0; p < P; p++)
            rc[p] = U.rec0[p];
    }
    for (int k0_ = 0; k0_ < ncells; k0_ += kStep)
    {
        const int k = k0_ + hk; // this lane's cell
        const bool kact = k < ncells;
        const int cell1 = __shfl_sync(0xffffffffu, ccell, (k + kStep) & 15);
        const int cell4 = __shfl_sync(0xffffffffu, ccell, (k + 4 * kStep) & 15);
        const int ijk = __shfl_sync(0xffffffffu, cij, k & 15);
        const int pok = __shfl_sync(0xffffffffu, cpo, k & 15);
        const int flk = __shfl_sync(0xffffffffu, cfl, k & 15);
        if (CURVED)
        {
            if (k + kStep < ncells)
                load_recs(rn, cell1);
            if (k + 4 * kStep < ncells)
                prefetch_recs(cell4);
        }
        const float *cellp = patch + pok; // node (i - 1, j - 1) of cell k
        float *Sk = S + k * ss;
        float v[PM];
        bool far[PM];
#pragma unroll
        for (int p = 0; p < P; p++)
            v[p] = 0.f, far[p] = false;
        if (kact && !(CURVED && (flk & 2))) // a cell inside the excision streams zeros
        {
            // every lane gathers (a direction past the last has a zero record: its
            // window reads valid patch nodes and is scaled by 0)
#pragma unroll
            for (int p = 0; p < P; p++)
            {
                if (CURVED)
                {
                    const uint4 r = rc[p];
                    far[p] = (r.w >> 31) != 0;
                    const unsigned word = r.x;
                    const float t = (float)(word & ((1u << packed32::kTBits) - 1u)) *
                                    (1.f / (float)(1u << packed32::kTBits));
                    const float4 *row =
                        reinterpret_cast<const float4 *>(rowtab + ((word >> packed32::kTypeShift) & 31u) * 12);
                    const float4 R0 = row[0], R1 = row[1], R2 = row[2];
                    const float w0 = fmaf(t, R1.x, R0.x), w1 = fmaf(t, R1.y, R0.y), w2 = fmaf(t, R1.z, R0.z);
                    const float w3 = fmaf(t, R1.w, R0.w), w4 = fmaf(t, R2.y, R2.x);
                    const int s = (int)((word >> packed32::kStartShift) & 255u);
                    const float *p00 = cellp + (int)(r.y >> 31) * dps + (int)(r.z >> 31) * pdp + s;
                    const float c00 = window5(p00, w0, w1, w2, w3, w4);
                    const float c10 = window5(p00 + dps, w0, w1, w2, w3, w4);
                    const float c01 = window5(p00 + pdp, w0, w1, w2, w3, w4);
                    const float c11 = window5(p00 + pdp + dps, w0, w1, w2, w3, w4);
                    const float fx = __uint_as_float(r.y & 0x7fffffffu), fy = __uint_as_float(r.z & 0x7fffffffu);
                    const float f0 = fmaf(fx, c10 - c00, c00);
                    const float f1 = fmaf(fx, c11 - c01, c01);
                    v[p] = __uint_as_float(r.w & 0x7fffffffu) * fmaf(fy, f1 - f0, f0);
                }
                else
                {
                    far[p] = !LF.near[p];
                    const float *b = cellp + LF.off[p];
                    const float c00 = b[0], c10 = b[dps], c01 = b[pdp], c11 = b[pdp + dps];
                    const float f0 = fmaf(LF.fx[p], c10 - c00, c00);
                    const float f1 = fmaf(LF.fx[p], c11 - c01, c01);
                    v[p] = fmaf(LF.fy[p], f1 - f0, f0);
                }
            }
        }
        // departures outside the 3x3 neighbourhood (rare): from global memory
        bool any = false;
#pragma unroll
        for (int p = 0; p < P; p++)
            any |= far[p];
        if (__any_sync(0xffffffffu, any))
        {
            const int i = ijk % nxn, j = ijk / nxn;
            const int cell = (i - 1) + (j - 1) * nx_;
#pragma unroll
            for (int p = 0; p < P; p++)
            {
                const int d = dl + 32 * p;
                if (far[p] && d < nd)
                    v[p] = CURVED ? stream_far32(a.Iin, __ldg(a.side + (unsigned)cell * (unsigned)nd + (unsigned)d),
                                                 dp, nxn, (int)a.g.ny, nd, a.ng, rowtab, dt.q, dt.p, dt.inv_q, i, j)
                                  : stream_flat_far32(a.Iin, LF.ox[p], LF.oy[p], dp, nxn, (int)a.g.ny, d, i, j);
            }
        }
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = dl + 32 * p;
            if (kact && d < nd)
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
    float og = 1.f, oa = 0.f, ob1 = 0.f, ob2 = 0.f;
    if (cact)
    {
        // the two lanes of this cell (every shuffle of phase 2 is between them)
        const unsigned pair = 0x10001u << c;
        float *Sc = S + c * ss;
        // Kahan sums of FP32 partial sums over chunks of 8 of the lane's directions
        float ks[6], kc[6];
#pragma unroll
        for (int q = 0; q < 6; q++)
            ks[q] = kc[q] = 0.f;
        for (int d0 = h; d0 < nd; d0 += 16)
        {
            // FP32 partial sums over 8 of the lane's directions (a direction
            // past the last contributes zero), then folded into the Kahan sums
            float pp[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 8; kk++)
            {
                const int d = d0 + 2 * kk;
                const int dd = min(d, nd - 1);
                const float v = d < nd ? Sc[dd] : 0.f;
                const float4 c0 = dirc[2 * dd], c1 = dirc[2 * dd + 1];
                pp[0] = fmaf(c0.x, v, pp[0]);
                pp[1] = fmaf(c0.y, v, pp[1]);
                pp[2] = fmaf(c0.z, v, pp[2]);
                pp[3] = fmaf(c0.w, v, pp[3]);
                pp[4] = fmaf(c1.x, v, pp[4]);
                pp[5] = fmaf(c1.y, v, pp[5]);
            }
#pragma unroll
            for (int q = 0; q < 6; q++)
            {
                const float y = pp[q] - kc[q];
                const float t = ks[q] + y;
                kc[q] = (t - ks[q]) - y;
                ks[q] = t;
            }
        }
        float m[6];
#pragma unroll
        for (int q = 0; q < 6; q++)
        {
            // the two lanes' compensated sums combined symmetrically (an exact
            // two-sum of their sums, plus both compensations), so that both
            // lanes hold the same moments
            const float os = __shfl_xor_sync(pair, ks[q], 16), oc = __shfl_xor_sync(pair, kc[q], 16);
            const float x = ks[q] + os;
            const float bp = x - ks[q];
            const float err = (ks[q] - (x - bp)) + (os - bp);
            m[q] = x + (err - (kc[q] + oc));
        }
        const bool collides = !(cfl & 1);
        if (collides)
        {
            int cycles = 0;
            const bool rest = (u1 == 0.f) && (u2 == 0.f);
            // m_new[q] = A[q] + (eta + k0 fE) B[q] + k3 (fFx C[q] + fFy D[q])
            float A6[6], B6[6], C6[6], D6[6];
            float g0 = 0.f, h0 = 0.f;
            if (rest)
            {
                g0 = 1.f / (1.f + adt * kak0);
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
                    A6[q] = B6[q] = C6[q] = D6[q] = 0.f;
                for (int d = h; d < nd; d += 2)
                {
                    const float4 c0 = dirc[2 * d], c1 = dirc[2 * d + 1];
                    const float n1 = c1.z, n2 = c1.w, w = c0.x;
                    float g, hh, q1, q2;
                    collide_coeffs32(n1, n2, u1, u2, lor, adt, kak0, g, hh, q1, q2);
                    const float mu[6] = {1.f, n1, n2, n1 * n1, n1 * n2, n2 * n2};
                    const float gs = w * g * Sc[d], wh = w * hh;
#pragma unroll
                    for (int q = 0; q < 6; q++)
                    {
                        A6[q] += gs * mu[q];
                        B6[q] += wh * mu[q];
                        C6[q] += wh * q1 * mu[q];
                        D6[q] += wh * q2 * mu[q];
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
            float diff = 1.f;
            float fE = 0.f, fFx = 0.f, fFy = 0.f;
            while (fabsf(diff) > 1e-4f && cycles < 100)
            {
                cycles++;
                const float pE = m[0], pFx = m[1], pFy = m[2], pPxx = m[3], pPxy = m[4], pPyy = m[5];
                const float uF = u1 * pFx + u2 * pFy;
                const float uxP = u1 * pPxx + u2 * pPxy;
                const float uyP = u1 * pPxy + u2 * pPyy;
                const float uuP = u1 * uxP + u2 * uyP;
                fE = lor * lor * (pE - 2.f * uF + uuP);
                const float rr = lor / (1.f + lor) * ((2.f * lor + 1.f) * uF - lor * uuP);
                fFx = lor * lor * (pFx - lor * pE * u1 - uxP + u1 * rr);
                fFy = lor * lor * (pFy - lor * pE * u2 - uyP + u2 * rr);
                const float ee = eta + k0 * fE;
                const float prev[6] = {pE, pFx, pFy, pPxx, pPxy, pPyy};
                float s2 = 0.f;
#pragma unroll
                for (int q = 0; q < 6; q++)
                {
                    m[q] = A6[q] + ee * B6[q] + k3 * (fFx * C6[q] + fFy * D6[q]);
                    // the exit test's relative change, with the fast quotient (the
                    // FP32 form's choice: a noise moment near zero would otherwise
                    // take the IEEE division's slow path; 0 / 0 is still NaN)
                    const float x = __fdividef(prev[q] - m[q], m[q]);
                    s2 += x * x;
                }
                diff = sqrtf(s2);
            }
            // the intensities of the last iterate (its moments m are the stored
            // ones): for a fluid at rest the affine map with the coefficients
            // phase 3 applies, I_d = g0 S_d + ra + rb1 n1_d + rb2 n2_d (times the
            // state's scale); a moving fluid's here, per direction
            const float ee = eta + k0 * fE;
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
                    const float4 c1 = dirc[2 * d + 1];
                    const float n1 = c1.z, n2 = c1.w;
                    float g, hh, q1, q2;
                    collide_coeffs32(n1, n2, u1, u2, lor, adt, kak0, g, hh, q1, q2);
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
            a.mom[(unsigned)cij + (unsigned)(3 * h + q) * nxy] = h ? m[3 + q] : m[q];
    }
    __syncwarp();

    // ---- phase 3: the cells' new state, coalesced along the directions
    // (and the mirrored directions 0..3 after the last one) ----
    for (int k0_ = 0; k0_ < ncells; k0_ += kStep)
    {
        const int k = k0_ + hk;
        const bool kact = k < ncells;
        const int ij = __shfl_sync(0xffffffffu, cij, k & 15);
        const float g = __shfl_sync(0xffffffffu, og, k & 15), ca = __shfl_sync(0xffffffffu, oa, k & 15);
        const float cb1 = __shfl_sync(0xffffffffu, ob1, k & 15), cb2 = __shfl_sync(0xffffffffu, ob2, k & 15);
        float *o = a.Iout + (unsigned)ij * (unsigned)dp;
        const float *Sk = S + k * ss;
        float first = 0.f;
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = dl + 32 * p;
            const float v = kact ? fmaf(g, Sk[min(d, nd - 1)], fmaf(cb1, LN[p].x, fmaf(cb2, LN[p].y, ca))) : 0.f;
            if (kact && d < nd)
                o[d] = v;
            if (p == 0)
                first = v;
        }
        if (kact && dl < kStateMirror)
            o[nd + dl] = first;
    }
    __syncwarp(); // S is rewritten by the next tile's phase 1
}

// shared layout of the single-problem kernel: the warps' mbarriers, the
// row-type table, the direction coefficients, then the warps' buffers
__device__ __forceinline__ int step32_header(int nd) { return kRowtabOffset + kMaxRowTypes * 12 * 4 + 32 * nd; }

template <bool CURVED, int P, bool H>
__global__ void __launch_bounds__(kThreads, P == 1 ? GRLBM_STEP32_MIN_BLOCKS_1 : GRLBM_STEP32_MIN_BLOCKS)
    k_step_prec(const __grid_constant__ Step32Args a, const __grid_constant__ DirTable dt, int warp_stride)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float *rowtab = reinterpret_cast<float *>(smem + kRowtabOffset);
    float4 *dirc = reinterpret_cast<float4 *>(smem + kRowtabOffset + kMaxRowTypes * 12 * 4);
    const unsigned bar = smem_addr(smem) + 8u * (unsigned)(threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0)
        mbar_init(bar, 1);
    if (CURVED)
        for (int k = threadIdx.x; k < dt.q * 12; k += kThreads)
            rowtab[k] = dt.rowtab[k];
    for (int k = threadIdx.x; k < 2 * a.nd; k += kThreads)
        dirc[k] = reinterpret_cast<const float4 *>(dt.dirc)[k];
    __syncthreads();
    float *patch = step::warp_buffers<float>(smem, step32_header(a.nd), warp_stride);
    float *S = patch + a.patch_floats;
    LaneFlat<P> LF;
    if (!CURVED)
        load_lane_flat<P, H>(LF, dt, a.nd, a.dps, a.tx + 2);
    float2 LN[P];
    load_lane_dirs<P, H>(LN, dirc, a.nd);
    step::IterStats st{0ull, 0u};
    unsigned parity = 0;
    int tile = step::take_tile(a.tiles);
    UnitCells<P> U;
    if (tile < a.ntiles)
    {
        stage_tile(a, tile, patch, bar);
        load_unit<CURVED, P, H>(a, tile, U);
    }
    while (tile < a.ntiles)
    {
        if (!step::wait_tile(bar, parity, a.fault))
            break;
        int next = a.ntiles;
        UnitCells<P> N;
        step_unit32<CURVED, P, H>(a, dt, rowtab, dirc, LF, LN, U, patch, S, st, [&]() {
            next = step::take_tile(a.tiles);
            if (next < a.ntiles)
            {
                stage_tile(a, next, patch, bar);
                load_unit<CURVED, P, H>(a, next, N);
            }
        });
        U = N;
        tile = next;
    }
    step::flush_stats(st, a.iter_sum, a.iter_max);
    step::retire_warp(a.tiles, kWarps);
}

// Many problems in one persistent launch: the warps take tiles from one
// counter over the concatenated tile lists (problem k owns tiles
// [first_tile[k], first_tile[k + 1])) and step each with the single-problem
// tile function at the problem's own passes (or half-warp mode), so every
// problem's result is the one it gets alone.
__device__ __forceinline__ int batch_item_of(const int *__restrict__ first_tile, int n_items, int tile)
{
    int lo = 0, hi = n_items - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (first_tile[mid] <= tile)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int V>
using IntC = std::integral_constant<int, V>;
template <bool V>
using BoolC = std::integral_constant<bool, V>;

// Calls f(IntC<P>, BoolC<H>) for an item's mode (0: half-warp mode, else its
// passes), among the modes a kernel of PM passes holds.
template <int PM, class F>
__device__ __forceinline__ void with_mode(int mode, F &&f)
{
    if (mode == 0)
        f(IntC<1>{}, BoolC<true>{});
    else if (mode == 1)
        f(IntC<1>{}, BoolC<false>{});
    else if constexpr (PM >= 2)
    {
        if (mode == 2)
            f(IntC<2>{}, BoolC<false>{});
        else if constexpr (PM >= 3)
        {
            if (mode == 3)
                f(IntC<3>{}, BoolC<false>{});
            else if constexpr (PM >= 4)
            {
                if (mode == 4)
                    f(IntC<4>{}, BoolC<false>{});
                else if constexpr (PM >= 6)
                {
                    if (mode == 6)
                        f(IntC<6>{}, BoolC<false>{});
                    else if constexpr (PM >= 8)
                        f(IntC<8>{}, BoolC<false>{});
                }
            }
        }
    }
}

// The scalars of a problem's direction tables that the tile function reads
// (the batch kernel keeps a copy per warp in shared memory; 16-byte aligned,
// as the row types that follow it are read as float4).
struct alignas(16) DirScalars
{
    float wmom[18];
    int q, p;
    float inv_q;
};

template <int PM>
__global__ void __launch_bounds__(kThreads, GRLBM_STEP32_MIN_BLOCKS)
    k_step_batch32(const Batch32Item *__restrict__ items, const int *__restrict__ first_tile, int n_items,
                   int total_tiles, int flip, unsigned *counters, int warp_stride, int s_offset, int item_bytes)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const unsigned bar = smem_addr(smem) + 8u * (unsigned)(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (lane == 0)
        mbar_init(bar, 1);
    __syncthreads();
    // the warp's copy of its current problem's step arguments, direction
    // scalars and row types (read by every cell and direction), then its
    // patch and streamed-value buffers
    unsigned char *mine = step::align128(smem + kRowtabOffset) + (size_t)(threadIdx.x >> 5) * (size_t)warp_stride;
    Step32Args &wa = *reinterpret_cast<Step32Args *>(mine);
    DirScalars &wd = *reinterpret_cast<DirScalars *>(mine + sizeof(Step32Args));
    float *wrow = reinterpret_cast<float *>(mine + sizeof(Step32Args) + sizeof(DirScalars));
    float *buf = reinterpret_cast<float *>(mine + item_bytes);
    LaneFlat<PM> LF;
    float2 LN[PM];
    step::IterStats st{0ull, 0u};
    unsigned parity = 0;
    int cur = -1;
    // stage a tile of the batch and load its cells' tables
    auto start_tile = [&](int t, UnitCells<PM> &u) {
        const int nk = batch_item_of(first_tile, n_items, t);
        const Batch32Item &nit = items[nk];
        const Step32Args &na = nit.a[nit.cur0 ^ flip];
        stage_tile(na, t - first_tile[nk], buf, bar);
        with_mode<PM>(nit.mode, [&](auto pc, auto hc) {
            if (nit.curved)
                load_unit<true, decltype(pc)::value, decltype(hc)::value>(na, t - first_tile[nk], u);
            else
                load_unit<false, decltype(pc)::value, decltype(hc)::value>(na, t - first_tile[nk], u);
        });
    };
    int tile = step::take_tile(counters);
    UnitCells<PM> U;
    if (tile < total_tiles)
        start_tile(tile, U);
    while (tile < total_tiles)
    {
        const int k = batch_item_of(first_tile, n_items, tile);
        const Batch32Item &it = items[k];
        if (!step::wait_tile(bar, parity, it.a[it.cur0 ^ flip].fault))
            break;
        const float4 *dirc = reinterpret_cast<const float4 *>(it.dt->dirc);
        if (k != cur)
        {
            if (cur >= 0)
                step::flush_stats(st, wa.iter_sum, wa.iter_max);
            st = step::IterStats{0ull, 0u};
            cur = k;
            __syncwarp(); // the lanes are done with the previous problem's copy
            {
                const unsigned *src = reinterpret_cast<const unsigned *>(&it.a[it.cur0 ^ flip]);
                unsigned *dst = reinterpret_cast<unsigned *>(&wa);
                for (int w = lane; w < (int)(sizeof(Step32Args) / 4); w += 32)
                    dst[w] = src[w];
                const DirTable &dt = *it.dt;
                for (int w = lane; w < 18; w += 32)
                    wd.wmom[w] = dt.wmom[w];
                if (lane == 0)
                    wd.q = dt.q, wd.p = dt.p, wd.inv_q = dt.inv_q;
                if (it.curved)
                    for (int w = lane; w < dt.q * 12; w += 32)
                        wrow[w] = dt.rowtab[w];
            }
            __syncwarp();
            with_mode<PM>(it.mode, [&](auto pc, auto hc) {
                constexpr int P = decltype(pc)::value;
                constexpr bool H = decltype(hc)::value;
                if (!it.curved)
                    load_lane_flat<P, H>(LF, *it.dt, wa.nd, wa.dps, wa.tx + 2);
                load_lane_dirs<P, H>(LN, dirc, wa.nd);
            });
        }
        int next = total_tiles;
        UnitCells<PM> N;
        auto stage_next = [&]() {
            next = step::take_tile(counters);
            if (next < total_tiles)
                start_tile(next, N);
        };
        // (the streamed values sit past the largest patch of the batch: the
        // next tile's copy, of any problem, never reaches them)
        float *S = buf + s_offset;
        with_mode<PM>(it.mode, [&](auto pc, auto hc) {
            constexpr int P = decltype(pc)::value;
            constexpr bool H = decltype(hc)::value;
            if (it.curved)
                step_unit32<true, P, H>(wa, wd, wrow, dirc, LF, LN, U, buf, S, st, stage_next);
            else
                step_unit32<false, P, H>(wa, wd, wrow, dirc, LF, LN, U, buf, S, st, stage_next);
        });
        U = N;
        tile = next;
    }
    if (cur >= 0)
        step::flush_stats(st, wa.iter_sum, wa.iter_max);
    step::retire_warp(counters, kWarps);
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

template <bool CURVED, int P, bool H = false>
cudaError_t set_smem_limit()
{
    return cudaFuncSetAttribute(k_step_prec<CURVED, P, H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kStep32MaxSmem);
}

// the instantiated pass counts
constexpr int kPassSet[] = {1, 2, 3, 4, 6, 8};
} // namespace

int step32_passes(int nd)
{
    const int need = (nd + 31) / 32;
    for (int p : kPassSet)
        if (p >= need)
            return p;
    return -1;
}

int step32_mode(int nd)
{
    const int p = step32_passes(nd);
    return p == 1 && nd <= 16 ? 0 : p;
}

int step32_s_stride(int nd) { return nd + ((2 - nd) % 32 + 32) % 32; }

// A node's run in the patch: a multiple of 32 floats, so that lanes reading
// different corners of one cell use the banks of their windows' own offsets
// only.  In half-warp mode (at most 16 directions: dp <= 20) the two cells a
// pass streams are x-neighbours, and runs of 16 mod 32 floats put the two
// half-warps' reads in opposite halves of the banks instead (1.6 M shared-
// memory conflicts per launch at 400^2 x 16 down to 0.28 M; the step's time
// stayed within 1%).
int step32_patch_node_floats(int dp)
{
    if (dp <= 20)
        return dp <= 16 ? 16 : 48;
    const int padded = (dp + 31) / 32 * 32;
    return padded <= 256 ? padded : dp;
}

int step32_patch_floats(int tx, int ty, int dp)
{
    return ((tx + 2) * (ty + 2) * step32_patch_node_floats(dp) + 31) / 32 * 32;
}

int step32_warp_stride(int tx, int ty, int dp, int nd)
{
    return ((step32_patch_floats(tx, ty, dp) + kUnitCells * step32_s_stride(nd)) * 4 + 127) / 128 * 128;
}

size_t step32_smem(int tx, int ty, int dp, int nd)
{
    const int header = kRowtabOffset + kMaxRowTypes * 12 * 4 + 32 * nd;
    return (size_t)header + 128 + (size_t)kWarps * (size_t)step32_warp_stride(tx, ty, dp, nd);
}

int step32_batch_item_bytes(int q) { return (int)((sizeof(Step32Args) + sizeof(DirScalars) + 4 * 12 * q + 127) / 128 * 128); }

size_t step32_batch_smem(int warp_stride) { return (size_t)kRowtabOffset + 128 + (size_t)kWarps * warp_stride; }

cudaError_t prepare_step32()
{
    cudaError_t e = cudaSuccess;
#define GRLBM_PREP(P)                                                                                       \
    if (e == cudaSuccess)                                                                                   \
        e = set_smem_limit<true, P>();                                                                      \
    if (e == cudaSuccess)                                                                                   \
        e = set_smem_limit<false, P>();                                                                     \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_step_batch32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStep32MaxSmem);
    GRLBM_PREP(1)
    GRLBM_PREP(2)
    GRLBM_PREP(3)
    GRLBM_PREP(4)
    GRLBM_PREP(6)
    GRLBM_PREP(8)
#undef GRLBM_PREP
    if (e == cudaSuccess)
        e = set_smem_limit<true, 1, true>();
    if (e == cudaSuccess)
        e = set_smem_limit<false, 1, true>();
    return e;
}

// resident blocks per SM of the step kernel for P passes at a shared-memory
// size (single problem of nd directions, or the batch kernel)
cudaError_t step32_occupancy(int P, bool curved, bool batch, size_t smem, int *blocks, int nd)
{
    const void *f = nullptr;
    if (!batch && P == 1 && nd <= 16)
        f = curved ? (const void *)k_step_prec<true, 1, true> : (const void *)k_step_prec<false, 1, true>;
#define GRLBM_PICK(PP)                                                                                      \
    if (P == PP && !f)                                                                                      \
        f = batch ? (const void *)k_step_batch32<PP>                                                        \
                  : (curved ? (const void *)k_step_prec<true, PP, false> : (const void *)k_step_prec<false, PP, false>);
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

void launch_step32(const Step32Args &a, const DirTable &dt, bool curved, int P, int blocks, cudaStream_t s)
{
    if (a.ntiles <= 0)
        return;
    const size_t smem = step32_smem(a.tx, a.ty, a.dp, a.nd);
    const int stride = step32_warp_stride(a.tx, a.ty, a.dp, a.nd);
    const unsigned grid = (unsigned)std::max(1, std::min(blocks, (int)nblk(a.ntiles, kWarps)));
    if (P == 1 && a.nd <= 16) // half-warp mode: two cells at a time
    {
        if (curved)
            k_step_prec<true, 1, true><<<grid, kThreads, smem, s>>>(a, dt, stride);
        else
            k_step_prec<false, 1, true><<<grid, kThreads, smem, s>>>(a, dt, stride);
        return;
    }
#define GRLBM_LAUNCH(PP)                                                                                    \
    if (P == PP)                                                                                            \
    {                                                                                                       \
        if (curved)                                                                                         \
            k_step_prec<true, PP, false><<<grid, kThreads, smem, s>>>(a, dt, stride);                       \
        else                                                                                                \
            k_step_prec<false, PP, false><<<grid, kThreads, smem, s>>>(a, dt, stride);                      \
        return;                                                                                             \
    }
    GRLBM_LAUNCH(1)
    GRLBM_LAUNCH(2)
    GRLBM_LAUNCH(3)
    GRLBM_LAUNCH(4)
    GRLBM_LAUNCH(6)
    GRLBM_LAUNCH(8)
#undef GRLBM_LAUNCH
}

void launch_step_batch32(const Batch32Item *items, const int *first_tile, int n_items, int total_tiles, int flip,
                         unsigned *counters, int P, int blocks, size_t smem, int warp_stride, int s_offset,
                         int item_bytes, cudaStream_t s)
{
#define GRLBM_LAUNCH(PP)                                                                                    \
    if (P == PP)                                                                                            \
    {                                                                                                       \
        k_step_batch32<PP><<<blocks, kThreads, smem, s>>>(items, first_tile, n_items, total_tiles, flip,    \
                                                          counters, warp_stride, s_offset, item_bytes);     \
        return;                                                                                             \
    }
    GRLBM_LAUNCH(1)
    GRLBM_LAUNCH(2)
    GRLBM_LAUNCH(3)
    GRLBM_LAUNCH(4)
    GRLBM_LAUNCH(6)
    GRLBM_LAUNCH(8)
#undef GRLBM_LAUNCH
}

// The cell-major state as a 4D tensor {c0, dp / c0, nx, ny} read in boxes
// {box0, dp / c0, tx + 2, ty + 2}: one box is a tile's whole patch, landing
// in shared memory as [node row][node][direction].  When dp is at most 256,
// c0 = dp and the box's first extent is the padded node run
// (step32_patch_node_floats: its floats past dp are the copy's zero fill);
// else c0 is the largest multiple of 4 that divides dp and is at most 256,
// the box's extent limit, and the run is not padded.
cudaError_t encode_state_map32(CUtensorMap *map, const float *state, int64_t nx, int64_t ny, int dp, int tx, int ty)
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
    if (dp % 4 != 0 || reinterpret_cast<uintptr_t>(state) % 16 != 0 || tx < 1 || ty < 1 || tx + 2 > 256 ||
        ty + 2 > 256)
        return cudaErrorInvalidValue;
    int c0 = 0, box0 = 0;
    if (dp <= 256)
        c0 = dp, box0 = step32_patch_node_floats(dp);
    else
    {
        for (int c = 4; c <= 256 && c <= dp; c += 4)
            if (dp % c == 0)
                c0 = c;
        box0 = c0;
    }
    if (c0 == 0 || dp / c0 > 256 || (box0 != c0 && dp / c0 != 1))
        return cudaErrorInvalidValue;
    const cuuint64_t dims[4] = {(cuuint64_t)c0, (cuuint64_t)(dp / c0), (cuuint64_t)nx, (cuuint64_t)ny};
    const cuuint64_t strides[3] = {(cuuint64_t)c0 * sizeof(float), (cuuint64_t)dp * sizeof(float),
                                   (cuuint64_t)nx * (cuuint64_t)dp * sizeof(float)};
    const cuuint32_t box[4] = {(cuuint32_t)box0, (cuuint32_t)(dp / c0), (cuuint32_t)(tx + 2), (cuuint32_t)(ty + 2)};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(state), dims, strides, box,
                              elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
} // namespace grlbm
