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
// Work split: every warp works alone.  It takes tiles of tx x ty cells from a
// counter, stages the tile's (tx + 2) x (ty + 2) node patch of the whole state
// (all directions) into its own shared-memory buffer with one TMA tensor copy,
// and steps the tile's cells one after another with its lanes over the
// directions (direction d = lane + 32 p on pass p).  A lane's streamed values
// stay in registers through the moments, the lambda iteration and the write
// of the collided state, which is coalesced along the directions.
//
// Per (cell, direction) the lane reads its 16-byte packed departure record
// (window row type, window start, blend t, corner fractions with the corner in
// their sign bits, s^3 alpha_c^3 with the far flag in its sign bit), takes the
// window's weights W0 + t D from the row-type table, gathers the 5-tap window
// at the 4 bilinear corners from the patch (contiguous runs), clamps each at
// zero and interpolates.  Departures outside the cell's 3x3 neighbourhood read
// a side record and gather from global memory (cold code).
//
// Moments: per-lane products with the direction's quadrature coefficients,
// summed over the warp by a compensated butterfly (each level an error-free
// two-sum, the rounding errors carried alongside), so every lane holds the
// same compensated sums.
//
// Collide: the lambda iteration of src/Radiation.cpp:661-722 is affine in
// the previous moments -- I_d = g_d S_d + h_d (eta + kappa0 E_ff + 3 kappa1
// nFF_d . F_ff) -- so each iteration runs on the six moments (the same scalar
// work on every lane); the last iterate's moments, the affine map's moments of
// exactly the written intensities, are the stored ones.
#include <cudaTypedefs.h>

#include <algorithm>

#include "device_common.cuh"
#include "tma_util.cuh"

#ifndef GRLBM_STEP32_MIN_BLOCKS
#define GRLBM_STEP32_MIN_BLOCKS 5
#endif

namespace grlbm
{
namespace
{
constexpr int kWarps = kStep32Warps;
constexpr int kThreads = 32 * kWarps;
// time limits of a staging wait (a copy lands within microseconds) and of the
// drain of a copy in flight after a wait has run out
constexpr unsigned long long kWaitNs = 200000000ull, kDrainNs = 2000000000ull;
// shared layout: the warps' mbarriers, the row-type table, then the warps'
// patch buffers from the next 128-byte boundary
constexpr int kBarBytes = 8 * kWarps;
constexpr int kRowtabOffset = 64;
constexpr int kPatchOffset = (kRowtabOffset + kMaxRowTypes * 12 * 4 + 127) / 128 * 128;
static_assert(kBarBytes <= kRowtabOffset, "mbarriers before the row-type table");

__device__ __forceinline__ unsigned char *align128(unsigned char *p)
{
    const unsigned a = smem_addr(p);
    return p + ((128u - (a & 127u)) & 127u);
}

// (s, e) += (b, eb): s + e holds a sum, e the rounding errors of its two-sums
__device__ __forceinline__ void two_sum_acc(float &s, float &e, float b, float eb)
{
    const float x = s + b;
    const float bp = x - s;
    const float err = (s - (x - bp)) + (b - bp);
    s = x;
    e = (e + eb) + err;
}

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

// A lane's per-direction constants for its P passes: the moment
// coefficients {w, w n1, w n2, w n1^2, w n1 n2, w n2^2}, the rotated
// direction (n1, n2), and for flat streaming the departure's corner offset
// in the patch, its fractions and whether it lies within the 3x3
// neighbourhood.
template <int P>
struct LaneDirs
{
    float c[P][6];
    float n1[P], n2[P];
    float ox[P], oy[P], fx[P], fy[P];
    int off[P];
    bool near[P];
};

template <int P>
__device__ __forceinline__ void load_lane_dirs(LaneDirs<P> &L, const DirTable &dt, int nd, int dp, int px,
                                               bool curved)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int p = 0; p < P; p++)
    {
        const int d = lane + 32 * p;
        const bool ok = d < nd;
        const int dd = ok ? d : 0;
#pragma unroll
        for (int k = 0; k < 6; k++)
            L.c[p][k] = ok ? dt.dirc[8 * dd + k] : 0.f;
        L.n1[p] = dt.dirc[8 * dd + 6];
        L.n2[p] = dt.dirc[8 * dd + 7];
        L.ox[p] = L.oy[p] = L.fx[p] = L.fy[p] = 0.f;
        L.off[p] = 0;
        L.near[p] = true;
        if (!curved)
        {
            const float ox = dt.ox[dd], oy = dt.oy[dd];
            const float fli = floorf(ox), flj = floorf(oy);
            L.ox[p] = ox;
            L.oy[p] = oy;
            L.fx[p] = ox - fli;
            L.fy[p] = oy - flj;
            L.near[p] = (fli == -1.f || fli == 0.f) && (flj == -1.f || flj == 0.f);
            L.off[p] = L.near[p] ? ((int)fli + 1 + ((int)flj + 1) * px) * dp + dd : 0;
        }
    }
}

// Per-warp running statistics of the lambda iteration.
struct IterStats
{
    unsigned long long sum;
    unsigned max;
};

// One tile of one step, by one warp: stage the patch, then every cell of the
// tile.  Returns false when the staging copy did not land within its time
// limit (the fault word is then raised and the warp must stop).
template <bool CURVED, int P>
__device__ __forceinline__ bool step_tile32(const Step32Args &a, const DirTable &dt, const float *rowtab,
                                            const LaneDirs<P> &L, int tile, float *patch, unsigned bar,
                                            unsigned &parity, IterStats &st)
{
    const int lane = threadIdx.x & 31;
    const int tx = a.tx, ty = a.ty, px = tx + 2, dp = a.dp, nd = a.nd;
    const int bx = tile % a.tiles_x, by = tile / a.tiles_x;
    const int x0 = bx * tx, y0 = (int)a.g.jlo - 1 + by * ty; // patch origin (node coordinates)
    if (lane == 0)
    {
        // the lanes' reads of the previous tile are done (__syncwarp at the end)
        fence_proxy_async_smem();
        mbar_arrive_expect(bar, (unsigned)(px * (ty + 2) * dp) * 4u);
        tma_load_4d(smem_addr(patch), &a.in_map, 0, 0, x0, y0, bar);
    }
    const bool landed = mbar_wait(bar, parity, kWaitNs, a.fault);
    if (!__all_sync(0xffffffffu, landed))
    {
        // report it and let the copy in flight land (bounded) before leaving
        if (lane == 0 && a.fault)
            *reinterpret_cast<volatile unsigned *>(a.fault) = 1u;
        mbar_wait(bar, parity, kDrainNs, nullptr);
        return false;
    }
    parity ^= 1u;

    const int nxn = (int)a.g.nx;
    const unsigned nxy = (unsigned)a.g.nxy;
    const int txv = min(tx, (int)a.g.nx_ - x0), tyv = min(ty, (int)a.g.jhi - 1 - y0);
    const int ncells = txv * tyv;
    const int pdp = px * dp;
    // records of the cell being stepped and of the next one (prefetched)
    uint4 rc[P], rn[P];
    auto load_recs = [&](uint4(&r)[P], int k) {
        const int cx = k % txv, cy = k / txv;
        const int c = (x0 + cx) + (y0 + cy) * (int)a.g.nx_; // interior cell index of node (i, j)
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            r[p] = d < nd ? __ldcs(a.rec + (unsigned)c * (unsigned)nd + (unsigned)d) : make_uint4(0u, 0u, 0u, 0u);
        }
    };
    if (CURVED)
        load_recs(rc, 0);
    for (int k = 0; k < ncells; k++)
    {
        if (CURVED && k + 1 < ncells)
            load_recs(rn, k + 1);
        const int cx = k % txv, cy = k / txv;
        const int i = 1 + x0 + cx, j = 1 + y0 + cy;
        const int ij = i + j * nxn;
        const uint8_t fl = a.flags[ij];
        const bool live = !(CURVED && (fl & 2));
        const bool collides = !(fl & 1);
        // per-cell fields, loaded before the gather so that they land meanwhile
        float u1 = 0.f, u2 = 0.f, lor = 1.f, adt = 0.f, eta = 0.f, k0 = 0.f, k3 = 0.f, kak0 = 0.f;
        if (collides)
        {
            u1 = __ldg(a.u1 + ij), u2 = __ldg(a.u2 + ij), lor = __ldg(a.lor + ij), adt = __ldg(a.adt + ij);
            eta = __ldg(a.eta + ij), k0 = __ldg(a.k0 + ij), k3 = __ldg(a.k3 + ij), kak0 = __ldg(a.ka + ij) + k0;
        }
        const float scale = CURVED ? __ldg(a.ia3 + ij) : 1.f;
        // patch offset of node (i - 1, j - 1), the cell's lower-left neighbour
        const float *cellp = patch + (cy * px + cx) * dp;
        float S[P];
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            float v = 0.f;
            if (d < nd && live)
            {
                if (CURVED)
                {
                    const uint4 r = rc[p];
                    if (r.w >> 31)
                        v = stream_far32(a.Iin,
                                         __ldg(a.side + (unsigned)((x0 + cx) + (y0 + cy) * (int)a.g.nx_) *
                                                            (unsigned)nd +
                                               (unsigned)d),
                                         dp, nxn, (int)a.g.ny, nd, a.ng, rowtab, dt.q, dt.p, dt.inv_q, i, j);
                    else
                    {
                        const unsigned word = r.x;
                        const float t = (float)(word & ((1u << packed32::kTBits) - 1u)) *
                                        (1.f / (float)(1u << packed32::kTBits));
                        const float4 *row =
                            reinterpret_cast<const float4 *>(rowtab + ((word >> packed32::kTypeShift) & 31u) * 12);
                        const float4 R0 = row[0], R1 = row[1], R2 = row[2];
                        const float w0 = fmaf(t, R1.x, R0.x), w1 = fmaf(t, R1.y, R0.y), w2 = fmaf(t, R1.z, R0.z);
                        const float w3 = fmaf(t, R1.w, R0.w), w4 = fmaf(t, R2.y, R2.x);
                        const int s = (int)((word >> packed32::kStartShift) & 255u);
                        const float *p00 = cellp + (int)(r.y >> 31) * dp + (int)(r.z >> 31) * pdp + s;
                        const float c00 = window5(p00, w0, w1, w2, w3, w4);
                        const float c10 = window5(p00 + dp, w0, w1, w2, w3, w4);
                        const float c01 = window5(p00 + pdp, w0, w1, w2, w3, w4);
                        const float c11 = window5(p00 + pdp + dp, w0, w1, w2, w3, w4);
                        const float fx = __uint_as_float(r.y & 0x7fffffffu), fy = __uint_as_float(r.z & 0x7fffffffu);
                        const float f0 = fmaf(fx, c10 - c00, c00);
                        const float f1 = fmaf(fx, c11 - c01, c01);
                        v = __uint_as_float(r.w) * fmaf(fy, f1 - f0, f0);
                    }
                }
                else if (L.near[p])
                {
                    const float *b = cellp + L.off[p];
                    const float c00 = b[0], c10 = b[dp], c01 = b[pdp], c11 = b[pdp + dp];
                    const float f0 = fmaf(L.fx[p], c10 - c00, c00);
                    const float f1 = fmaf(L.fx[p], c11 - c01, c01);
                    v = fmaf(L.fy[p], f1 - f0, f0);
                }
                else
                    v = stream_flat_far32(a.Iin, L.ox[p], L.oy[p], dp, nxn, (int)a.g.ny, d, i, j);
            }
            S[p] = v;
        }
        // moments of the streamed values: per-lane two-sums over the passes,
        // then the compensated butterfly over the lanes
        float m[6], e[6];
#pragma unroll
        for (int q = 0; q < 6; q++)
        {
            // (products rounded on their own: an FMA would break the two-sum)
            m[q] = __fmul_rn(L.c[0][q], S[0]);
            e[q] = 0.f;
#pragma unroll
            for (int p = 1; p < P; p++)
                two_sum_acc(m[q], e[q], __fmul_rn(L.c[p][q], S[p]), 0.f);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < 6; q++)
            {
                const float bs = __shfl_xor_sync(0xffffffffu, m[q], o), be = __shfl_xor_sync(0xffffffffu, e[q], o);
                two_sum_acc(m[q], e[q], bs, be);
            }
#pragma unroll
        for (int q = 0; q < 6; q++)
            m[q] += e[q];

        float out[P];
#pragma unroll
        for (int p = 0; p < P; p++)
            out[p] = S[p] * scale;
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
                // per-direction sums over the warp (plain FP32 butterfly)
#pragma unroll
                for (int q = 0; q < 6; q++)
                    A6[q] = B6[q] = C6[q] = D6[q] = 0.f;
#pragma unroll
                for (int p = 0; p < P; p++)
                {
                    if (lane + 32 * p >= nd)
                        continue;
                    const float n1 = L.n1[p], n2 = L.n2[p], w = L.c[p][0];
                    float g, h, q1, q2;
                    collide_coeffs32(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                    const float mu[6] = {1.f, n1, n2, n1 * n1, n1 * n2, n2 * n2};
                    const float gs = w * g * S[p], wh = w * h;
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
                for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                    for (int q = 0; q < 6; q++)
                    {
                        A6[q] += __shfl_xor_sync(0xffffffffu, A6[q], o);
                        B6[q] += __shfl_xor_sync(0xffffffffu, B6[q], o);
                        C6[q] += __shfl_xor_sync(0xffffffffu, C6[q], o);
                        D6[q] += __shfl_xor_sync(0xffffffffu, D6[q], o);
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
                    const float x = (prev[q] - m[q]) / m[q];
                    s2 += x * x;
                }
                diff = sqrtf(s2);
            }
            // the intensities of the last iterate; its moments m are the stored ones
            const float ee = eta + k0 * fE;
            const float ra = h0 * ee, rb1 = h0 * k3 * fFx, rb2 = h0 * k3 * fFy;
#pragma unroll
            for (int p = 0; p < P; p++)
            {
                const float n1 = L.n1[p], n2 = L.n2[p];
                float v;
                if (rest)
                    v = fmaf(g0, S[p], fmaf(rb1, n1, fmaf(rb2, n2, ra)));
                else
                {
                    float g, h, q1, q2;
                    collide_coeffs32(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                    v = g * S[p] + h * (ee + k3 * (q1 * fFx + q2 * fFy));
                }
                out[p] = v * scale;
            }
            st.sum += (unsigned)cycles;
            st.max = max(st.max, (unsigned)cycles);
        }
        // the cell's new state, coalesced along the directions (and the
        // mirrored directions 0..3 after the last one)
        float *o = a.Iout + (unsigned)ij * (unsigned)dp;
#pragma unroll
        for (int p = 0; p < P; p++)
        {
            const int d = lane + 32 * p;
            if (d < nd)
                o[d] = out[p];
            if (p == 0 && lane < kStateMirror)
                o[nd + lane] = out[0];
        }
        if (lane < 6)
        {
            float mv = m[0];
#pragma unroll
            for (int q = 1; q < 6; q++)
                mv = lane == q ? m[q] : mv;
            a.mom[(unsigned)ij + (unsigned)lane * nxy] = mv;
        }
        if (CURVED)
        {
#pragma unroll
            for (int p = 0; p < P; p++)
                rc[p] = rn[p];
        }
    }
    __syncwarp();
    return true;
}

// the warp's share of the block's shared memory
__device__ __forceinline__ float *warp_patch(unsigned char *smem, int patch_stride)
{
    const int warp = threadIdx.x >> 5;
    return reinterpret_cast<float *>(align128(smem + kPatchOffset) + (size_t)warp * (size_t)patch_stride);
}

// The warp is done taking tiles from counter[0]; the launch's last warp
// clears both words for the next launch.
__device__ __forceinline__ void retire_warp(unsigned *counter)
{
    if ((threadIdx.x & 31) == 0)
    {
        __threadfence(); // this warp's last take is ordered before its retirement
        if (atomicAdd(counter + 1, 1u) == gridDim.x * (unsigned)kWarps - 1u)
        {
            counter[0] = 0u;
            counter[1] = 0u;
        }
    }
}

__device__ __forceinline__ void flush_stats(const IterStats &st, unsigned long long *iter_sum, unsigned *iter_max)
{
    if ((threadIdx.x & 31) == 0 && st.sum)
    {
        atomicAdd(iter_sum, st.sum);
        atomicMax(iter_max, st.max);
    }
}

template <bool CURVED, int P>
__global__ void __launch_bounds__(kThreads, GRLBM_STEP32_MIN_BLOCKS)
    k_step_prec(const __grid_constant__ Step32Args a, const __grid_constant__ DirTable dt, int patch_stride)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float *rowtab = reinterpret_cast<float *>(smem + kRowtabOffset);
    const int lane = threadIdx.x & 31;
    const unsigned bar = smem_addr(smem) + 8u * (unsigned)(threadIdx.x >> 5);
    if (lane == 0)
        mbar_init(bar, 1);
    if (CURVED)
        for (int k = threadIdx.x; k < dt.q * 12; k += kThreads)
            rowtab[k] = dt.rowtab[k];
    __syncthreads();
    float *patch = warp_patch(smem, patch_stride);
    LaneDirs<P> L;
    load_lane_dirs<P>(L, dt, a.nd, a.dp, a.tx + 2, CURVED);
    IterStats st{0ull, 0u};
    unsigned parity = 0;
    for (;;)
    {
        int tile = 0;
        if (lane == 0)
            tile = (int)atomicAdd(a.tiles, 1u);
        tile = __shfl_sync(0xffffffffu, tile, 0);
        if (tile >= a.ntiles)
            break;
        if (!step_tile32<CURVED, P>(a, dt, rowtab, L, tile, patch, bar, parity, st))
            break;
    }
    flush_stats(st, a.iter_sum, a.iter_max);
    retire_warp(a.tiles);
}

// Many problems in one persistent launch: the warps take tiles from one
// counter over the concatenated tile lists (problem k owns tiles
// [first_tile[k], first_tile[k + 1])) and step each with the single-problem
// tile function, so every problem's result is the one it gets alone.  A
// warp reloads its direction constants when its problem changes.
template <int P>
__global__ void __launch_bounds__(kThreads, GRLBM_STEP32_MIN_BLOCKS)
    k_step_batch32(const Batch32Item *__restrict__ items, const int *__restrict__ first_tile, int n_items,
                   int total_tiles, int flip, unsigned *counters, int patch_stride)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const unsigned bar = smem_addr(smem) + 8u * (unsigned)(threadIdx.x >> 5);
    if (lane == 0)
        mbar_init(bar, 1);
    __syncthreads();
    float *patch = warp_patch(smem, patch_stride);
    LaneDirs<P> L;
    IterStats st{0ull, 0u};
    unsigned parity = 0;
    int cur = -1;
    const Step32Args *ca = nullptr;
    for (;;)
    {
        int tile = 0;
        if (lane == 0)
            tile = (int)atomicAdd(counters, 1u);
        tile = __shfl_sync(0xffffffffu, tile, 0);
        if (tile >= total_tiles)
            break;
        int lo = 0, hi = n_items - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (first_tile[mid] <= tile)
                lo = mid;
            else
                hi = mid - 1;
        }
        const Batch32Item &it = items[lo];
        if (lo != cur)
        {
            if (ca)
                flush_stats(st, ca->iter_sum, ca->iter_max);
            st = IterStats{0ull, 0u};
            cur = lo;
            ca = &it.a[it.cur0 ^ flip];
            load_lane_dirs<P>(L, *it.dt, ca->nd, ca->dp, ca->tx + 2, it.curved != 0);
        }
        const int local = tile - first_tile[lo];
        const bool ok = it.curved ? step_tile32<true, P>(*ca, *it.dt, it.dt->rowtab, L, local, patch, bar, parity, st)
                                  : step_tile32<false, P>(*ca, *it.dt, it.dt->rowtab, L, local, patch, bar, parity, st);
        if (!ok)
            break; // the barrier's phase is unknown: the warp stops (the fault word is set)
    }
    if (ca)
        flush_stats(st, ca->iter_sum, ca->iter_max);
    retire_warp(counters);
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

template <bool CURVED, int P>
cudaError_t set_smem_limit()
{
    return cudaFuncSetAttribute(k_step_prec<CURVED, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
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

int step32_patch_stride(int tx, int ty, int dp) { return ((tx + 2) * (ty + 2) * dp * 4 + 127) / 128 * 128; }

size_t step32_smem_base() { return (size_t)kPatchOffset + 128; }

size_t step32_smem(int tx, int ty, int dp)
{
    return step32_smem_base() + (size_t)kWarps * (size_t)step32_patch_stride(tx, ty, dp);
}

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
    return e;
}

// resident blocks per SM of the step kernel for P passes at a shared-memory size
cudaError_t step32_occupancy(int P, bool curved, bool batch, size_t smem, int *blocks)
{
    const void *f = nullptr;
#define GRLBM_PICK(PP)                                                                                      \
    if (P == PP)                                                                                            \
        f = batch ? (const void *)k_step_batch32<PP>                                                        \
                  : (curved ? (const void *)k_step_prec<true, PP> : (const void *)k_step_prec<false, PP>);
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
    const size_t smem = step32_smem(a.tx, a.ty, a.dp);
    const int stride = step32_patch_stride(a.tx, a.ty, a.dp);
    const unsigned grid = (unsigned)std::max(1, std::min(blocks, (int)nblk(a.ntiles, kWarps)));
#define GRLBM_LAUNCH(PP)                                                                                    \
    if (P == PP)                                                                                            \
    {                                                                                                       \
        if (curved)                                                                                         \
            k_step_prec<true, PP><<<grid, kThreads, smem, s>>>(a, dt, stride);                              \
        else                                                                                                \
            k_step_prec<false, PP><<<grid, kThreads, smem, s>>>(a, dt, stride);                             \
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
                         unsigned *counters, int P, int blocks, size_t smem, int patch_stride, cudaStream_t s)
{
#define GRLBM_LAUNCH(PP)                                                                                    \
    if (P == PP)                                                                                            \
    {                                                                                                       \
        k_step_batch32<PP><<<blocks, kThreads, smem, s>>>(items, first_tile, n_items, total_tiles, flip,    \
                                                          counters, patch_stride);                          \
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

// The cell-major state as a 4D tensor {c0, dp / c0, nx, ny} (c0: the largest
// multiple of 4 that divides dp and is at most 256, the TMA's box limit), read
// in boxes {c0, dp / c0, tx + 2, ty + 2}: one box is a tile's whole patch,
// landing in shared memory as [node row][node][direction].
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
    int c0 = 0;
    for (int c = 4; c <= 256 && c <= dp; c += 4)
        if (dp % c == 0)
            c0 = c;
    if (c0 == 0 || dp / c0 > 256)
        return cudaErrorInvalidValue;
    const cuuint64_t dims[4] = {(cuuint64_t)c0, (cuuint64_t)(dp / c0), (cuuint64_t)nx, (cuuint64_t)ny};
    const cuuint64_t strides[3] = {(cuuint64_t)c0 * sizeof(float), (cuuint64_t)dp * sizeof(float),
                                   (cuuint64_t)nx * (cuuint64_t)dp * sizeof(float)};
    const cuuint32_t box[4] = {(cuuint32_t)c0, (cuuint32_t)(dp / c0), (cuuint32_t)(tx + 2), (cuuint32_t)(ty + 2)};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(state), dims, strides, box,
                              elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
} // namespace grlbm
