// Precision form of the adaptive streaming types (FlatAdaptive,
// CurvedAdaptive): FP32 intensities and stream/collide arithmetic (contracted
// FMAs allowed), Kahan-compensated FP32 moment sums, on a direction-major
// FP32 state (J = I / alpha^3 for curved streaming).  The fixed streaming
// types have their own kernel (kernels_step32.cu).  Also here: the bounded
// mbarrier wait's self-test and the FP32 coefficient copy of adaptive
// streaming.
#include <cudaTypedefs.h>

#include "approx_math.hpp"
#include "device_common.cuh"
#include "tma_util.cuh"

namespace grlbm
{
namespace
{
struct Kahan
{
    float s, c;
    __device__ __forceinline__ void zero() { s = 0.f, c = 0.f; }
    __device__ __forceinline__ void add(float v)
    {
        const float y = v - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// Moment sums compensated per block of directions: plain FP32 partial sums
// over up to kChunk directions, folded into Kahan accumulators by the caller
// after each block.  The direction coefficients c0 = {w, w n1, w n2, w n1^2},
// c1 = {w n1 n2, w n2^2, n1, n2} come from the shared direction table.
struct KMoments
{
    Kahan E, Fx, Fy, Pxx, Pxy, Pyy;
    float p[6];
    __device__ __forceinline__ void zero()
    {
        E.zero(), Fx.zero(), Fy.zero(), Pxx.zero(), Pxy.zero(), Pyy.zero();
#pragma unroll
        for (int q = 0; q < 6; q++)
            p[q] = 0.f;
    }
    __device__ __forceinline__ void fold()
    {
        E.add(p[0]), Fx.add(p[1]), Fy.add(p[2]), Pxx.add(p[3]), Pxy.add(p[4]), Pyy.add(p[5]);
#pragma unroll
        for (int q = 0; q < 6; q++)
            p[q] = 0.f;
    }
    __device__ __forceinline__ void add(float v, const float4 &c0, const float4 &c1)
    {
        p[0] = fmaf(c0.x, v, p[0]);
        p[1] = fmaf(c0.y, v, p[1]);
        p[2] = fmaf(c0.z, v, p[2]);
        p[3] = fmaf(c0.w, v, p[3]);
        p[4] = fmaf(c1.x, v, p[4]);
        p[5] = fmaf(c1.y, v, p[5]);
    }
};

// direction coefficients of the affine collide map for a moving fluid
__device__ __forceinline__ void collide_coeffs(float n1, float n2, float u1, float u2, float lor, float adt,
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

// ---------------------------------------------------------------------------
// Adaptive streaming in the precision form (FlatAdaptive, CurvedAdaptive;
// src/Radiation.cpp:415-452, 513-575), as two kernels: one thread per (cell,
// direction) streams into S, then one thread per cell takes the moments and
// collides.  FP32 arithmetic, FP32 state (J = I / alpha^3 for curved
// streaming); the Fourier series sum in FP64 over an FP32 basis.
constexpr int kATileX = 16, kATileY = kStepBlock / kATileX;

// The reference's polynomial atan2 and Phi (MyAtan2<9>, Tensor2::Phi;
// src/Utility.hh:179-254, src/DataTypes.hh:166-170) evaluated in FP32, in
// grid-row units: nGrid * Phi(x, y) / (2 pi).  The same octants and
// polynomial as approx_phi, with the fast FP32 quotient (within 2 ulp, and
// |z| <= 1 here); the FP32 rounding adds an error of the order of the FP32
// rounding of the row coordinate itself.
__device__ __forceinline__ float atan_poly9_f(float z)
{
    const float zz = z * z;
    return z * (0.9998660f + zz * (-0.3302995f + zz * (0.1801410f + zz * (-0.0851330f + zz * 0.0208351f))));
}
__device__ __forceinline__ float grid_row_of(float x, float y, float rows_per_rad)
{
    const float pi = 3.14159265358979f, half_pi = 1.57079632679490f;
    float p;
    if (x != 0.f)
    {
        if (fabsf(x) > fabsf(y))
        {
            p = atan_poly9_f(__fdividef(y, x));
            if (x < 0.f)
                p = (y >= 0.f) ? p + pi : p - pi;
        }
        else
        {
            const float q = atan_poly9_f(__fdividef(x, y));
            p = (y > 0.f) ? half_pi - q : -q - half_pi;
        }
    }
    else
        p = y > 0.f ? half_pi : (y < 0.f ? -half_pi : 0.f);
    if (p < 0.f)
        p += 2.f * pi;
    return p * rows_per_rad;
}

// IntensityAt (src/Radiation.cpp:322-343) on the FP32 state: the direction
// (v1, v2) rotated into node n's previous frame, the two cubic rows of the
// interpolation grid at its angle, blended and clamped at zero.  sidx: the
// node's place in a state plane.
__device__ __forceinline__ float intensity_at32(const PrecStepArgs &a, int n, unsigned sidx, float v1, float v2)
{
    // the inverse of the node's previous rotation, with the reference's
    // polynomial trigonometry (the plain form's values)
    const float2 rinv = a.rot_inv[n];
    const float sn = rinv.x, cs = rinv.y;
    const float w1 = v1 * cs - v2 * sn, w2 = v1 * sn + v2 * cs;
    float dd = grid_row_of(w1, w2, (float)a.ng * 0.159154943091895f);
    dd = fminf(fmaxf(dd, 1e-8f), nextafterf((float)a.ng, 0.f)); // InterpolationGrid's clamp, in FP32
    const int g0 = min((int)dd, a.ng - 1), g1 = g0 + 1 == a.ng ? 0 : g0 + 1;
    const float t = dd - (float)g0;
    const IgRow32 R0 = a.ig_rows[g0], R1 = a.ig_rows[g1];
    const int idx0[4] = {R0.idx.x, R0.idx.y, R0.idx.z, R0.idx.w};
    const int idx1[4] = {R1.idx.x, R1.idx.y, R1.idx.z, R1.idx.w};
    const float wa[4] = {R0.w.x, R0.w.y, R0.w.z, R0.w.w};
    const float wb[4] = {R1.w.x, R1.w.y, R1.w.z, R1.w.w};
    float x0 = 0.f, x1 = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++)
    {
        x0 = fmaf(wa[k], __ldg(a.Iin + (unsigned)idx0[k] * a.plane + sidx), x0);
        x1 = fmaf(wb[k], __ldg(a.Iin + (unsigned)idx1[k] * a.plane + sidx), x1);
    }
    return fmaxf(fmaf(t, x1 - x0, x0), 0.f);
}

// One adaptive stream value (I, not J) of cell (i, j) for its direction d
// rotated by the cell's new angle.  Curved streaming reads coefficient k of
// series q of the cell at cf[q * qs + k * ks] (FP32, X and Y about the node).
template <bool CURVED>
__device__ __forceinline__ float stream_adaptive32(const PrecStepArgs &a, int d, int i, int j, int ij,
                                                   const float *cf, int ks, int qs)
{
    const int nx = (int)a.g.nx;
    const float2 rn = a.rot_new[ij];
    const float sc = rn.x, cc = rn.y;
    const float cxd = a.cx[d], cyd = a.cy[d];
    const float dir1 = cxd * cc - cyd * sc, dir2 = cxd * sc + cyd * cc;
    float it, jt, v1, v2, s3 = 1.f;
    if constexpr (CURVED)
    {
        // the five series (S, X - x, Y - y, Cx, Cy) at the direction's angle:
        // basis {1, sqrt2 cos(m phi), sqrt2 sin(m phi)} from one sincos and
        // the angle-addition recurrence
        const float phi = grid_row_of(dir1, dir2, 1.f);
        float s1, c1;
        sincosf(phi, &s1, &c1);
        float r[5];
#pragma unroll
        for (int q = 0; q < 5; q++)
            r[q] = cf[q * qs];
        float cm = 1.f, sm = 0.f;
        const float sqrt2 = 1.41421356237f;
        for (int k = 1; k < a.nf; k++)
        {
            if (k & 1) // the next multiple of phi
            {
                const float c2 = cm * c1 - sm * s1;
                sm = sm * c1 + cm * s1;
                cm = c2;
            }
            const float b = sqrt2 * ((k & 1) ? cm : sm);
            const float *ck = cf + k * ks;
#pragma unroll
            for (int q = 0; q < 5; q++)
                r[q] = fmaf(ck[q * qs], b, r[q]);
        }
        // the departure point, absolute for the excision test
        const double xt = a.g.startx + (double)i * a.g.dx + (double)r[1];
        const double yt = a.g.starty + (double)j * a.g.dy + (double)r[2];
        if (dev_inside_bh(a.g, xt, yt))
            return 0.f;
        it = (float)i + r[1] * a.inv_dx;
        jt = (float)j + r[2] * a.inv_dy;
        const float sh = r[0];
        s3 = sh * sh * sh;
        v1 = r[3];
        v2 = r[4];
    }
    else
    {
        it = (float)i - dir1 * (float)(a.g.dt / a.g.dx);
        jt = (float)j - dir2 * (float)(a.g.dt / a.g.dy);
        v1 = dir1;
        v2 = dir2;
    }
    const int i0 = min(max((int)floorf(it), 0), nx - 2);
    const int j0 = min(max((int)floorf(jt), 0), (int)a.g.ny - 2);
    const float fx = it - (float)i0, fy = jt - (float)j0;
    float Iq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) // corners 00, 01, 10, 11
    {
        const int ci = i0 + (q >> 1), cj = j0 + (q & 1);
        Iq[q] = intensity_at32(a, ci + cj * nx, (unsigned)ci + (unsigned)cj * a.pitch, v1, v2);
    }
    const float f0 = fmaf(fx, Iq[2] - Iq[0], Iq[0]);
    const float f1 = fmaf(fx, Iq[3] - Iq[1], Iq[1]);
    const float bil = fmaf(fy, f1 - f0, f0);
    // corners hold J = I / alpha^3: (alpha_ij / alpha_c)^3 I_c = alpha_ij^3 J_c
    return CURVED ? s3 * bil / a.ia3[ij] : bil;
}

// Flat stream: blocks are 16 x 8 tiles of cells of one direction,
// directions fastest in the grid.
__global__ void __launch_bounds__(kStepBlock) k_stream_prec_adaptive_flat(PrecStepArgs a)
{
    const int d = blockIdx.x;
    const int i = 1 + (int)blockIdx.y * kATileX + (int)(threadIdx.x % kATileX);
    const int j = (int)a.g.jlo + (int)blockIdx.z * kATileY + (int)(threadIdx.x / kATileX);
    if (i > a.g.nx_ || j >= a.g.jhi)
        return;
    const int ij = i + j * (int)a.g.nx;
    a.S[(size_t)d * (size_t)a.g.nxy + (size_t)ij] = stream_adaptive32<false>(a, d, i, j, ij, nullptr, 0, 0);
}

// Curved stream: a block takes 16 cells of one row for kADirs directions
// (16: 6% faster than 8, and 32 slower, at 400^2 x 64).
// It first stages the row's Fourier coefficients (5 nF x 16 floats, at most
// 20 KB) in shared memory, where its directions share them; each warp then
// covers 16 cells x 2 directions, so a tap load reads two 16-node runs.
constexpr int kADirs = kAdaptiveBlock / kATileX;
__global__ void __launch_bounds__(kAdaptiveBlock) k_stream_prec_adaptive_curved(PrecStepArgs a)
{
    extern __shared__ float sco[]; // [q * nF + k][cell]
    // blockIdx.x: direction group fastest, then the row; blockIdx.y: the run of 16 cells
    const int ndg = (a.nd + kADirs - 1) / kADirs;
    const int t = threadIdx.x, c = t % kATileX;
    const int d = (int)(blockIdx.x % (unsigned)ndg) * kADirs + t / kATileX;
    const int x0 = 1 + (int)blockIdx.y * kATileX, i = x0 + c;
    const int j = (int)a.g.jlo + (int)(blockIdx.x / (unsigned)ndg);
    const int nrow = min(kATileX, (int)a.g.nx_ + 1 - x0);
    const int row0 = x0 + j * (int)a.g.nx;
    // coefficient k of series q of node ij sits at coef32[(q nF + k) nxy + ij]
    for (int e = t; e < 5 * a.nf * kATileX; e += kAdaptiveBlock)
    {
        const int p = e / kATileX, cc = e % kATileX;
        sco[e] = cc < nrow ? a.coef32[(size_t)p * (size_t)a.g.nxy + (size_t)(row0 + cc)] : 0.f;
    }
    __syncthreads();
    if (c >= nrow || d >= a.nd)
        return;
    const int ij = row0 + c;
    float v = 0.f;
    if (!(a.flags[ij] & 2))
        v = stream_adaptive32<true>(a, d, i, j, ij, sco + c, kATileX, a.nf * kATileX);
    a.S[(size_t)d * (size_t)a.g.nxy + (size_t)ij] = v;
}

// Moments and collide of one cell from its streamed values, with its
// stencil rotated by its new angle: Kahan moments of the streamed values,
// the lambda iteration in moment space (as the fixed-streaming kernel's
// moving-fluid path), the collided state J = I / alpha^3, and the last
// iterate's moments as the stored ones.
template <bool CURVED>
__global__ void __launch_bounds__(kStepBlock) k_collide_prec_adaptive(PrecStepArgs a, const __grid_constant__ DirTable dt)
{
    const int ti = 1 + (int)blockIdx.x * kATileX + (int)(threadIdx.x % kATileX);
    const int tj = (int)a.g.jlo + (int)blockIdx.y * kATileY + (int)(threadIdx.x / kATileX);
    const bool active = ti <= a.g.nx_ && tj < a.g.jhi;
    const int i = active ? ti : 1, j = active ? tj : 1;
    const int ij = i + j * (int)a.g.nx;
    const unsigned nxy = (unsigned)a.g.nxy;
    const uint8_t fl = active ? a.flags[ij] : (uint8_t)3;
    const bool collides = active && !(fl & 1);
    const float *S = a.S + ij;
    // the cell's stencil, rotated (shared by the block's threads per direction)
    __shared__ float sw[kMaxDirs], scx[kMaxDirs], scy[kMaxDirs];
    for (int d = threadIdx.x; d < a.nd; d += kStepBlock)
        sw[d] = dt.w[d], scx[d] = a.cx[d], scy[d] = a.cy[d];
    __syncthreads();
    // the unrotated stencil's weighted moments sum w, sum w c_a, sum w c_a c_b,
    // sum w c_a c_b c_c (a <= b <= c), from the direction table's stencil sums
    // (its directions are the stencil's under RotationMatrix(0), the identity)
    const float smom[10] = {dt.wmom[0], dt.wmom[1], dt.wmom[2],  dt.wmom[3],  dt.wmom[4],
                            dt.wmom[5], dt.wmom[9], dt.wmom[10], dt.wmom[11], dt.wmom[17]};
    const float2 rn = a.rot_new[ij];
    const float rs = rn.x, rc = rn.y;
#define GRLBM_RN1(d) (scx[d] * rc - scy[d] * rs)
#define GRLBM_RN2(d) (scx[d] * rs + scy[d] * rc)
    KMoments km;
    km.zero();
    for (int d0 = 0; d0 < a.nd; d0 += kChunk)
    {
        // the streamed values of a chunk, loaded together
        float Sv[kChunk];
#pragma unroll
        for (int k = 0; k < kChunk; k++)
            Sv[k] = d0 + k < a.nd ? S[(unsigned)(d0 + k) * nxy] : 0.f;
#pragma unroll
        for (int k = 0; k < kChunk; k++)
        {
            const int d = d0 + k;
            if (d >= a.nd)
                break;
            const float n1 = GRLBM_RN1(d), n2 = GRLBM_RN2(d), w = sw[d];
            const float wn1 = w * n1, wn2 = w * n2;
            km.add(Sv[k], make_float4(w, wn1, wn2, wn1 * n1), make_float4(wn1 * n2, wn2 * n2, n1, n2));
        }
        km.fold();
    }
    float m[6] = {km.E.s, km.Fx.s, km.Fy.s, km.Pxx.s, km.Pxy.s, km.Pyy.s};
    int cycles = 0;
    if (collides)
    {
        const float u1 = a.u1[ij], u2 = a.u2[ij], lor = a.lor[ij], adt = a.adt[ij];
        const float eta = a.eta[ij], k0 = a.k0[ij], k3 = a.k3[ij], kak0 = a.ka[ij] + a.k0[ij];
        // m_new[q] = A[q] + (eta + k0 fE) B[q] + k3 (fFx C[q] + fFy D[q]);
        // at rest g and h are the same for every direction and q = n
        const bool rest = (u1 == 0.f) && (u2 == 0.f);
        const float g0 = 1.f / (1.f + adt * kak0), h0 = adt * g0;
        float A6[6], B6[6], C6[6], D6[6];
        if (rest)
        {
            // A = g0 m; B, C, D: h0 times the rotated stencil's weighted
            // moments of orders 0-3, from the unrotated ones (n = R c,
            // R = {{rc, -rs}, {rs, rc}})
            const float R[2][2] = {{rc, -rs}, {rs, rc}};
            const float m1[2] = {smom[1], smom[2]};
            const float m2[2][2] = {{smom[3], smom[4]}, {smom[4], smom[5]}};
            float m3[2][2][2];
#pragma unroll
            for (int x = 0; x < 2; x++)
#pragma unroll
                for (int y = 0; y < 2; y++)
#pragma unroll
                    for (int z = 0; z < 2; z++)
                        m3[x][y][z] = smom[6 + x + y + z];
            float r1[2], r2[2][2], r3[2][2][2];
#pragma unroll
            for (int p = 0; p < 2; p++)
            {
                r1[p] = R[p][0] * m1[0] + R[p][1] * m1[1];
#pragma unroll
                for (int q = 0; q < 2; q++)
                {
                    float s2 = 0.f;
#pragma unroll
                    for (int x = 0; x < 2; x++)
#pragma unroll
                        for (int y = 0; y < 2; y++)
                            s2 += R[p][x] * R[q][y] * m2[x][y];
                    r2[p][q] = s2;
#pragma unroll
                    for (int o = 0; o < 2; o++)
                    {
                        float s3 = 0.f;
#pragma unroll
                        for (int x = 0; x < 2; x++)
#pragma unroll
                            for (int y = 0; y < 2; y++)
#pragma unroll
                                for (int z = 0; z < 2; z++)
                                    s3 += R[p][x] * R[q][y] * R[o][z] * m3[x][y][z];
                        r3[p][q][o] = s3;
                    }
                }
            }
            const float b6[6] = {smom[0], r1[0], r1[1], r2[0][0], r2[0][1], r2[1][1]};
            const float c6[6] = {r1[0], r2[0][0], r2[0][1], r3[0][0][0], r3[0][0][1], r3[0][1][1]};
            const float d6[6] = {r1[1], r2[0][1], r2[1][1], r3[0][0][1], r3[0][1][1], r3[1][1][1]};
#pragma unroll
            for (int q = 0; q < 6; q++)
            {
                A6[q] = g0 * m[q];
                B6[q] = h0 * b6[q];
                C6[q] = h0 * c6[q];
                D6[q] = h0 * d6[q];
            }
        }
        else
        {
#pragma unroll
            for (int q = 0; q < 6; q++)
                A6[q] = B6[q] = C6[q] = D6[q] = 0.f;
            for (int d = 0; d < a.nd; d++)
            {
                const float n1 = GRLBM_RN1(d), n2 = GRLBM_RN2(d), w = sw[d];
                float g, h, q1, q2;
                collide_coeffs(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                const float mu[6] = {1.f, n1, n2, n1 * n1, n1 * n2, n2 * n2};
                const float gs = w * g * S[(unsigned)d * nxy], wh = w * h;
#pragma unroll
                for (int q = 0; q < 6; q++)
                {
                    A6[q] += gs * mu[q];
                    B6[q] += wh * mu[q];
                    C6[q] += wh * q1 * mu[q];
                    D6[q] += wh * q2 * mu[q];
                }
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
            const float e = eta + k0 * fE;
            const float prev[6] = {pE, pFx, pFy, pPxx, pPxy, pPyy};
            float s2 = 0.f;
#pragma unroll
            for (int q = 0; q < 6; q++)
            {
                m[q] = A6[q] + e * B6[q] + k3 * (fFx * C6[q] + fFy * D6[q]);
                const float x = (prev[q] - m[q]) / m[q];
                s2 += x * x;
            }
            diff = sqrtf(s2);
        }
        // the intensities of the last iterate; its moments m, the affine
        // map's moments of exactly these intensities, are the stored ones
        const float e = eta + k0 * fE;
        const float scale = CURVED ? a.ia3[ij] : 1.f;
        float *out = a.Iout + (unsigned)i + (unsigned)j * a.pitch;
        for (int d0 = 0; d0 < a.nd; d0 += kChunk)
        {
            float Sv[kChunk];
#pragma unroll
            for (int k = 0; k < kChunk; k++)
                Sv[k] = d0 + k < a.nd ? S[(unsigned)(d0 + k) * nxy] : 0.f;
#pragma unroll
            for (int k = 0; k < kChunk; k++)
            {
                const int d = d0 + k;
                if (d >= a.nd)
                    break;
                const float n1 = GRLBM_RN1(d), n2 = GRLBM_RN2(d);
                float g = g0, h = h0, q1 = n1, q2 = n2;
                if (!rest)
                    collide_coeffs(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                const float v = g * Sv[k] + h * (e + k3 * (q1 * fFx + q2 * fFy));
                out[(unsigned)d * a.plane] = v * scale;
            }
        }
    }
#undef GRLBM_RN1
#undef GRLBM_RN2
    if (active)
    {
#pragma unroll
        for (int q = 0; q < 6; q++)
            a.mom[(unsigned)ij + q * nxy] = m[q];
    }
    // lambda-iteration statistics: warp sums and maxima, one atomic per warp
    unsigned sum = (unsigned)cycles, mx = (unsigned)cycles;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0 && sum)
    {
        atomicAdd(a.iter_sum, (unsigned long long)sum);
        atomicMax(a.iter_max, mx);
    }
}

// The bounded staging wait on its own: one block waits on a phase of its
// mbarrier that nothing completes (arrive = 0) or that thread 0 completes
// (arrive = 1); the wait returns either way.
__global__ void k_wait_selftest(int arrive, unsigned long long limit_ns, int *completed, unsigned long long *waited_ns)
{
    __shared__ __align__(8) unsigned long long bar_word;
    const unsigned bar = smem_addr(&bar_word);
    if (threadIdx.x == 0)
        mbar_init(bar, 1);
    __syncthreads();
    if (arrive && threadIdx.x == 0)
        mbar_arrive_expect(bar, 0u);
    const unsigned long long t0 = global_ns();
    const bool done = mbar_wait(bar, 0u, limit_ns, nullptr);
    const unsigned long long t1 = global_ns();
    if (threadIdx.x == 0)
    {
        *completed = done ? 1 : 0;
        *waited_ns = t1 - t0;
    }
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }
} // namespace

cudaError_t run_wait_selftest(int arrive, unsigned long long limit_ns, int *completed, unsigned long long *waited_ns)
{
    void *buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, 16);
    if (e != cudaSuccess)
        return e;
    int *d_done = static_cast<int *>(buf);
    unsigned long long *d_ns = reinterpret_cast<unsigned long long *>(static_cast<char *>(buf) + 8);
    k_wait_selftest<<<1, 32>>>(arrive, limit_ns, d_done, d_ns);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(completed, d_done, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(waited_ns, d_ns, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    return e;
}

__global__ void k_coef_about_node32(GridDev g, const double *coef, float *coef32, int nf)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per = g.nxy * nf;
    if (t >= 5 * per)
        return;
    const int64_t q = t / per, r = t - q * per; // r = k * nxy + ij
    const int64_t k = r / g.nxy, ij = r - k * g.nxy;
    double v = coef[q * per + ij * nf + k];
    if (k == 0 && q == 1)
        v -= g.startx + (double)(ij % g.nx) * g.dx;
    else if (k == 0 && q == 2)
        v -= g.starty + (double)(ij / g.nx) * g.dy;
    coef32[t] = (float)v;
}
void launch_coef_about_node32(const GridDev &g, const double *coef, float *coef32, int nf, cudaStream_t s)
{
    k_coef_about_node32<<<nblk(5 * g.nxy * nf, 256), 256, 0, s>>>(g, coef, coef32, nf);
}

void launch_step_prec_adaptive(const PrecStepArgs &a, const DirTable &dt, bool curved, cudaStream_t s)
{
    const int64_t rows = a.g.jhi - a.g.jlo;
    if (rows <= 0 || a.g.nx_ <= 0)
        return;
    const unsigned tx = nblk(a.g.nx_, kATileX), ty = nblk(rows, kATileY);
    // UpdateRotationMatrizes from the previous moments, before the stream
    launch_rotation_update32(a.g, a.mom, a.ang_old, const_cast<double *>(a.ang_new), s);
    launch_rotation_trig32(a.g.nxy, a.ang_old, a.ang_new, const_cast<float2 *>(a.rot_inv),
                           const_cast<float2 *>(a.rot_new), s);
    const dim3 cgrid(tx, ty);
    if (curved)
    {
        const dim3 sgrid(nblk(a.nd, kADirs) * (unsigned)rows, tx);
        const size_t coef_bytes = (size_t)5 * a.nf * kATileX * sizeof(float);
        k_stream_prec_adaptive_curved<<<sgrid, kAdaptiveBlock, coef_bytes, s>>>(a);
        k_collide_prec_adaptive<true><<<cgrid, kStepBlock, 0, s>>>(a, dt);
    }
    else
    {
        k_stream_prec_adaptive_flat<<<dim3((unsigned)a.nd, tx, ty), kStepBlock, 0, s>>>(a);
        k_collide_prec_adaptive<false><<<cgrid, kStepBlock, 0, s>>>(a, dt);
    }
    // the halo moments, which the reference recomputes from unwritten (zero) intensities
    launch_zero_halo_moments32(a.g, a.mom, s);
}

} // namespace grlbm
