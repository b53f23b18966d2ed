// Precision form of the radiation step: FP32 intensities and stream/collide
// arithmetic (contracted FMAs allowed), Kahan-compensated FP32 moment sums,
// on departure records derived from the FP64 geodesic tables.
//
// Stream: one thread per interior cell loops over the directions; each
// (cell, direction) reads a 16-byte record, gathers the 4 bilinear corners
// of a <= 5-direction angular window (the two cubic rows of IntensityAt
// blended into one set of weights) and applies (s alpha_c / alpha_n)^3.
//
// Collide: the lambda iteration of src/Radiation.cpp:661-722 is affine in
// the previous moments -- I_d = g_d S_d + h_d (eta + kappa0 E_ff + 3 kappa1
// nFF_d . F_ff) -- so each iteration is evaluated on the six moments with
// per-cell sums of the direction terms (O(1) per iteration instead of a pass
// over the directions); the converged intensities are written in one final
// pass whose Kahan sums give the stored moments.
#include "device_common.cuh"

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

struct KMoments
{
    Kahan E, Fx, Fy, Pxx, Pxy, Pyy;
    __device__ __forceinline__ void zero()
    {
        E.zero(), Fx.zero(), Fy.zero(), Pxx.zero(), Pxy.zero(), Pyy.zero();
    }
    __device__ __forceinline__ void add(float w, float v, float n1, float n2)
    {
        const float c = w * v;
        const float c1 = c * n1, c2 = c * n2;
        E.add(c);
        Fx.add(c1);
        Fy.add(c2);
        Pxx.add(c1 * n1);
        Pxy.add(c1 * n2);
        Pyy.add(c2 * n2);
    }
};

template <bool CURVED>
__device__ __forceinline__ float stream_value(const PrecStepArgs &a, int d, int64_t c, int64_t i, int64_t j, int64_t ij)
{
    const int64_t nxy = a.g.nxy, nx = a.g.nx;
    if constexpr (CURVED)
    {
        const float4 r = a.rec[(int64_t)d * a.g.ncell + c];
        if (r.w == 0.f)
            return 0.f;
        const float fli = floorf(r.x), flj = floorf(r.y);
        const float fx = r.x - fli, fy = r.y - flj;
        const int64_t i0 = min(max(i + (int64_t)fli, (int64_t)0), nx - 2);
        const int64_t j0 = min(max(j + (int64_t)flj, (int64_t)0), a.g.ny - 2);
        const int64_t c00 = i0 + j0 * nx;
        int g0 = (int)floorf(r.z);
        g0 = max(0, min(g0, a.ng - 1));
        const float tt = r.z - (float)g0;
        const int g1 = (g0 + 1 == a.ng) ? 0 : g0 + 1;
        const int base = __ldg(a.ig_base + g0);
        const int shift = __ldg(a.ig_shift + g0);
        const float u = 1.f - tt;
        float w[5];
#pragma unroll
        for (int k = 0; k < 4; k++)
            w[k] = u * __ldg(a.ig_w + 4 * g0 + k);
        w[4] = 0.f;
#pragma unroll
        for (int k = 0; k < 4; k++)
        {
            const float b = tt * __ldg(a.ig_w + 4 * g1 + k);
            if (shift == 0)
                w[k] += b;
            else
                w[k + 1] += b;
        }
        const float *plane[5];
#pragma unroll
        for (int k = 0; k < 5; k++)
        {
            int dk = base + k;
            dk = dk >= a.nd ? dk - a.nd : dk;
            plane[k] = a.Iin + (int64_t)dk * nxy;
        }
        const int64_t corner[4] = {c00, c00 + nx, c00 + 1, c00 + 1 + nx}; // 00 01 10 11
        float cv[4];
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            float v = w[0] * __ldg(plane[0] + corner[q]);
#pragma unroll
            for (int k = 1; k < 4; k++)
                v += w[k] * __ldg(plane[k] + corner[q]);
            if (shift)
                v += w[4] * __ldg(plane[4] + corner[q]);
            v = v > 0.f ? v : 0.f;
            cv[q] = v * __ldg(a.ia3 + corner[q]);
        }
        const float f0 = cv[0] * (1.f - fx) + cv[2] * fx;
        const float f1 = cv[1] * (1.f - fx) + cv[3] * fx;
        return r.w * (f0 * (1.f - fy) + f1 * fy);
    }
    else
    {
        const double xt = (a.g.startx + (double)i * a.g.dx) - __ldg(a.cx + d) * a.g.dt;
        const double yt = (a.g.starty + (double)j * a.g.dy) - __ldg(a.cy + d) * a.g.dt;
        const double it = (xt - a.g.startx) / a.g.dx, jt = (yt - a.g.starty) / a.g.dy;
        const int64_t i0 = min(max((int64_t)floor(it), (int64_t)0), nx - 2);
        const int64_t j0 = min(max((int64_t)floor(jt), (int64_t)0), a.g.ny - 2);
        const float fx = (float)(it - (double)i0), fy = (float)(jt - (double)j0);
        const float *plane = a.Iin + (int64_t)d * nxy;
        const int64_t c00 = i0 + j0 * nx;
        const float f0 = __ldg(plane + c00) * (1.f - fx) + __ldg(plane + c00 + 1) * fx;
        const float f1 = __ldg(plane + c00 + nx) * (1.f - fx) + __ldg(plane + c00 + nx + 1) * fx;
        return f0 * (1.f - fy) + f1 * fy;
    }
}

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

template <bool CURVED>
__global__ void __launch_bounds__(kStepBlock) k_step_prec(PrecStepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *Is = reinterpret_cast<float *>(smem_raw);
    const int t = threadIdx.x;
    const int64_t c = (int64_t)blockIdx.x * kStepBlock + t;
    const bool active = c < a.g.ncell;
    const int64_t cc = active ? c : 0;
    const int64_t i = 1 + cc % a.g.nx_, j = 1 + cc / a.g.nx_;
    const int64_t ij = i + j * a.g.nx;
    const int64_t nxy = a.g.nxy;
    const uint8_t fl = active ? a.flags[ij] : (uint8_t)3;
    const bool zero_stream = CURVED && (fl & 2);

    KMoments km;
    km.zero();
    for (int d = 0; d < a.nd; d++)
    {
        const float val = (active && !zero_stream) ? stream_value<CURVED>(a, d, cc, i, j, ij) : 0.f;
        Is[d * kStepBlock + t] = val;
        km.add(__ldg(a.w + d), val, __ldg(a.n1 + d), __ldg(a.n2 + d));
    }
    float m[6] = {km.E.s, km.Fx.s, km.Fy.s, km.Pxx.s, km.Pxy.s, km.Pyy.s};

    int cycles = 0;
    if (active && !(fl & 1))
    {
        const float u1 = a.u1[ij], u2 = a.u2[ij], lor = a.lor[ij], adt = a.adt[ij];
        const float eta = a.eta[ij], k0 = a.k0[ij], k3 = a.k3[ij], kak0 = a.ka[ij] + a.k0[ij];
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
                B6[q] = h0 * __ldg(a.wmom + q);
                C6[q] = h0 * __ldg(a.wmom + 6 + q);
                D6[q] = h0 * __ldg(a.wmom + 12 + q);
            }
        }
        else
        {
#pragma unroll
            for (int q = 0; q < 6; q++)
                A6[q] = B6[q] = C6[q] = D6[q] = 0.f;
            for (int d = 0; d < a.nd; d++)
            {
                const float n1 = __ldg(a.n1 + d), n2 = __ldg(a.n2 + d), w = __ldg(a.w + d);
                float g, h, q1, q2;
                collide_coeffs(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                const float mu[6] = {1.f, n1, n2, n1 * n1, n1 * n2, n2 * n2};
                const float gs = w * g * Is[d * kStepBlock + t], wh = w * h;
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
            const float r = lor / (1.f + lor) * ((2.f * lor + 1.f) * uF - lor * uuP);
            fFx = lor * lor * (pFx - lor * pE * u1 - uxP + u1 * r);
            fFy = lor * lor * (pFy - lor * pE * u2 - uyP + u2 * r);
            const float e = eta + k0 * fE;
            float prev[6] = {pE, pFx, pFy, pPxx, pPxy, pPyy};
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
        // write the last iterate; its Kahan sums are the stored moments
        km.zero();
        const float e = eta + k0 * fE;
        for (int d = 0; d < a.nd; d++)
        {
            const float n1 = __ldg(a.n1 + d), n2 = __ldg(a.n2 + d);
            float v;
            if (rest)
                v = g0 * Is[d * kStepBlock + t] + h0 * (e + k3 * (n1 * fFx + n2 * fFy));
            else
            {
                float g, h, q1, q2;
                collide_coeffs(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                v = g * Is[d * kStepBlock + t] + h * (e + k3 * (q1 * fFx + q2 * fFy));
            }
            a.Iout[(int64_t)d * nxy + ij] = v;
            km.add(__ldg(a.w + d), v, n1, n2);
        }
        m[0] = km.E.s, m[1] = km.Fx.s, m[2] = km.Fy.s, m[3] = km.Pxx.s, m[4] = km.Pxy.s, m[5] = km.Pyy.s;
    }
    if (active)
    {
#pragma unroll
        for (int q = 0; q < 6; q++)
            a.mom[ij + q * nxy] = m[q];
    }
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

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }
} // namespace

cudaError_t prepare_step_prec(int smem_bytes)
{
    cudaError_t e = cudaFuncSetAttribute(k_step_prec<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_step_prec<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
}
void launch_step_prec(const PrecStepArgs &a, bool curved, cudaStream_t s)
{
    const size_t smem = (size_t)a.nd * kStepBlock * sizeof(float);
    if (curved)
        k_step_prec<true><<<nblk(a.g.ncell, kStepBlock), kStepBlock, smem, s>>>(a);
    else
        k_step_prec<false><<<nblk(a.g.ncell, kStepBlock), kStepBlock, smem, s>>>(a);
}
} // namespace grlbm
