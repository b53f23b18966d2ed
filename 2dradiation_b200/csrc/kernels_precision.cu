// Precision form of the radiation step: FP32 intensities and stream/collide
// arithmetic (contracted FMAs allowed), Kahan-compensated FP32 moment sums,
// on departure records derived from the FP64 geodesic tables.
//
// State: for curved streaming the stored intensity is J = I / alpha^3 (I
// itself for flat streaming).  The reference multiplies each corner's
// angular interpolation by (alpha_c / alpha_n)^3 after clamping it at zero
// (src/Radiation.cpp:502-505, 342); as alpha_n^-3 > 0 commutes with the clamp,
// gathering J gives the same value without loading alpha at every corner.
//
// Stream: one thread per interior cell loops over the directions; each
// (cell, direction) reads a 16-byte record and a 48-byte angular row (the
// two cubic rows of IntensityAt pre-blended into a 5-direction window whose
// weights are W0 + t D), gathers the window at the 4 bilinear corners and
// multiplies by s^3 alpha_c^3.  Offsets are 32-bit.
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

// Moment sums compensated per block of directions: plain FP32 partial sums
// over kBlockDirs directions, folded into Kahan accumulators.
constexpr int kBlockDirs = 8;
struct KMoments
{
    Kahan E, Fx, Fy, Pxx, Pxy, Pyy;
    float p[6];
    int n;
    __device__ __forceinline__ void zero()
    {
        E.zero(), Fx.zero(), Fy.zero(), Pxx.zero(), Pxy.zero(), Pyy.zero();
#pragma unroll
        for (int q = 0; q < 6; q++)
            p[q] = 0.f;
        n = 0;
    }
    __device__ __forceinline__ void fold()
    {
        E.add(p[0]), Fx.add(p[1]), Fy.add(p[2]), Pxx.add(p[3]), Pxy.add(p[4]), Pyy.add(p[5]);
#pragma unroll
        for (int q = 0; q < 6; q++)
            p[q] = 0.f;
        n = 0;
    }
    __device__ __forceinline__ void add(float w, float v, float n1, float n2)
    {
        const float c = w * v;
        const float c1 = c * n1, c2 = c * n2;
        p[0] += c;
        p[1] += c1;
        p[2] += c2;
        p[3] += c1 * n1;
        p[4] += c1 * n2;
        p[5] += c2 * n2;
        if (++n == kBlockDirs)
            fold();
    }
    __device__ __forceinline__ void finish() { fold(); }
};

// Tile of cells per block and the shared-memory stage of the state around it:
// a (kTileX + 2) x (kTileY + 2) patch of each direction plane, for a rolling
// window of planes.  Chunk k covers directions [kChunk k, kChunk (k+1)) and
// reads virtual planes [kChunk k - kBelow, kChunk k + kSpan - kBelow) (a
// departure's angular window starts at most 3 directions below its own and
// spans 5; plane v holds direction v mod nDir).  Plane v lives in ring slot
// (v + kBelow) mod kRing; the next chunk's planes are loaded by cp.async into
// slots the current chunk does not read.
constexpr int kTileX = 32, kTileY = 4;
static_assert(kTileX * kTileY == kStepBlock, "tile = block");
constexpr int kPatchX = kTileX + 2, kPatchY = kTileY + 2, kPatch = kPatchX * kPatchY;
static_assert(kPatch > kStepBlock && kPatch <= 2 * kStepBlock, "two staging loads per thread and plane");
constexpr int kChunk = 8, kBelow = 4, kSpan = kChunk + 8, kRing = 32;
static_assert(kSpan + kChunk <= kRing && (kRing & (kRing - 1)) == 0, "ring");

__device__ __forceinline__ void cp_async4(float *dst, const float *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// this thread's share of one patch plane: patch nodes t and t + kStepBlock
struct StageSlots
{
    int node0, node1;        // patch node indices (node1 < 0: none)
    unsigned goff0, goff1;   // node offsets in a global plane
    bool ok0, ok1;           // node inside the grid
};

__device__ __forceinline__ StageSlots stage_slots(const GridDev &g, int x0, int y0)
{
    StageSlots s;
    const int t = threadIdx.x;
    s.node0 = t;
    int py = t / kPatchX, px = t - py * kPatchX;
    s.ok0 = (x0 + px < (int)g.nx) && (y0 + py < (int)g.ny);
    s.goff0 = (unsigned)((x0 + px) + (y0 + py) * (int)g.nx);
    const int n1 = t + kStepBlock;
    s.node1 = n1 < kPatch ? n1 : -1;
    py = n1 / kPatchX;
    px = n1 - py * kPatchX;
    s.ok1 = s.node1 >= 0 && (x0 + px < (int)g.nx) && (y0 + py < (int)g.ny);
    s.goff1 = (unsigned)((x0 + px) + (y0 + py) * (int)g.nx);
    return s;
}

// stage virtual planes [v0, v0 + n) into their ring slots
__device__ __forceinline__ void stage_planes(const PrecStepArgs &a, const StageSlots &ss, float *ring, int v0, int n)
{
    const unsigned nxy = (unsigned)a.g.nxy;
    int d = v0 % a.nd;
    d = d < 0 ? d + a.nd : d;
    for (int p = 0; p < n; p++)
    {
        float *slot = ring + ((v0 + p + kBelow) & (kRing - 1)) * kPatch;
        const float *plane = a.Iin + (unsigned)d * nxy;
        if (ss.ok0)
            cp_async4(slot + ss.node0, plane + ss.goff0);
        if (ss.ok1)
            cp_async4(slot + ss.node1, plane + ss.goff1);
        d = (d + 1 == a.nd) ? 0 : d + 1;
    }
    cp_async_commit();
}

// cubic Lagrange weights at position f in [0,1) for nodes -1, 0, 1, 2
__device__ __forceinline__ void cubic_weights(float f, float *l)
{
    const float fm = f - 1.f, fp = f + 1.f, f2 = f - 2.f;
    l[0] = -f * fm * f2 * (1.f / 6.f);
    l[1] = fp * fm * f2 * 0.5f;
    l[2] = -fp * f * f2 * 0.5f;
    l[3] = fp * f * fm * (1.f / 6.f);
}

// one stream value from its departure record (curved) or from the flat
// departure of direction d; taps inside the staged patch come from shared
// memory, any other from global memory
template <bool CURVED>
__device__ __forceinline__ float stream_value(const PrecStepArgs &a, const DirTable &dt, const float *ring, int d,
                                              int chunk0, const float4 &r, int i, int j, int x0, int y0)
{
    const int nx = (int)a.g.nx;
    const unsigned nxy = (unsigned)a.g.nxy;
    float fx, fy, w[5];
    int i0, j0, base, ntap;
    if constexpr (CURVED)
    {
        if (r.w == 0.f)
            return 0.f;
        const float fli = floorf(r.x), flj = floorf(r.y);
        fx = r.x - fli;
        fy = r.y - flj;
        i0 = min(max(i + (int)fli, 0), nx - 2);
        j0 = min(max(j + (int)flj, 0), (int)a.g.ny - 2);
        int g = (int)floorf(r.z);
        g = max(0, min(g, a.ng - 1));
        const float t = r.z - (float)g;
        // Row g of the interpolation grid sits at direction coordinate
        // u = g nDir/nGrid - 1/2 and interpolates with the cubic Lagrange
        // polynomial through the 4 directions around it (src/Stencil.cpp:109-162);
        // IntensityAt blends rows g and g+1 linearly in t.
        const float u0 = (float)g * a.dir_per_row - 0.5f;
        const float b0 = floorf(u0), b1 = floorf(u0 + a.dir_per_row);
        float l0[4], l1[4];
        cubic_weights(u0 - b0, l0);
        cubic_weights(u0 + a.dir_per_row - b1, l1);
        const float s = 1.f - t;
        if (b1 == b0)
        {
            w[0] = s * l0[0] + t * l1[0];
            w[1] = s * l0[1] + t * l1[1];
            w[2] = s * l0[2] + t * l1[2];
            w[3] = s * l0[3] + t * l1[3];
            w[4] = 0.f;
            ntap = 4;
        }
        else
        {
            w[0] = s * l0[0];
            w[1] = s * l0[1] + t * l1[0];
            w[2] = s * l0[2] + t * l1[1];
            w[3] = s * l0[3] + t * l1[2];
            w[4] = t * l1[3];
            ntap = 5;
        }
        base = (int)b0 - 1;
        base = base < 0 ? base + a.nd : base;
    }
    else
    {
        const float ox = dt.ox[d], oy = dt.oy[d];
        const float fli = floorf(ox), flj = floorf(oy);
        fx = ox - fli;
        fy = oy - flj;
        i0 = min(max(i + (int)fli, 0), nx - 2);
        j0 = min(max(j + (int)flj, 0), (int)a.g.ny - 2);
        w[0] = 1.f;
        w[1] = w[2] = w[3] = w[4] = 0.f;
        base = d;
        ntap = 1;
    }
    const int lx = i0 - x0, ly = j0 - y0;
    // window start relative to the chunk's first staged plane, modulo nDir
    int rel = base - chunk0 + kBelow;
    rel = rel < 0 ? rel + a.nd : (rel >= a.nd ? rel - a.nd : rel);
    float cv[4];
    if (lx >= 0 && lx <= kTileX && ly >= 0 && ly <= kTileY && rel + ntap <= kSpan)
    {
        const int o = ly * kPatchX + lx;
        const int s0 = chunk0 + rel; // ring slot of the window's first plane
        const float *p0 = ring + (s0 & (kRing - 1)) * kPatch + o;
        const float *pk[5];
#pragma unroll
        for (int k = 0; k < 5; k++)
            pk[k] = ring + ((s0 + k) & (kRing - 1)) * kPatch + o;
        const int off[4] = {0, kPatchX, 1, kPatchX + 1}; // corners 00 01 10 11
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            float v = w[0] * p0[off[q]];
#pragma unroll
            for (int k = 1; k < 5; k++)
                if (k < ntap)
                    v = fmaf(w[k], pk[k][off[q]], v);
            cv[q] = v > 0.f ? v : 0.f;
        }
    }
    else
    {
        const unsigned c00 = (unsigned)(i0 + j0 * nx);
        const unsigned off[4] = {c00, c00 + (unsigned)nx, c00 + 1u, c00 + (unsigned)nx + 1u};
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            float v = 0.f;
#pragma unroll
            for (int k = 0; k < 5; k++)
                if (k < ntap)
                {
                    int dk = base + k;
                    dk = dk >= a.nd ? dk - a.nd : dk;
                    v = fmaf(w[k], __ldg(a.Iin + (unsigned)dk * nxy + off[q]), v);
                }
            cv[q] = v > 0.f ? v : 0.f;
        }
    }
    const float f0 = cv[0] * (1.f - fx) + cv[2] * fx;
    const float f1 = cv[1] * (1.f - fx) + cv[3] * fx;
    const float bil = f0 * (1.f - fy) + f1 * fy;
    return CURVED ? r.w * bil : bil;
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
__global__ void __launch_bounds__(kStepBlock, 6) k_step_prec(PrecStepArgs a, const __grid_constant__ DirTable dt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *ring = reinterpret_cast<float *>(smem_raw);
    const int t = threadIdx.x;
    const int tx = t % kTileX, ty = t / kTileX;
    const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY; // patch origin (node coordinates)
    const int i = 1 + x0 + tx, j = 1 + y0 + ty;
    const bool active = i <= (int)a.g.nx_ && j <= (int)a.g.ny_;
    const int ii = active ? i : 1, jj = active ? j : 1;
    const int ij = ii + jj * (int)a.g.nx;
    const int cc = (ii - 1) + (jj - 1) * (int)a.g.nx_;
    const unsigned nxy = (unsigned)a.g.nxy;
    const uint8_t fl = active ? a.flags[ij] : (uint8_t)3;
    const bool live = active && !(CURVED && (fl & 2));
    const bool collides = active && !(fl & 1);
    // The streamed intensities of a colliding cell wait in its own output
    // slots until the lambda iteration has converged (nothing else reads or
    // writes them in this step).
    float *Is = a.Iout + (unsigned)ij;

    const StageSlots ss = stage_slots(a.g, x0, y0);
    stage_planes(a, ss, ring, -kBelow, kSpan);

    KMoments km;
    km.zero();
    // records are read once per step: streaming loads, prefetched two
    // directions ahead, two directions per iteration
    const float4 *rp = a.rec + cc;
    const unsigned rs = (unsigned)a.g.ncell;
    const float4 none = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 r0 = none, r1 = none;
    if (CURVED && live)
    {
        r0 = __ldcs(rp);
        if (a.nd > 1)
            r1 = __ldcs(rp + rs);
    }
    int chunk0 = 0;
    for (int d = 0; d < a.nd; d += 2)
    {
        if (d % kChunk == 0)
        {
            chunk0 = d;
            cp_async_wait_all();
            __syncthreads(); // this chunk's planes visible; the previous chunk is done with its slots
            if (d + kChunk < a.nd)
                stage_planes(a, ss, ring, d + kSpan - kBelow, kChunk);
        }
        float4 r2 = none, r3 = none;
        if (CURVED && live)
        {
            if (d + 2 < a.nd)
                r2 = __ldcs(rp + (unsigned)(d + 2) * rs);
            if (d + 3 < a.nd)
                r3 = __ldcs(rp + (unsigned)(d + 3) * rs);
        }
        const bool second = d + 1 < a.nd;
        const float v0 = live ? stream_value<CURVED>(a, dt, ring, d, chunk0, r0, ii, jj, x0, y0) : 0.f;
        const float v1 = (live && second) ? stream_value<CURVED>(a, dt, ring, d + 1, chunk0, r1, ii, jj, x0, y0) : 0.f;
        if (collides)
        {
            Is[(unsigned)d * nxy] = v0;
            if (second)
                Is[(unsigned)(d + 1) * nxy] = v1;
        }
        km.add(dt.w[d], v0, dt.n1[d], dt.n2[d]);
        if (second)
            km.add(dt.w[d + 1], v1, dt.n1[d + 1], dt.n2[d + 1]);
        r0 = r2;
        r1 = r3;
    }
    km.finish();
    float m[6] = {km.E.s, km.Fx.s, km.Fy.s, km.Pxx.s, km.Pxy.s, km.Pyy.s};

    int cycles = 0;
    if (collides)
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
            for (int d = 0; d < a.nd; d++)
            {
                const float n1 = dt.n1[d], n2 = dt.n2[d], w = dt.w[d];
                float g, h, q1, q2;
                collide_coeffs(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                const float mu[6] = {1.f, n1, n2, n1 * n1, n1 * n2, n2 * n2};
                const float gs = w * g * Is[(unsigned)d * nxy], wh = w * h;
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
        // write the last iterate; its compensated sums are the stored moments
        km.zero();
        const float e = eta + k0 * fE;
        const float scale = CURVED ? a.ia3[ij] : 1.f;
        const float ra = h0 * e, rb1 = h0 * k3 * fFx, rb2 = h0 * k3 * fFy;
        for (int d0 = 0; d0 < a.nd; d0 += 8)
        {
            // the parked stream values of 8 directions, loaded together
            float S[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
                S[k] = (d0 + k < a.nd) ? Is[(unsigned)(d0 + k) * nxy] : 0.f;
#pragma unroll
            for (int k = 0; k < 8; k++)
            {
                const int d = d0 + k;
                if (d >= a.nd)
                    break;
                const float n1 = dt.n1[d], n2 = dt.n2[d];
                float v;
                if (rest)
                    v = fmaf(g0, S[k], fmaf(rb1, n1, fmaf(rb2, n2, ra)));
                else
                {
                    float g, h, q1, q2;
                    collide_coeffs(n1, n2, u1, u2, lor, adt, kak0, g, h, q1, q2);
                    v = g * S[k] + h * (e + k3 * (q1 * fFx + q2 * fFy));
                }
                Is[(unsigned)d * nxy] = v * scale;
                km.add(dt.w[d], v, n1, n2);
            }
        }
        km.finish();
        m[0] = km.E.s, m[1] = km.Fx.s, m[2] = km.Fy.s, m[3] = km.Pxx.s, m[4] = km.Pxy.s, m[5] = km.Pyy.s;
    }
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
    if ((t & 31) == 0 && sum)
    {
        atomicAdd(a.iter_sum, (unsigned long long)sum);
        atomicMax(a.iter_max, mx);
    }
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }
} // namespace

size_t step_prec_smem(int) { return (size_t)kRing * kPatch * sizeof(float); }

cudaError_t prepare_step_prec(int smem_bytes)
{
    cudaError_t e = cudaFuncSetAttribute(k_step_prec<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_step_prec<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
}
void launch_step_prec(const PrecStepArgs &a, const DirTable &dt, bool curved, cudaStream_t s)
{
    const size_t smem = step_prec_smem(a.nd);
    const dim3 grid(nblk(a.g.nx_, kTileX), nblk(a.g.ny_, kTileY));
    if (curved)
        k_step_prec<true><<<grid, kStepBlock, smem, s>>>(a, dt);
    else
        k_step_prec<false><<<grid, kStepBlock, smem, s>>>(a, dt);
}
} // namespace grlbm
