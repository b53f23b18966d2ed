// Hand-written adjoint of the plain step (stream + collide) for a fluid at
// rest without anisotropic scattering (u = 0, kappa1 = 0), the setting of
// gradient-based fitting of the emissivity eta, absorption kappaA and
// scattering kappa0 fields.
//
// Forward step n (src/Radiation.cpp:454-512, 641-736 with u = 0, kappa1 = 0):
//   S_d(c)   = s^3 sum_q b_q cube_q max(0, (1-t) sum_k w0_k I[idx0_k](n_q) + t sum_k w1_k I[idx1_k](n_q))
//   E_0      = sum_d w_d S_d,   E_k = (E_0 + adt W (eta + kappa0 E_{k-1})) / D,  W = sum_d w_d
//   I'_d(c)  = (S_d + adt (eta + kappa0 E_{K-1})) / D,  D = 1 + adt (kappaA + kappa0)
// with K the cell's lambda-iteration count of that step (recorded by the
// forward, so the adjoint is that of the iteration actually run).
//
// Adjoint step: the collide part is per cell and closed-form (k_adj_collide);
// the stream part is the transpose of a fixed linear gather (up to the clamp
// masks, recorded per corner), evaluated as an atomic-free gather over an
// inverse table in CSR form: for every target (direction d', node n) the
// list of (source (d, c), corner q, weight) whose stream reads I[d'](n).
// The table is built once per set of geodesic tables: every (d, c) writes its
// up to 32 entries at fixed slots, a stable radix sort on (target, source)
// orders them, entries of the same (target, source, corner) -- the two
// interpolation rows reading one direction -- are merged, and a binary search
// per target gives the row lengths: the order, and so every sum, is
// deterministic.  The rows are stored sliced (32 targets per slice, each
// slice as wide as its longest row, entry k of the slice's rows contiguous),
// so that the 32 threads of a warp read consecutive words.
//
// Adjoint state and table weights are FP32; the gradients accumulate in FP64.
#include <cub/cub.cuh>

#include <algorithm>

#include "device_common.cuh"

namespace grlbm
{
namespace
{
constexpr int kEntriesCurved = 32, kEntriesFlat = 4;
constexpr unsigned long long kNoEntry = ~0ull;
constexpr int kMaxCycles = 100; // the lambda iteration's cap (src/Radiation.cpp:16)

__global__ void __launch_bounds__(128) k_adj_entries(AdjEntryArgs a, unsigned long long *keys, float *vals)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n_src = (int64_t)a.nd * a.g.ncell;
    if (tid >= n_src)
        return;
    const int per = a.curved ? kEntriesCurved : kEntriesFlat;
    unsigned long long *K = keys + tid * per;
    float *V = vals + tid * per;
    for (int e = 0; e < per; e++)
        K[e] = kNoEntry, V[e] = 0.f;
    const int d = (int)(tid / a.g.ncell);
    const int64_t c = tid - (int64_t)d * a.g.ncell;
    const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
    const int64_t ij = i + j * a.g.nx, nx = a.g.nx, nxy = a.g.nxy;
    if (a.curved && (a.flags[ij] & 2)) // zero stream (inside the excision)
        return;
    const unsigned long long src4 = (unsigned long long)tid * 4ull;
    if (a.curved)
    {
        const double4 r = a.rec[tid];
        if (r.z < 0.0)
            return;
        const int64_t i0 = min(max((int64_t)floor(r.x), (int64_t)0), nx - 2);
        const int64_t j0 = min(max((int64_t)floor(r.y), (int64_t)0), a.g.ny - 2);
        int g0 = (int)floor(r.z) % a.ng;
        g0 = g0 < 0 ? 0 : g0;
        const int g1 = (g0 + 1) % a.ng;
        const double t = r.z - (double)g0;
        const IgRow R0 = a.ig_rows[g0], R1 = a.ig_rows[g1];
        const int idx[8] = {R0.idx.x, R0.idx.y, R0.idx.z, R0.idx.w, R1.idx.x, R1.idx.y, R1.idx.z, R1.idx.w};
        const double wt[8] = {(1.0 - t) * R0.w01.x, (1.0 - t) * R0.w01.y, (1.0 - t) * R0.w23.x, (1.0 - t) * R0.w23.y,
                              t * R1.w01.x,         t * R1.w01.y,         t * R1.w23.x,         t * R1.w23.y};
        const double fx = r.x - (double)i0, fy = r.y - (double)j0;
        const double al = a.alpha[ij];
        for (int q = 0; q < 4; q++) // corners 00, 01, 10, 11
        {
            const int64_t ci = i0 + (q >> 1), cj = j0 + (q & 1);
            const int64_t n = ci + cj * nx;
            const int64_t di = ci - i, dj = cj - j;
            double cube;
            if (di >= -1 && di <= 1 && dj >= -1 && dj <= 1)
                cube = a.acube[ij * 9 + 3 * (dj + 1) + (di + 1)];
            else
            {
                const double rr = al / a.alpha[n];
                cube = rr * (rr * rr);
            }
            const double bq = ((q >> 1) ? fx : 1.0 - fx) * ((q & 1) ? fy : 1.0 - fy);
            const double f = r.w * bq * cube;
            for (int k = 0; k < 8; k++)
            {
                K[8 * q + k] = ((unsigned long long)((int64_t)idx[k] * nxy + n) << 32) | (src4 + (unsigned)q);
                V[8 * q + k] = (float)(f * wt[k]);
            }
        }
    }
    else
    {
        // StreamFlatFixed's departure point (src/Radiation.cpp:394-410)
        double xt = a.g.startx + (double)i * a.g.dx, yt = a.g.starty + (double)j * a.g.dy;
        xt -= a.cx[d] * a.g.dt;
        yt -= a.cy[d] * a.g.dt;
        const double it = (xt - a.g.startx) / a.g.dx, jt = (yt - a.g.starty) / a.g.dy;
        const int64_t i0 = min(max((int64_t)floor(it), (int64_t)0), nx - 2);
        const int64_t j0 = min(max((int64_t)floor(jt), (int64_t)0), a.g.ny - 2);
        const double fx = it - (double)i0, fy = jt - (double)j0;
        for (int q = 0; q < 4; q++)
        {
            const int64_t n = (i0 + (q >> 1)) + (j0 + (q & 1)) * nx;
            const double bq = ((q >> 1) ? fx : 1.0 - fx) * ((q & 1) ? fy : 1.0 - fy);
            K[q] = ((unsigned long long)((int64_t)d * nxy + n) << 32) | (src4 + (unsigned)q);
            V[q] = (float)bq;
        }
    }
}

// row offsets: first sorted entry of each target (binary search)
__global__ void k_adj_offsets(const unsigned long long *keys, int64_t n, int64_t n_targets, int64_t *offsets)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_targets)
        return;
    const unsigned long long key = (unsigned long long)t << 32;
    int64_t lo = 0, hi = n;
    while (lo < hi)
    {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    offsets[t] = lo;
}

// slice widths: the longest row of each slice of kSlice targets
constexpr int kSlice = 32;
__global__ void k_adj_slice_width(const int64_t *offsets, int64_t n_targets, int64_t n_slices, int64_t *width)
{
    const int64_t sl = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= n_slices)
        return;
    int64_t w = 0;
    for (int64_t t = sl * kSlice; t < min((sl + 1) * kSlice, n_targets); t++)
        w = max(w, offsets[t + 1] - offsets[t]);
    width[sl] = w * kSlice;
}

// rows into the sliced layout, short rows padded with weight 0
__global__ void k_adj_slice_fill(const int64_t *offsets, const unsigned long long *keys, const float *vals,
                                 const int64_t *slice_start, int64_t n_targets, unsigned *srcq, float *coef)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_targets)
        return;
    const int64_t sl = t / kSlice, lane = t % kSlice;
    const int64_t base = slice_start[sl], width = (slice_start[sl + 1] - base) / kSlice;
    const int64_t e0 = offsets[t], cnt = offsets[t + 1] - e0;
    for (int64_t k = 0; k < width; k++)
    {
        const int64_t dst = base + k * kSlice + lane;
        srcq[dst] = k < cnt ? (unsigned)(keys[e0 + k] & 0xffffffffull) : 0u;
        coef[dst] = k < cnt ? vals[e0 + k] : 0.f;
    }
}

// adjoint of the final moments E: lambda_I[d](ij) = w_d dL/dE(ij) at colliding cells
__global__ void k_adj_seed(GridDev g, int nd, const double *w, const uint8_t *flags, const double *dLdE, float *lam)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nd * g.nxy)
        return;
    const int d = (int)(t / g.nxy);
    const int64_t ij = t - (int64_t)d * g.nxy;
    const int64_t i = ij % g.nx, j = ij / g.nx;
    const bool interior = i >= 1 && i <= g.nx_ && j >= 1 && j <= g.ny_;
    lam[t] = (interior && !(flags[ij] & 1)) ? (float)(w[d] * dLdE[ij]) : 0.f;
}

// Collide adjoint, one thread per interior cell.
__global__ void __launch_bounds__(128) k_adj_collide(AdjCollideArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.g.ncell)
        return;
    const int64_t i = 1 + c % a.g.nx_, j = 1 + c / a.g.nx_;
    const int64_t ij = i + j * a.g.nx, nxy = a.g.nxy, ncell = a.g.ncell;
    const int nd = a.nd;
    if (a.flags[ij] & 1)
    {
        for (int d = 0; d < nd; d++)
            a.lamS[(int64_t)d * ncell + c] = 0.f;
        return;
    }
    const double adt = a.adt[ij], eta = a.eta[ij], k0 = a.k0[ij], ka = a.ka[ij];
    const double D = 1.0 + adt * (ka + k0);
    const int K = a.cycles[c];
    const double E0 = a.e0[c];
    double W = 0.0, Lsum = 0.0, LI = 0.0;
    for (int d = 0; d < nd; d++)
    {
        const double l = (double)a.lam[(int64_t)d * nxy + ij];
        W += a.w[d];
        Lsum += l;
        LI += l * a.Iout[(int64_t)d * nxy + ij];
    }
    // the iterates E_0 .. E_{K-1}
    double Ek[kMaxCycles + 1];
    Ek[0] = E0;
    const int kh = min(max(K - 1, 0), kMaxCycles);
    for (int k = 1; k <= kh; k++)
        Ek[k] = (E0 + adt * W * (eta + k0 * Ek[k - 1])) / D;
    const double Ehat = Ek[kh];
    double lE = Lsum * adt * k0 / D; // adjoint of E_{K-1}
    double l_eta = Lsum * adt / D, l_k0 = Lsum * adt * Ehat / D, l_D = -LI / D, l_Sbar = 0.0;
    for (int k = kh; k >= 1; k--)
    {
        l_Sbar += lE / D;
        l_eta += lE * adt * W / D;
        l_k0 += lE * adt * W * Ek[k - 1] / D;
        l_D -= lE * Ek[k] / D;
        lE = lE * adt * k0 * W / D;
    }
    l_Sbar += lE;
    for (int d = 0; d < nd; d++)
    {
        const double l = (double)a.lam[(int64_t)d * nxy + ij];
        a.lamS[(int64_t)d * ncell + c] = (float)(l / D + a.w[d] * l_Sbar);
    }
    a.g_eta[ij] += l_eta;
    a.g_ka[ij] += adt * l_D;
    a.g_k0[ij] += l_k0 + adt * l_D;
}

// Stream adjoint: lambda[d'](n) = sum over the inverse-table row of (d', n)
// of weight * (corner kept by the clamp) * lambda_S(source), rows read from
// the sliced layout.
__global__ void __launch_bounds__(256) k_adj_stream(const int64_t *slice_start, const unsigned *srcq,
                                                    const float *coef, const uint8_t *clamp, const float *lamS,
                                                    int64_t n_targets, float *lam)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_targets)
        return;
    const int64_t sl = t / kSlice;
    const int64_t e1 = slice_start[sl + 1];
    float acc = 0.f;
    for (int64_t e = slice_start[sl] + t % kSlice; e < e1; e += kSlice)
    {
        const unsigned sq = __ldcs(srcq + e);
        const float w = __ldcs(coef + e);
        const unsigned src = sq >> 2;
        const bool kept = clamp ? ((clamp[src] >> (sq & 3u)) & 1u) : true;
        if (kept)
            acc = fmaf(w, lamS[src], acc);
    }
    lam[t] = acc;
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }
} // namespace

int64_t adj_entries_per_source(bool curved) { return curved ? kEntriesCurved : kEntriesFlat; }

cudaError_t adj_build_table(const AdjEntryArgs &a, int64_t *slice_start, unsigned **srcq_out, float **coef_out,
                            int64_t *n_entries_out, cudaStream_t s)
{
    const int64_t n_src = (int64_t)a.nd * a.g.ncell;
    const int64_t n = n_src * adj_entries_per_source(a.curved);
    const int64_t n_targets = (int64_t)a.nd * a.g.nxy;
    const int64_t n_slices = (n_targets + kSlice - 1) / kSlice;
    unsigned long long *k0 = nullptr, *k1 = nullptr, *uk = nullptr;
    float *v0 = nullptr, *v1 = nullptr, *uv = nullptr;
    int64_t *offsets = nullptr, *n_unique_d = nullptr, *widths = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, tmp2 = 0;
    int64_t n_unique = 0, total = 0;
    cudaError_t e = cudaSuccess;
    *srcq_out = nullptr;
    *coef_out = nullptr;
    cub::DoubleBuffer<unsigned long long> kb;
    cub::DoubleBuffer<float> vb;
#define ADJ_TRY(x)                                                                                             \
    do                                                                                                         \
    {                                                                                                          \
        if ((e = (x)) != cudaSuccess)                                                                          \
            goto done;                                                                                         \
    } while (0)
    ADJ_TRY(cudaMallocAsync(&k0, n * sizeof(unsigned long long), s));
    ADJ_TRY(cudaMallocAsync(&k1, n * sizeof(unsigned long long), s));
    ADJ_TRY(cudaMallocAsync(&v0, n * sizeof(float), s));
    ADJ_TRY(cudaMallocAsync(&v1, n * sizeof(float), s));
    ADJ_TRY(cudaMallocAsync(&offsets, (n_targets + 1) * sizeof(int64_t), s));
    ADJ_TRY(cudaMallocAsync(&n_unique_d, sizeof(int64_t), s));
    ADJ_TRY(cudaMallocAsync(&widths, (n_slices + 1) * sizeof(int64_t), s));
    k_adj_entries<<<nblk(n_src, 128), 128, 0, s>>>(a, k0, v0);
    ADJ_TRY(cudaGetLastError());
    kb = cub::DoubleBuffer<unsigned long long>(k0, k1);
    vb = cub::DoubleBuffer<float>(v0, v1);
    ADJ_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, n, 0, 64, s));
    // merge equal keys (the same target, source and corner) into the other buffers
    uk = kb.Alternate();
    uv = vb.Alternate();
    ADJ_TRY(cub::DeviceReduce::ReduceByKey(nullptr, tmp2, kb.Current(), uk, vb.Current(), uv, n_unique_d,
                                           cub::Sum(), n, s));
    ADJ_TRY(cudaMallocAsync(&tmp, std::max(tmp_bytes, tmp2), s));
    ADJ_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, n, 0, 64, s));
    uk = kb.Alternate();
    uv = vb.Alternate();
    ADJ_TRY(cub::DeviceReduce::ReduceByKey(tmp, tmp2, kb.Current(), uk, vb.Current(), uv, n_unique_d, cub::Sum(), n,
                                           s));
    ADJ_TRY(cudaMemcpyAsync(&n_unique, n_unique_d, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ADJ_TRY(cudaStreamSynchronize(s));
    // rows (the run of invalid keys, if any, sorts last and is excluded)
    k_adj_offsets<<<nblk(n_targets + 1, 256), 256, 0, s>>>(uk, n_unique, n_targets, offsets);
    ADJ_TRY(cudaGetLastError());
    k_adj_slice_width<<<nblk(n_slices, 256), 256, 0, s>>>(offsets, n_targets, n_slices, widths);
    ADJ_TRY(cudaGetLastError());
    ADJ_TRY(cudaMemsetAsync(widths + n_slices, 0, sizeof(int64_t), s));
    {
        size_t tmp3 = 0;
        ADJ_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp3, widths, slice_start, n_slices + 1, s));
        if (tmp3 > std::max(tmp_bytes, tmp2))
        {
            cudaFreeAsync(tmp, s);
            tmp = nullptr;
            ADJ_TRY(cudaMallocAsync(&tmp, tmp3, s));
        }
        ADJ_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp3, widths, slice_start, n_slices + 1, s));
    }
    ADJ_TRY(cudaMemcpyAsync(&total, slice_start + n_slices, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ADJ_TRY(cudaStreamSynchronize(s));
    *n_entries_out = total;
    ADJ_TRY(cudaMalloc(srcq_out, (size_t)std::max<int64_t>(total, 1) * sizeof(unsigned)));
    ADJ_TRY(cudaMalloc(coef_out, (size_t)std::max<int64_t>(total, 1) * sizeof(float)));
    k_adj_slice_fill<<<nblk(n_targets, 256), 256, 0, s>>>(offsets, uk, uv, slice_start, n_targets, *srcq_out,
                                                          *coef_out);
    ADJ_TRY(cudaGetLastError());
    ADJ_TRY(cudaStreamSynchronize(s));
done:
#undef ADJ_TRY
    cudaFreeAsync(k0, s);
    cudaFreeAsync(k1, s);
    cudaFreeAsync(v0, s);
    cudaFreeAsync(v1, s);
    cudaFreeAsync(offsets, s);
    cudaFreeAsync(n_unique_d, s);
    cudaFreeAsync(widths, s);
    if (tmp)
        cudaFreeAsync(tmp, s);
    cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
        cudaFree(*srcq_out);
        cudaFree(*coef_out);
        *srcq_out = nullptr;
        *coef_out = nullptr;
    }
    return e;
}

int64_t adj_slices(int64_t n_targets) { return (n_targets + kSlice - 1) / kSlice; }

void launch_adj_seed(const GridDev &g, int nd, const double *w, const uint8_t *flags, const double *dLdE, float *lam,
                     cudaStream_t s)
{
    k_adj_seed<<<nblk((int64_t)nd * g.nxy, 256), 256, 0, s>>>(g, nd, w, flags, dLdE, lam);
}
void launch_adj_collide(const AdjCollideArgs &a, cudaStream_t s)
{
    k_adj_collide<<<nblk(a.g.ncell, 128), 128, 0, s>>>(a);
}
void launch_adj_stream(const int64_t *slice_start, const unsigned *srcq, const float *coef, const uint8_t *clamp,
                       const float *lamS, int64_t n_targets, float *lam, cudaStream_t s)
{
    k_adj_stream<<<nblk(n_targets, 256), 256, 0, s>>>(slice_start, srcq, coef, clamp, lamS, n_targets, lam);
}
} // namespace grlbm
