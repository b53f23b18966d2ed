// Plain FP64 form of the radiation step, and the FP64 utility kernels.
//
// Built with -fmad=false: every multiply and add rounds on its own, and every
// expression below follows the association order of the reference's C++
// (src/Radiation.cpp), so that -- given the same geodesic tables -- the state
// after each step is bit-identical to the reference's IEEE build.  That is
// what the 1e-12 parity needs: the lambda iteration stops on the relative
// change of all six moments, including ones that are pure rounding noise
// (e.g. Fy of a nearly isotropic cell), so its iteration counts, and through
// them E, follow the last bits of the streamed intensities.
#include <type_traits>

#include "approx_math.hpp"
#include "device_common.cuh"

namespace grlbm
{
namespace
{
// one stream value: StreamFlatFixed (src/Radiation.cpp:394-410) or
// StreamCurvedFixed with IntensityAt (:478-508, 322-343)
// `clamp_mask` receives bit q set where corner q's angular interpolation was
// positive (kept by the clamp at zero); flat streaming keeps every corner.
// Off: the type of the state's element offsets (unsigned when the state has
// fewer than 2^32 elements, int64_t otherwise).
template <bool CURVED, typename Off>
__device__ __forceinline__ double stream_value(const PlainStepArgs &a, int d, const double4 &r, int64_t i, int64_t j,
                                               int64_t ij, unsigned &clamp_mask)
{
    clamp_mask = 0xFu;
    const int64_t nxy = a.g.nxy;
    const int nx = (int)a.g.nx; // node indices fit in 32 bits (nx * ny < 2^31)
    if constexpr (CURVED)
    {
        if (r.z < 0.0) // departure point inside the excision
            return 0.0;
        const double it = r.x, jt = r.y;
        // corners kept on the grid whatever the record holds
        const int i0 = min(max((int)floor(it), 0), nx - 2); // the conversion saturates: same clamp
        const int j0 = min(max((int)floor(jt), 0), (int)a.g.ny - 2);
        // g0 = floor(z) % nGrid, taken without the division when in range
        const int gz = (int)floor(r.z);
        int g0 = (unsigned)gz < (unsigned)a.ng ? gz : gz % a.ng;
        g0 = g0 < 0 ? 0 : g0;
        const int g1 = g0 + 1 == a.ng ? 0 : g0 + 1; // (g0 + 1) % nGrid
        const double t = r.z - (double)g0;
        const IgRow R0 = a.ig_rows[g0], R1 = a.ig_rows[g1];
        const int idx0[4] = {R0.idx.x, R0.idx.y, R0.idx.z, R0.idx.w};
        const int idx1[4] = {R1.idx.x, R1.idx.y, R1.idx.z, R1.idx.w};
        const double w0[4] = {R0.w01.x, R0.w01.y, R0.w23.x, R0.w23.y};
        const double w1[4] = {R1.w01.x, R1.w01.y, R1.w23.x, R1.w23.y};
        const double al = __ldg(a.alpha + ij);
        // element offsets of the 8 rows' planes
        Off o0[4], o1[4];
#pragma unroll
        for (int k = 0; k < 4; k++)
        {
            o0[k] = (Off)idx0[k] * (Off)nxy;
            o1[k] = (Off)idx1[k] * (Off)nxy;
        }
        double Iq[4];
#pragma unroll
        for (int q = 0; q < 4; q++) // corners 00, 01, 10, 11
        {
            const int ci = i0 + (q >> 1), cj = j0 + (q & 1);
            const int n = ci + cj * nx;
            double v0 = 0.0, v1 = 0.0;
#pragma unroll
            for (int k = 0; k < 4; k++)
            {
                v0 += w0[k] * __ldg(a.Iin + (o0[k] + (Off)n));
                v1 += w1[k] * __ldg(a.Iin + (o1[k] + (Off)n));
            }
            double v = v0 * (1.0 - t) + v1 * t;
            if (!(0.0 < v))
                clamp_mask &= ~(1u << q);
            v = (0.0 < v) ? v : 0.0;
            const int di = ci - (int)i, dj = cj - (int)j;
            double cube;
            if (di >= -1 && di <= 1 && dj >= -1 && dj <= 1)
                cube = __ldg(a.acube + ij * 9 + 3 * (dj + 1) + (di + 1));
            else
            {
                const double rr = al / __ldg(a.alpha + n);
                cube = rr * (rr * rr);
            }
            Iq[q] = cube * v;
        }
        const double fx = it - (double)i0, fy = jt - (double)j0;
        const double f0 = Iq[0] * (1.0 - fx) + Iq[2] * fx;
        const double f1 = Iq[1] * (1.0 - fx) + Iq[3] * fx;
        return r.w * (f0 * (1.0 - fy) + f1 * fy);
    }
    else
    {
        double xt = a.g.startx + (double)i * a.g.dx;
        double yt = a.g.starty + (double)j * a.g.dy;
        xt -= __ldg(a.cx + d) * a.g.dt;
        yt -= __ldg(a.cy + d) * a.g.dt;
        const double it = (xt - a.g.startx) / a.g.dx, jt = (yt - a.g.starty) / a.g.dy;
        const int i0 = min(max((int)floor(it), 0), nx - 2);
        const int j0 = min(max((int)floor(jt), 0), (int)a.g.ny - 2);
        const double *plane = a.Iin + (int64_t)d * nxy;
        const int c00 = i0 + j0 * nx;
        const double fx = it - (double)i0, fy = jt - (double)j0;
        const double f0 = __ldg(plane + c00) * (1.0 - fx) + __ldg(plane + c00 + 1) * fx;
        const double f1 = __ldg(plane + c00 + nx) * (1.0 - fx) + __ldg(plane + c00 + nx + 1) * fx;
        return f0 * (1.0 - fy) + f1 * fy;
    }
}

struct Moments
{
    double E, Fx, Fy, Pxx, Pxy, Pyy;
    __device__ __forceinline__ void zero() { E = Fx = Fy = Pxx = Pxy = Pyy = 0.0; }
    // ComputeMomentsIF / Collide accumulation order (src/Radiation.cpp:259-266, 706-712)
    __device__ __forceinline__ void add(double w, double v, double n1, double n2)
    {
        const double c = w * v;
        E += c;
        Fx += c * n1;
        Fy += c * n2;
        Pxx += c * n1 * n1;
        Pxy += c * n1 * n2;
        Pyy += c * n2 * n2;
    }
};

// one collided intensity (src/Radiation.cpp:690-703).  Divisions by A, A*A
// and (lorentz + 1) are skipped only where they are exact no-ops (A == 1,
// un == 0), so the result is the reference's bit for bit.
__device__ __forceinline__ double collide_value(double I, double n1, double n2, double u1, double u2, double lor,
                                                double adt, double eta, double k0, double k3, double kak0,
                                                double fE, double fFx, double fFy)
{
    const double un = u1 * n1 + u2 * n2;
    const double A = lor * (1.0 - un);
    const double sc = (un == 0.0) ? lor : (1 - (lor * un) / (lor + 1)) * lor;
    double nF1 = n1 - sc * u1, nF2 = n2 - sc * u2;
    if (A != 1.0)
    {
        nF1 = nF1 / A;
        nF2 = nF2 / A;
    }
    const double nF = nF1 * fFx + nF2 * fFy;
    const double M = k0 * fE + k3 * nF;
    double src = adt * (eta + M);
    const double AA = A * A;
    if (AA != 1.0)
        src = src / AA;
    return (I + src) / (1.0 + adt * kak0 * A);
}

// num / den, correctly rounded, from r = RN(1/den): one refinement brings
// RN(num r) (within 1.5 ulp of the quotient) to within one ulp, then one
// Markstein step (P. Markstein, IBM J. Res. Dev. 34(1), 1990: with r within
// half an ulp of 1/den and q within one ulp of num/den, the remainder
// num - den q is exact in one fma and RN(q + rem r) is the correctly rounded
// quotient) gives the IEEE result.  Used where den is the same for many
// divisions; outside the range in which no step can underflow or overflow
// the ordinary division is taken.  Requires 1 <= den < 2^100.
__device__ __forceinline__ double div_rn(double num, double den, double r)
{
    const double an = fabs(num);
    if (an != 0.0 && !(an > 0x1p-900 && an < 0x1p+900))
        return num / den;
    double q = __dmul_rn(num, r);
    q = __fma_rn(__fma_rn(-q, den, num), r, q);
    return __fma_rn(__fma_rn(-q, den, num), r, q);
}

// Fourier::GetValue (src/FourierHarmonics.cpp:56-61) with Fourier::Basis
// (:5-14) at a run-time angle, for the five series of a node's geodesic
// tables (S, X, Y, Cx, Cy) at once: coefficient k of series q at
// coef[q * fs + k * sk].  Each basis value is computed once and used by all
// five, and every sum keeps its order over k.
__device__ __forceinline__ void fourier_values5(const double *coef, int64_t fs, int64_t sk, int nf, double phi,
                                                double out[5])
{
    const double sqrt2 = 1.4142135623730951; // sqrt(2), correctly rounded
    double r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0;
    // the argument of term 2m - 1, phi * (2m - 1 + 1.0) / 2.0, and of term 2m,
    // phi * 2m / 2.0, round alike: one sincos serves both
    double sin_m = 0.0, cos_m = 1.0;
    for (int k = 0; k < nf; k++)
    {
        double b;
        if (k == 0)
            b = 1.0;
        else if (k % 2 != 0)
        {
            sincos(phi * (k + 1.0) / 2.0, &sin_m, &cos_m);
            b = sqrt2 * cos_m;
        }
        else
            b = sqrt2 * sin_m;
        const double *c = coef + k * sk;
        r0 += c[0] * b;
        r1 += c[fs] * b;
        r2 += c[2 * fs] * b;
        r3 += c[3 * fs] * b;
        r4 += c[4 * fs] * b;
    }
    out[0] = r0, out[1] = r1, out[2] = r2, out[3] = r3, out[4] = r4;
}

// IntensityAt (src/Radiation.cpp:322-343) of node n for the (unrotated)
// direction (v1, v2): rotated into the node's stencil frame by the inverse of
// its previous rotation angle, then the two cubic rows of the interpolation
// grid, blended and clamped at zero.
__device__ __forceinline__ double intensity_at(const PlainStepArgs &a, int64_t n, double v1, double v2)
{
    const double2 rinv = a.rot_inv[n]; // RotationMatrix(angle).Inverse()
    const double sn = rinv.x, cs = rinv.y;
    const double w1 = v1 * cs - v2 * sn, w2 = v1 * sn + v2 * cs;
    double dd = (double)a.ng * approx_phi(w1, w2) / (2.0 * kPi); // InterpolationGrid::d
    dd = dd < 1e-8 ? 1e-8 : ((double)a.ng - 1e-8 < dd ? (double)a.ng - 1e-8 : dd);
    // g0 = floor(dd) % nGrid, g1 = (g0 + 1) % nGrid, without the divisions
    // on the in-range path (the clamp keeps floor(dd) in [0, nGrid))
    const int gz = (int)floor(dd);
    int g0 = (unsigned)gz < (unsigned)a.ng ? gz : gz % a.ng;
    g0 = g0 < 0 ? 0 : g0;
    const int g1 = g0 + 1 == a.ng ? 0 : g0 + 1;
    const IgRow R0 = a.ig_rows[g0], R1 = a.ig_rows[g1];
    const int idx0[4] = {R0.idx.x, R0.idx.y, R0.idx.z, R0.idx.w};
    const int idx1[4] = {R1.idx.x, R1.idx.y, R1.idx.z, R1.idx.w};
    const double w0[4] = {R0.w01.x, R0.w01.y, R0.w23.x, R0.w23.y};
    const double wr1[4] = {R1.w01.x, R1.w01.y, R1.w23.x, R1.w23.y};
    double value0 = 0, value1 = 0;
#pragma unroll
    for (int k = 0; k < 4; k++)
    {
        value0 += w0[k] * __ldg(a.Iin + (int64_t)idx0[k] * a.g.nxy + n);
        value1 += wr1[k] * __ldg(a.Iin + (int64_t)idx1[k] * a.g.nxy + n);
    }
    const double t = dd - (double)g0;
    const double v = value0 * (1.0 - t) + value1 * t;
    return (0.0 < v) ? v : 0.0;
}

// One stream value of adaptive streaming: StreamFlatAdaptive
// (src/Radiation.cpp:415-452) or StreamCurvedAdaptive (:513-575), for the
// cell's direction d rotated by the cell's new angle (sine sc, cosine cc).
// Curved streaming reads coefficient k of series q of the cell at
// cf[q * qs + k * ks].
template <bool CURVED>
__device__ __forceinline__ double stream_value_adaptive(const PlainStepArgs &a, int d, int64_t i, int64_t j,
                                                        int64_t ij, double sc, double cc, const double *cf,
                                                        int qs, int ks)
{
    const int64_t nx = a.g.nx;
    const double cx = __ldg(a.cx + d), cy = __ldg(a.cy + d);
    const double dir1 = cx * cc - cy * sc, dir2 = cx * sc + cy * cc;
    double it, jt, v1, v2, s3 = 1.0;
    if constexpr (CURVED)
    {
        const double phi = approx_phi(dir1, dir2);
        double fv[5];
        fourier_values5(cf, qs, ks, a.nf, phi, fv);
        const double sh = fv[0], xt = fv[1], yt = fv[2];
        v1 = fv[3];
        v2 = fv[4];
        if (dev_inside_bh(a.g, xt, yt))
            return 0.0;
        it = (xt - a.g.startx) / a.g.dx;
        jt = (yt - a.g.starty) / a.g.dy;
        s3 = sh * (sh * sh);
    }
    else
    {
        double xt = a.g.startx + (double)i * a.g.dx, yt = a.g.starty + (double)j * a.g.dy;
        xt -= dir1 * a.g.dt;
        yt -= dir2 * a.g.dt;
        it = (xt - a.g.startx) / a.g.dx;
        jt = (yt - a.g.starty) / a.g.dy;
        v1 = dir1;
        v2 = dir2;
    }
    // corners kept on the grid whatever the departure
    const int64_t i0 = min(max((int64_t)floor(it), (int64_t)0), nx - 2);
    const int64_t j0 = min(max((int64_t)floor(jt), (int64_t)0), a.g.ny - 2);
    const double al = CURVED ? __ldg(a.alpha + ij) : 1.0;
    double Iq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) // corners 00, 01, 10, 11
    {
        const int64_t n = (i0 + (q >> 1)) + (j0 + (q & 1)) * nx;
        double v = intensity_at(a, n, v1, v2);
        if (CURVED)
        {
            const double rr = al / __ldg(a.alpha + n);
            v = rr * (rr * rr) * v;
        }
        Iq[q] = v;
    }
    const double fx = it - (double)i0, fy = jt - (double)j0;
    const double f0 = Iq[0] * (1.0 - fx) + Iq[2] * fx;
    const double f1 = Iq[1] * (1.0 - fx) + Iq[3] * fx;
    const double bil = f0 * (1.0 - fy) + f1 * fy;
    return CURVED ? s3 * bil : bil;
}

// Template switches of the step's kernels.  RECORD: also write what the
// adjoint needs about this step -- per (d, c) the corner clamp mask, per cell
// the lambda-iteration count and the first iterate's E -- without changing
// any result.  ADAPTIVE: the adaptive streaming types -- each cell's stencil
// is rotated by its new angle (its directions in stream, moments and
// collide) and corners are read in their previous frames.
//
// Direction d of a cell's stencil (tn1, tn2: the stencil's directions;
// rotated by the cell's angle in adaptive streaming).
#define GRLBM_N1(d) (ADAPTIVE ? tn1[d] * rot_c - tn2[d] * rot_s : tn1[d])
#define GRLBM_N2(d) (ADAPTIVE ? tn1[d] * rot_s + tn2[d] * rot_c : tn2[d])

// The rest of a step for one cell once its streamed values are known: m
// holds their moments; Sin points at them (direction stride sst), Sout at the
// cell's output slots (the same slots in the fused step).  Collide
// (src/Radiation.cpp:641-736) for a colliding cell, then the stored moments
// and the lambda-iteration statistics.
// tw, tn1, tn2: the stencil's weights and directions (global or shared memory).
// rot_s, rot_c: the cell's rotation (adaptive streaming).
// Unroll of the lambda iteration's direction loops for a fluid at rest (the
// directions' updates are independent; only the moment sums chain them).
#ifndef GRLBM_ITER_UNROLL
#define GRLBM_ITER_UNROLL 4
#endif
constexpr int kIterUnroll = GRLBM_ITER_UNROLL;
template <bool RECORD, bool ADAPTIVE>
__device__ __forceinline__ void finish_cell(const PlainStepArgs &a, const StepRecord &rec, bool active, bool collides,
                                            int64_t ij, int64_t cc, Moments m, const double *Sin, int64_t sst,
                                            double *Sout,
                                            double rot_s, double rot_c, const double *tw, const double *tn1,
                                            const double *tn2)
{
    const int t = threadIdx.x;
    const int64_t nxy = a.g.nxy;
    int cycles = 0;
    if (RECORD && active)
        rec.e0[cc] = m.E;
    if (collides)
    {
        const double u1 = a.u1[ij], u2 = a.u2[ij], lor = a.lor[ij], adt = a.adt[ij];
        const double eta = a.eta[ij], k0 = a.k0[ij], k3 = a.k3[ij], kak0 = a.ka[ij] + a.k0[ij];
        // A fluid at rest has u = 0 and lorentz = 1, so in collide_value
        // A = 1, n_ff = n and AA = 1 exactly: the update reduces to
        // (I + adt (eta + (k0 fE + k3 (n1 fFx + n2 fFy)))) / (1 + adt kak0)
        // with the same roundings.
        const bool rest = u1 == 0.0 && u2 == 0.0 && lor == 1.0;
        const double den = 1.0 + adt * kak0;
        const bool fast_div = rest && den >= 1.0 && den < 0x1p+100;
        const double rden = __drcp_rn(den);
        double diff = 1;
        double fE = 0, fFx = 0, fFy = 0;
        while (fabs(diff) > 1e-4 && cycles < 100)
        {
            cycles++;
            const double pE = m.E, pFx = m.Fx, pFy = m.Fy, pPxx = m.Pxx, pPxy = m.Pxy, pPyy = m.Pyy;
            // fluid-frame moments of the previous iterate (src/Radiation.cpp:672-678)
            const double uF = u1 * pFx + u2 * pFy;
            const double uxP = u1 * pPxx + u2 * pPxy;
            const double uyP = u1 * pPxy + u2 * pPyy;
            const double uuP = u1 * uxP + u2 * uyP;
            fE = lor * lor * (pE - 2.0 * uF + uuP);
            fFx = lor * lor * (pFx - lor * pE * u1 - uxP + u1 * lor / (1.0 + lor) * ((2.0 * lor + 1.0) * uF - lor * uuP));
            fFy = lor * lor * (pFy - lor * pE * u2 - uyP + u2 * lor / (1.0 + lor) * ((2.0 * lor + 1.0) * uF - lor * uuP));
            m.zero();
            if (rest)
            {
                const double k0fE = k0 * fE;
#pragma unroll kIterUnroll
                for (int d = 0; d < a.nd; d++)
                {
                    const double n1 = GRLBM_N1(d), n2 = GRLBM_N2(d);
                    const double num = Sin[(int64_t)d * sst] + adt * (eta + (k0fE + k3 * (n1 * fFx + n2 * fFy)));
                    const double v = fast_div ? div_rn(num, den, rden) : num / den;
                    m.add(tw[d], v, n1, n2);
                }
            }
            else
                for (int d = 0; d < a.nd; d++)
                {
                    const double n1 = GRLBM_N1(d), n2 = GRLBM_N2(d);
                    const double v = collide_value(Sin[(int64_t)d * sst], n1, n2, u1, u2, lor, adt, eta, k0, k3,
                                                   kak0, fE, fFx, fFy);
                    m.add(tw[d], v, n1, n2);
                }
            const double e1 = (pE - m.E) / m.E, e2 = (pFx - m.Fx) / m.Fx, e3 = (pFy - m.Fy) / m.Fy;
            const double e4 = (pPxx - m.Pxx) / m.Pxx, e5 = (pPxy - m.Pxy) / m.Pxy, e6 = (pPyy - m.Pyy) / m.Pyy;
            diff = sqrt(e1 * e1 + e2 * e2 + e3 * e3 + e4 * e4 + e5 * e5 + e6 * e6);
        }
        // the last iterate, recomputed from the same operands, over the parked values
        if (rest)
        {
            const double k0fE = k0 * fE;
#pragma unroll kIterUnroll
            for (int d = 0; d < a.nd; d++)
            {
                const double n1 = GRLBM_N1(d), n2 = GRLBM_N2(d);
                const double num = Sin[(int64_t)d * sst] + adt * (eta + (k0fE + k3 * (n1 * fFx + n2 * fFy)));
                Sout[(int64_t)d * nxy] = fast_div ? div_rn(num, den, rden) : num / den;
            }
        }
        else
            for (int d = 0; d < a.nd; d++)
                Sout[(int64_t)d * nxy] = collide_value(Sin[(int64_t)d * sst], GRLBM_N1(d), GRLBM_N2(d), u1, u2,
                                                     lor, adt, eta, k0, k3, kak0, fE, fFx, fFy);
    }
    if (RECORD && active)
        rec.cycles[cc] = cycles;
    if (active)
    {
        a.mom[ij] = m.E;
        a.mom[ij + nxy] = m.Fx;
        a.mom[ij + 2 * nxy] = m.Fy;
        a.mom[ij + 3 * nxy] = m.Pxx;
        a.mom[ij + 4 * nxy] = m.Pxy;
        a.mom[ij + 5 * nxy] = m.Pyy;
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


// The fixed streaming types run the step as two kernels, so that the
// stream's dependent gathers (record, interpolation rows, 32 corner taps)
// of different directions run in different threads instead of one after the
// other in one thread per cell.  Stream: one thread per (cell, direction) of
// the slab rows writes the streamed value to S (and, recording, the corner
// clamp mask).
// Blocks are 32 x 4 tiles of cells (blockIdx.x, blockIdx.y over the slab
// rows) of one direction (blockIdx.z).
#ifndef GRLBM_COLLIDE_UNROLL
#define GRLBM_COLLIDE_UNROLL 8
#endif
constexpr int kCollideUnroll = GRLBM_COLLIDE_UNROLL;
// Grid order of the stream kernel: directions fastest for adaptive streaming
// (the blocks of one tile, which read the same Fourier coefficients, run
// together), tiles fastest for fixed streaming (measured: 2% faster and 3%
// slower respectively the other way round).
constexpr bool kDirFastestAdaptive = true, kDirFastestFixed = false;
#ifndef GRLBM_SPLIT_TILE_X
#define GRLBM_SPLIT_TILE_X 16
#endif
constexpr int kSplitTileX = GRLBM_SPLIT_TILE_X, kSplitTileY = kStepBlock / kSplitTileX;
// resident blocks per SM the stream kernel's registers are sized for (6:
// 80 registers, no spills in the curved gather with 32-bit offsets)
#ifndef GRLBM_STREAM_MIN_BLOCKS
#define GRLBM_STREAM_MIN_BLOCKS 6
#endif
template <bool CURVED, bool RECORD, bool ADAPTIVE, bool WIDE = false>
__global__ void __launch_bounds__(kStepBlock, GRLBM_STREAM_MIN_BLOCKS) k_stream_plain(PlainStepArgs a, StepRecord rec)
{
    static_assert(!(CURVED && ADAPTIVE), "curved adaptive streaming runs k_stream_plain_curved_adaptive");
    constexpr bool DFAST = ADAPTIVE ? kDirFastestAdaptive : kDirFastestFixed;
    const int d = DFAST ? blockIdx.x : blockIdx.z;
    const int bx = DFAST ? blockIdx.y : blockIdx.x, by = DFAST ? blockIdx.z : blockIdx.y;
    const int i = 1 + bx * kSplitTileX + (int)(threadIdx.x % kSplitTileX);
    const int j = (int)a.g.jlo + by * kSplitTileY + (int)(threadIdx.x / kSplitTileX);
    if (i > a.g.nx_ || j >= a.g.jhi)
        return;
    const int64_t cc = (int64_t)(i - 1) + (int64_t)(j - 1) * a.g.nx_;
    const int64_t ij = (int64_t)i + (int64_t)j * a.g.nx;
    unsigned cm = 0xFu;
    double val = 0.0;
    if (!(CURVED && (a.flags[ij] & 2)))
    {
        if constexpr (ADAPTIVE)
        {
            // the cell's rotation (RotationMatrix(rotationAngle[ij]), src/DataTypes.hh:630-635)
            const double2 rn = a.rot_new[ij];
            val = stream_value_adaptive<CURVED>(a, d, i, j, ij, rn.x, rn.y, nullptr, 0, 0);
        }
        else
        {
            const double4 r = CURVED ? a.rec[(int64_t)d * a.g.ncell + cc] : make_double4(0, 0, 0, 0);
            val = stream_value<CURVED, std::conditional_t<WIDE, int64_t, unsigned>>(a, d, r, i, j, ij, cm);
        }
    }
    if (RECORD)
        rec.clamp[(int64_t)d * a.g.ncell + cc] = (uint8_t)cm;
    a.S[(int64_t)d * a.g.nxy + ij] = val;
}

// Curved adaptive stream: a block takes 16 cells of one row for kPDirs
// directions (16: 7% faster than 8, and 32 slower, at 400^2 x 64).  It first
// stages the row's Fourier coefficients (5 nF x 16 doubles, at most 40 KB)
// in shared memory, where its directions share them; each warp then covers
// 16 cells x 2 directions.
constexpr int kPDirs = kAdaptiveBlock / kSplitTileX;
__global__ void __launch_bounds__(kAdaptiveBlock) k_stream_plain_curved_adaptive(PlainStepArgs a)
{
    extern __shared__ double sco[]; // [q * nF + k][cell]
    // blockIdx.x: direction group fastest, then the row; blockIdx.y: the run of 16 cells
    const int ndg = (a.nd + kPDirs - 1) / kPDirs;
    const int t = threadIdx.x, c = t % kSplitTileX;
    const int d = (int)(blockIdx.x % (unsigned)ndg) * kPDirs + t / kSplitTileX;
    const int x0 = 1 + (int)blockIdx.y * kSplitTileX, i = x0 + c;
    const int j = (int)a.g.jlo + (int)(blockIdx.x / (unsigned)ndg);
    const int nrow = min(kSplitTileX, (int)a.g.nx_ + 1 - x0);
    const int64_t row0 = (int64_t)x0 + (int64_t)j * a.g.nx;
    // coefficient k of series q of node ij sits at coef[(q nF + k) nxy + ij]
    for (int e = t; e < 5 * a.nf * kSplitTileX; e += kAdaptiveBlock)
    {
        const int p = e / kSplitTileX, cc = e % kSplitTileX;
        sco[e] = cc < nrow ? a.coef[(int64_t)p * a.g.nxy + row0 + cc] : 0.0;
    }
    __syncthreads();
    if (c >= nrow || d >= a.nd)
        return;
    const int64_t ij = row0 + c;
    double val = 0.0;
    if (!(a.flags[ij] & 2))
    {
        // the cell's rotation (RotationMatrix(rotationAngle[ij]), src/DataTypes.hh:630-635)
        const double2 rn = a.rot_new[ij];
        val = stream_value_adaptive<true>(a, d, i, j, ij, rn.x, rn.y, sco + c, a.nf * kSplitTileX, kSplitTileX);
    }
    a.S[(int64_t)d * a.g.nxy + ij] = val;
}

// Moments and collide: one thread per cell sums the moments of its streamed
// values in direction order (ComputeMomentsIF's order, as the fused step
// does) and finishes the cell; the collided intensities go to Iout.  With
// COLUMN (when the block's values fit in 48 KB of shared memory) each thread
// keeps its cell's streamed values in its own column of shared memory for
// the lambda iteration's passes, instead of re-reading them from L2.
constexpr int kColumnTileY = 4; // 16 x 4 cells per block with COLUMN
template <bool RECORD, bool ADAPTIVE, bool COLUMN>
__global__ void __launch_bounds__(kStepBlock) k_collide_plain(PlainStepArgs a, StepRecord rec)
{
    constexpr int TY = COLUMN ? kColumnTileY : kSplitTileY, NT = kSplitTileX * TY;
    const int t = threadIdx.x;
    const int ti = 1 + (int)blockIdx.x * kSplitTileX + t % kSplitTileX;
    const int tj = (int)a.g.jlo + (int)blockIdx.y * TY + t / kSplitTileX;
    const bool active = ti <= a.g.nx_ && tj < a.g.jhi;
    const int64_t i = active ? ti : 1, j = active ? tj : 1;
    const int64_t cc = (i - 1) + (j - 1) * a.g.nx_;
    const int64_t ij = i + j * a.g.nx;
    const int64_t nxy = a.g.nxy;
    const bool collides = active && !(a.flags[ij] & 1);
    // the stencil's weights and directions, read by every cell of the block
    extern __shared__ double dyn[];
    double *sw = dyn, *sn1 = dyn + a.nd, *sn2 = dyn + 2 * a.nd;
    const double *dn1 = ADAPTIVE ? a.cx : a.n1, *dn2 = ADAPTIVE ? a.cy : a.n2;
    for (int d = t; d < a.nd; d += NT)
        sw[d] = a.w[d], sn1[d] = dn1[d], sn2[d] = dn2[d];
    __syncthreads();
    const double *tw = sw, *tn1 = sn1, *tn2 = sn2;
    // the cell's rotation (adaptive streaming)
    double rot_s = 0.0, rot_c = 1.0;
    if (ADAPTIVE)
    {
        const double2 rn = a.rot_new[ij];
        rot_s = rn.x;
        rot_c = rn.y;
    }
    const double *S = a.S + ij;
    double *col = dyn + 3 * a.nd + t; // COLUMN: this cell's values, stride NT
    Moments m;
    m.zero();
    if (active)
    {
#pragma unroll kCollideUnroll
        for (int d = 0; d < a.nd; d++)
        {
            const double v = S[(int64_t)d * nxy];
            if (COLUMN)
                col[d * NT] = v;
            m.add(tw[d], v, GRLBM_N1(d), GRLBM_N2(d));
        }
    }
    finish_cell<RECORD, ADAPTIVE>(a, rec, active, collides, ij, cc, m, COLUMN ? col : S, COLUMN ? NT : nxy,
                                  a.Iout + ij, rot_s, rot_c, tw, tn1, tn2);
}
#undef GRLBM_N1
#undef GRLBM_N2

// UpdateRotationMatrizes (src/Radiation.cpp:361-378): for the interior cells
// of the slab, the angle of the flux averaged over the 3x3 neighbourhood
// where at least 1% of the light moves along it, else the previous angle.
template <typename T>
__global__ void k_rotation_update(GridDev g, const T *mom, const double *ang_old, double *ang_new)
{
    const int64_t c0 = (g.jlo - 1) * g.nx_;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (g.jhi - g.jlo) * g.nx_)
        return;
    const int64_t cc = c0 + c;
    const int64_t i = 1 + cc % g.nx_, j = 1 + cc / g.nx_;
    const int64_t ij = i + j * g.nx, nxy = g.nxy;
    double fx = 0.0, fy = 0.0;
    for (int b = -1; b <= 1; b++)
        for (int a = -1; a <= 1; a++)
        {
            const int64_t n = (i + a) + (j + b) * g.nx;
            fx += (double)mom[n + nxy];
            fy += (double)mom[n + 2 * nxy];
        }
    fx /= 9.0;
    fy /= 9.0;
    const double norm = sqrt(fx * fx + fy * fy);
    const double E = (double)mom[ij];
    ang_new[ij] = (E > 1e-16 && norm / E > 0.01) ? approx_phi(fx, fy) : ang_old[ij];
}

// The rotations an adaptive step reads at every node: the inverse of the
// previous one (RotationMatrix(angle).Inverse(), src/DataTypes.hh:625-635,
// as IntensityAt uses it at each corner) and the new one (the cell's own
// stencil), as {sin, cos}.
// V2: double2, or float2 for the precision form (the FP64 values rounded).
template <typename V2>
__global__ void k_rotation_trig(int64_t nxy, const double *ang_old, const double *ang_new, V2 *rot_inv, V2 *rot_new)
{
    using T = decltype(V2::x);
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nxy)
        return;
    const double th = fmod(-ang_old[n] + 2.0 * kPi, 2.0 * kPi);
    rot_inv[n] = V2{(T)approx_sin(th), (T)approx_cos(th)};
    const double tn = ang_new[n];
    rot_new[n] = V2{(T)approx_sin(tn), (T)approx_cos(tn)};
}

// The moments at the halo nodes, which the reference recomputes after every
// stream from intensities it never writes there (zero).
template <typename T>
__global__ void k_zero_halo_moments(GridDev g, T *mom)
{
    const int64_t ij = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= g.nxy)
        return;
    const int64_t i = ij % g.nx, j = ij / g.nx;
    if (i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1)
        for (int q = 0; q < 6; q++)
            mom[ij + q * g.nxy] = (T)0;
}

// Radiation::ComputeMomentsIF (src/Radiation.cpp:239-269): the six moments
// of the current intensities at every node, halo included, in the
// reference's order.  The precision form's state is converted back to I
// (J / (1 / alpha^3)) first.
// With `ang` (adaptive streaming) the directions are the stencil's rotated
// by each node's angle, n1/n2 then holding the unrotated directions.
template <typename T, typename SC>
__global__ void k_moments_from_I(const T *I, int64_t nxy, StateLayout L, int nd, const double *w,
                                 const double *n1, const double *n2, const SC *scale, const double *ang,
                                 double *mom)
{
    const int64_t ij = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= nxy)
        return;
    double rs = 0.0, rc = 1.0;
    if (ang)
    {
        rs = approx_sin(ang[ij]);
        rc = approx_cos(ang[ij]);
    }
    Moments m;
    m.zero();
    const int64_t sij = L.at(ij);
    for (int d = 0; d < nd; d++)
    {
        const double wd = __ldg(w + d);
        if (wd == 0.0)
            continue;
        double v = (double)I[sij * L.sp + (int64_t)d * L.plane];
        if (scale)
            v = v / (double)scale[ij];
        const double c1 = __ldg(n1 + d), c2 = __ldg(n2 + d);
        if (ang)
            m.add(wd, v, c1 * rc - c2 * rs, c1 * rs + c2 * rc);
        else
            m.add(wd, v, c1, c2);
    }
    mom[ij] = m.E;
    mom[ij + nxy] = m.Fx;
    mom[ij + 2 * nxy] = m.Fy;
    mom[ij + 3 * nxy] = m.Pxx;
    mom[ij + 4 * nxy] = m.Pxy;
    mom[ij + 5 * nxy] = m.Pyy;
}

// Radiation::LoadInitialData for fixed streaming (src/Radiation.cpp:138-181)
template <typename T>
__global__ void k_sources(T *I, StateLayout L, int nd, const int64_t *nodes, const T *vals, int64_t nsrc)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nsrc * nd)
        return;
    const int64_t s = tid / nd;
    const int d = (int)(tid - s * nd);
    I[L.elem(nodes[s], d)] = vals[tid];
    if (d < L.mirror) // the cell-major state repeats the first directions after the last
        I[L.elem(nodes[s], nd + d)] = vals[tid];
}

// Radiation::ComputeMomentsLF (src/Radiation.cpp:270-301)
template <typename T>
__global__ void k_moments_lf(int64_t nxy, const T *mom, const double *lfp, const uint8_t *bh, double *out)
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
        // Norm2 (src/SpecialMath.cpp:20-27): sum_i sum_j gamma_ij v_i v_j
        double n2 = 0.0;
        n2 += g11 * o[1] * o[1];
        n2 += g12 * o[1] * o[2];
        n2 += g12 * o[2] * o[1];
        n2 += g22 * o[2] * o[2];
        o[6] = sqrt(fabs(n2));
    }
#pragma unroll
    for (int q = 0; q < 7; q++)
        out[ij + q * nxy] = o[q];
}

// global energy: fixed-order partial sums of interior E, then one block
template <typename T>
__global__ void __launch_bounds__(256) k_energy_partial(GridDev g, const T *E, double *partial)
{
    __shared__ double s[256];
    const int t = threadIdx.x;
    double acc = 0.0;
    const int64_t c0 = (g.jlo - 1) * g.nx_, c1 = (g.jhi - 1) * g.nx_; // the slab's cells
    for (int64_t c = c0 + (int64_t)blockIdx.x * 256 + t; c < c1; c += (int64_t)gridDim.x * 256)
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

// Fourier coefficients [5][nxy][nf] -> [5][nf][nxy]
__global__ void k_coef_k_major(const double *coef, double *coef_k, int64_t nxy, int nf)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per = nxy * nf;
    if (t >= 5 * per)
        return;
    const int64_t q = t / per, r = t - q * per; // r = k * nxy + ij
    const int64_t k = r / nxy, ij = r - k * nxy;
    coef_k[t] = coef[q * per + ij * nf + k];
}

// the boundary's cell-major double [ij][d] <-> a state buffer of layout L
template <class T, class SC>
__global__ void k_to_dirmajor(const double *in, T *out, int64_t nxy, StateLayout L, int nd, const SC *scale)
{
    __shared__ double tile[32][33];
    const int64_t ij0 = (int64_t)blockIdx.x * 32;
    const int d0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int64_t ij = ij0 + r;
        const int d = d0 + threadIdx.x;
        if (ij < nxy && d < nd)
            tile[r][threadIdx.x] = in[ij * nd + d];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int d = d0 + r;
        const int64_t ij = ij0 + threadIdx.x;
        if (ij < nxy && d < nd)
        {
            const T v = scale ? (T)tile[threadIdx.x][r] * (T)scale[ij] : (T)tile[threadIdx.x][r];
            out[L.elem(ij, d)] = v;
            if (d < L.mirror) // the cell-major state repeats the first directions after the last
                out[L.elem(ij, nd + d)] = v;
        }
    }
}
template <class T, class SC>
__global__ void k_to_cellmajor(const T *in, double *out, int64_t nxy, StateLayout L, int nd, const SC *scale)
{
    __shared__ double tile[32][33];
    const int64_t ij0 = (int64_t)blockIdx.x * 32;
    const int d0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int d = d0 + r;
        const int64_t ij = ij0 + threadIdx.x;
        if (ij < nxy && d < nd)
            tile[threadIdx.x][r] = scale ? (double)in[L.elem(ij, d)] / (double)scale[ij] : (double)in[L.elem(ij, d)];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8)
    {
        const int64_t ij = ij0 + r;
        const int d = d0 + threadIdx.x;
        if (ij < nxy && d < nd)
            out[ij * nd + d] = tile[r][threadIdx.x];
    }
}
__global__ void k_widen(const float *in, double *out, int64_t n)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        out[k] = (double)in[k];
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }
} // namespace

cudaError_t prepare_step_plain(int smem_bytes)
{
    (void)smem_bytes; // the plain step uses no dynamic shared memory
    return cudaSuccess;
}
void launch_step_plain(const PlainStepArgs &a, bool curved, cudaStream_t s, const StepRecord *record)
{
    const int64_t cells = (a.g.jhi - a.g.jlo) * a.g.nx_;
    if (cells <= 0)
        return;
    const bool adaptive = a.ang_new != nullptr;
    const StepRecord none{};
    const StepRecord &rec = record && !adaptive ? *record : none;
    const unsigned tx = nblk(a.g.nx_, kSplitTileX), ty = nblk(a.g.jhi - a.g.jlo, kSplitTileY);
    const dim3 sgrid(tx, ty, (unsigned)a.nd), sgrid_df((unsigned)a.nd, tx, ty), cgrid(tx, ty);
    if (adaptive) // UpdateRotationMatrizes from the previous moments, before the stream
    {
        k_rotation_update<double><<<nblk(cells, 128), 128, 0, s>>>(a.g, a.mom, a.ang_old, const_cast<double *>(a.ang_new));
        launch_rotation_trig(a.g.nxy, a.ang_old, a.ang_new, const_cast<double2 *>(a.rot_inv),
                             const_cast<double2 *>(a.rot_new), s);
    }
    // stream
    const dim3 ga = kDirFastestAdaptive ? sgrid_df : sgrid, gf = kDirFastestFixed ? sgrid_df : sgrid;
    if (adaptive && curved)
        k_stream_plain_curved_adaptive<<<dim3(nblk(a.nd, kPDirs) * (unsigned)(a.g.jhi - a.g.jlo), tx), kAdaptiveBlock,
                                         (size_t)5 * a.nf * kSplitTileX * sizeof(double), s>>>(a);
    else if (adaptive)
        k_stream_plain<false, false, true><<<ga, kStepBlock, 0, s>>>(a, rec);
    else if (curved && a.wide) // 64-bit state offsets
        record ? k_stream_plain<true, true, false, true><<<gf, kStepBlock, 0, s>>>(a, rec)
               : k_stream_plain<true, false, false, true><<<gf, kStepBlock, 0, s>>>(a, rec);
    else if (curved)
        record ? k_stream_plain<true, true, false><<<gf, kStepBlock, 0, s>>>(a, rec)
               : k_stream_plain<true, false, false><<<gf, kStepBlock, 0, s>>>(a, rec);
    else
        record ? k_stream_plain<false, true, false><<<gf, kStepBlock, 0, s>>>(a, rec)
               : k_stream_plain<false, false, false><<<gf, kStepBlock, 0, s>>>(a, rec);
    // moments and collide: with each cell's values in shared memory when they fit
    const size_t tables = 3 * (size_t)a.nd * sizeof(double);
    const size_t column = tables + (size_t)a.nd * kSplitTileX * kColumnTileY * sizeof(double);
    if (column <= 48 * 1024)
    {
        const dim3 kgrid(tx, nblk(a.g.jhi - a.g.jlo, kColumnTileY));
        const unsigned nt = kSplitTileX * kColumnTileY;
        if (adaptive)
            k_collide_plain<false, true, true><<<kgrid, nt, column, s>>>(a, rec);
        else if (record)
            k_collide_plain<true, false, true><<<kgrid, nt, column, s>>>(a, rec);
        else
            k_collide_plain<false, false, true><<<kgrid, nt, column, s>>>(a, rec);
    }
    else if (adaptive)
        k_collide_plain<false, true, false><<<cgrid, kStepBlock, tables, s>>>(a, rec);
    else if (record)
        k_collide_plain<true, false, false><<<cgrid, kStepBlock, tables, s>>>(a, rec);
    else
        k_collide_plain<false, false, false><<<cgrid, kStepBlock, tables, s>>>(a, rec);
    if (adaptive) // the halo moments, recomputed by the reference from unwritten (zero) intensities
        k_zero_halo_moments<double><<<nblk(a.g.nxy, 256), 256, 0, s>>>(a.g, a.mom);
}
void launch_sources64(double *I, int64_t nxy, int nd, const int64_t *nodes, const double *vals, int64_t nsrc,
                      cudaStream_t s)
{
    k_sources<double><<<nblk(nsrc * nd, 256), 256, 0, s>>>(I, StateLayout{nxy, nxy, nxy}, nd, nodes, vals, nsrc);
}
void launch_sources32(float *I, const StateLayout &L, int nd, const int64_t *nodes, const float *vals, int64_t nsrc,
                      cudaStream_t s)
{
    k_sources<float><<<nblk(nsrc * nd, 256), 256, 0, s>>>(I, L, nd, nodes, vals, nsrc);
}
void launch_coef_k_major(const double *coef, double *coef_k, int64_t nxy, int nf, cudaStream_t s)
{
    k_coef_k_major<<<nblk(5 * nxy * nf, 256), 256, 0, s>>>(coef, coef_k, nxy, nf);
}
void launch_rotation_trig(int64_t nxy, const double *ang_old, const double *ang_new, double2 *rot_inv,
                          double2 *rot_new, cudaStream_t s)
{
    k_rotation_trig<<<nblk(nxy, 256), 256, 0, s>>>(nxy, ang_old, ang_new, rot_inv, rot_new);
}
void launch_rotation_trig32(int64_t nxy, const double *ang_old, const double *ang_new, float2 *rot_inv,
                            float2 *rot_new, cudaStream_t s)
{
    k_rotation_trig<<<nblk(nxy, 256), 256, 0, s>>>(nxy, ang_old, ang_new, rot_inv, rot_new);
}
// UpdateRotationMatrizes before, and the halo moments after, an adaptive
// precision-form step (FP32 moments)
void launch_rotation_update32(const GridDev &g, const float *mom, const double *ang_old, double *ang_new,
                              cudaStream_t s)
{
    const int64_t cells = (g.jhi - g.jlo) * g.nx_;
    if (cells > 0)
        k_rotation_update<float><<<nblk(cells, 128), 128, 0, s>>>(g, mom, ang_old, ang_new);
}
void launch_zero_halo_moments32(const GridDev &g, float *mom, cudaStream_t s)
{
    k_zero_halo_moments<float><<<nblk(g.nxy, 256), 256, 0, s>>>(g, mom);
}
void launch_moments_lf64(int64_t nxy, const double *mom, const double *lfp, const uint8_t *bh, double *out,
                         cudaStream_t s)
{
    k_moments_lf<double><<<nblk(nxy, 256), 256, 0, s>>>(nxy, mom, lfp, bh, out);
}
void launch_moments_lf32(int64_t nxy, const float *mom, const double *lfp, const uint8_t *bh, double *out,
                         cudaStream_t s)
{
    k_moments_lf<float><<<nblk(nxy, 256), 256, 0, s>>>(nxy, mom, lfp, bh, out);
}
void launch_energy64(const GridDev &g, const double *E, double *partial, int nblocks, double *out, cudaStream_t s)
{
    k_energy_partial<double><<<nblocks, 256, 0, s>>>(g, E, partial);
    k_energy_final<<<1, 256, 0, s>>>(partial, nblocks, out);
}
void launch_energy32(const GridDev &g, const float *E, double *partial, int nblocks, double *out, cudaStream_t s)
{
    k_energy_partial<float><<<nblocks, 256, 0, s>>>(g, E, partial);
    k_energy_final<<<1, 256, 0, s>>>(partial, nblocks, out);
}
void launch_to_dirmajor64(const double *in, double *out, int64_t nxy, int nd, cudaStream_t s)
{
    k_to_dirmajor<double, double><<<dim3(nblk(nxy, 32), nblk(nd, 32)), dim3(32, 8), 0, s>>>(
        in, out, nxy, StateLayout{nxy, nxy, nxy}, nd, nullptr);
}
void launch_to_dirmajor32(const double *in, float *out, int64_t nxy, const StateLayout &L, int nd,
                          const float *scale, cudaStream_t s)
{
    k_to_dirmajor<float, float><<<dim3(nblk(nxy, 32), nblk(nd, 32)), dim3(32, 8), 0, s>>>(in, out, nxy, L, nd, scale);
}
void launch_to_cellmajor64(const double *in, double *out, int64_t nxy, int nd, cudaStream_t s)
{
    k_to_cellmajor<double, double><<<dim3(nblk(nxy, 32), nblk(nd, 32)), dim3(32, 8), 0, s>>>(
        in, out, nxy, StateLayout{nxy, nxy, nxy}, nd, nullptr);
}
void launch_to_cellmajor32(const float *in, double *out, int64_t nxy, const StateLayout &L, int nd,
                           const float *scale, cudaStream_t s)
{
    k_to_cellmajor<float, float><<<dim3(nblk(nxy, 32), nblk(nd, 32)), dim3(32, 8), 0, s>>>(in, out, nxy, L, nd, scale);
}
void launch_moments_from_I64(const double *I, int64_t nxy, int nd, const double *w, const double *n1,
                             const double *n2, const double *ang, double *mom, cudaStream_t s)
{
    k_moments_from_I<double, double><<<nblk(nxy, 128), 128, 0, s>>>(I, nxy, StateLayout{nxy, nxy, nxy}, nd, w, n1, n2,
                                                                     nullptr, ang, mom);
}
void launch_moments_from_I32(const float *J, int64_t nxy, const StateLayout &L, int nd, const double *w,
                             const double *n1, const double *n2, const float *scale, const double *ang, double *mom,
                             cudaStream_t s)
{
    k_moments_from_I<float, float><<<nblk(nxy, 128), 128, 0, s>>>(J, nxy, L, nd, w, n1, n2, scale, ang, mom);
}
void launch_widen32(const float *in, double *out, int64_t n, cudaStream_t s)
{
    k_widen<<<nblk(n, 256), 256, 0, s>>>(in, out, n);
}
void launch_sources64L(double *I, const StateLayout &L, int nd, const int64_t *nodes, const double *vals,
                       int64_t nsrc, cudaStream_t s)
{
    k_sources<double><<<nblk(nsrc * nd, 256), 256, 0, s>>>(I, L, nd, nodes, vals, nsrc);
}
void launch_to_state64(const double *in, double *out, int64_t nxy, const StateLayout &L, int nd, const double *scale,
                       cudaStream_t s)
{
    k_to_dirmajor<double, double><<<dim3(nblk(nxy, 32), nblk(nd, 32)), dim3(32, 8), 0, s>>>(in, out, nxy, L, nd, scale);
}
void launch_from_state64(const double *in, double *out, int64_t nxy, const StateLayout &L, int nd, const double *scale,
                         cudaStream_t s)
{
    k_to_cellmajor<double, double><<<dim3(nblk(nxy, 32), nblk(nd, 32)), dim3(32, 8), 0, s>>>(in, out, nxy, L, nd, scale);
}
void launch_moments_from_state64(const double *J, int64_t nxy, const StateLayout &L, int nd, const double *w,
                                 const double *n1, const double *n2, const double *scale, double *mom, cudaStream_t s)
{
    k_moments_from_I<double, double><<<nblk(nxy, 128), 128, 0, s>>>(J, nxy, L, nd, w, n1, n2, scale, nullptr, mom);
}
} // namespace grlbm
