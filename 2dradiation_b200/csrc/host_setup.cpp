// Host set-up tables; see host_setup.hpp.  Compiled with
// -ffp-contract=off and without fast-math so that every product below rounds
// exactly once, in the reference's association order.
#include "host_setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "approx_math.hpp"

namespace grlbm
{
GridGeom GridGeom::from(const grlbm_grid_desc &d)
{
    // src/Grid.cpp:4-24 with halo = 1, then SetCFL (:33-37)
    GridGeom g;
    const int halo = 1;
    g.nx = d.nx_ + 2 * halo;
    g.ny = d.ny_ + 2 * halo;
    g.nxy = g.nx * g.ny;
    g.dx = (d.endx - d.startx) / ((double)g.nx - 1.0 - 2.0 * halo);
    g.dy = (d.endy - d.starty) / ((double)g.ny - 1.0 - 2.0 * halo);
    g.startx = d.startx - g.dx;
    g.starty = d.starty - g.dy;
    g.endx = d.endx + g.dx;
    g.endy = d.endy + g.dy;
    g.cfl = d.cfl;
    g.dt = d.cfl * std::min(g.dx, g.dy);
    return g;
}

void invert3(const double *m, double *r)
{
    const double a = m[4] * m[8] - m[5] * m[7];
    const double b = m[5] * m[6] - m[3] * m[8];
    const double c = m[3] * m[7] - m[4] * m[6];
    const double inv = 1.0 / (m[0] * a + m[1] * b + m[2] * c);
    r[0] = a * inv;
    r[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
    r[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    r[3] = b * inv;
    r[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    r[6] = c * inv;
    r[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
}

double fourier_basis(int k, double phi)
{
    const double sqrt2 = 1.41421356237309504880;
    if (k == 0)
        return 1.0;
    if (k % 2 != 0)
        return sqrt2 * std::cos(phi * (k + 1.0) / 2.0);
    return sqrt2 * std::sin(phi * k / 2.0);
}

// ------------------------------------------------------------------ stencil
namespace
{
// Nearest direction and the 4-point cubic Lagrange stencil around phi
// (src/Stencil.cpp:109-162).
void cubic_row(const StencilTables &s, double phi, int64_t *idx, double *wt)
{
    int nearest = -1;
    double best = 10;
    for (int d = 0; d < s.n; d++)
    {
        const double delta = std::abs(phi - s.phi[d]);
        const double dist = std::min(delta, 2.0 * kPi - delta);
        if (dist < best)
        {
            best = dist;
            nearest = d;
        }
    }
    const int64_t n = s.n;
    const bool left = std::fmod(s.phi[nearest] + kPi - phi, 2.0 * kPi) < kPi;
    const int first = left ? nearest - 1 : nearest - 2;
    for (int k = 0; k < 4; k++)
        idx[k] = (first + k + n) % n;
    for (int i = 0; i < 4; i++)
    {
        double weight = 1;
        const double pi_ = std::fmod(s.phi[idx[i]] + kPi - phi + 2.0 * kPi, 2.0 * kPi);
        for (int j = 0; j < 4; j++)
        {
            const double pj = std::fmod(s.phi[idx[j]] + kPi - phi + 2.0 * kPi, 2.0 * kPi);
            if (i != j)
                weight *= (kPi - pj) / (pi_ - pj);
        }
        wt[i] = weight;
    }
}

// LookUpTable::Add (src/DataTypes.hh:644-670): sorted insert, duplicates dropped
void lut_insert(StencilTables &s, double in, double sigma, double norm)
{
    auto &v = s.lut_in;
    size_t pos;
    if (v.empty() || in < v.front())
        pos = 0;
    else if (in > v.back())
        pos = v.size();
    else
    {
        auto it = std::lower_bound(v.begin(), v.end(), in);
        if (it != v.end() && !(in < *it))
            return;
        pos = (size_t)(it - v.begin());
    }
    v.insert(v.begin() + pos, in);
    s.lut_sigma.insert(s.lut_sigma.begin() + pos, sigma);
    s.lut_norm.insert(s.lut_norm.begin() + pos, norm);
}

// Stencil::PopulateLookUpTable (src/Stencil.cpp:378-455), bounded.
void build_flux_table(StencilTables &s)
{
    const double deltaPhi = kPi / 8.0 + 1e-8;
    const double maxError = 0.01;
    std::vector<double> I(s.n);
    double sigma = 0, refinement = 1;
    for (long pass = 0; pass < 1000000; pass++)
    {
        // flux direction (1, 0): Dot(F, C(d)) = 1*cx + 0*cy
        double normalization = 0;
        for (int d = 0; d < s.n; d++)
            normalization += s.w[d] * std::exp(sigma * (1.0 * s.cx[d] + 0.0 * s.cy[d]));
        normalization = std::log(normalization);
        double fx = 0, fy = 0;
        for (int d = 0; d < s.n; d++)
        {
            I[d] = 1.0 * std::exp(sigma * (1.0 * s.cx[d] + 0.0 * s.cy[d]) - normalization);
            const double c = s.w[d] * I[d];
            fx += c * s.cx[d];
            fy += c * s.cy[d];
        }
        const double currentF = std::sqrt(fx * fx + fy * fy);
        double err = 0;
        int count = 0;
        for (int g = 0; g < s.ng; g++)
        {
            const double gphi = 2.0 * kPi * g / (double)s.ng;
            const double gcx = approx_cos(gphi), gcy = approx_sin(gphi);
            if (approx_acos(1.0 * gcx + 0.0 * gcy) > deltaPhi / 2.0)
                continue;
            const double exact = 1.0 * std::exp(sigma * (1.0 * gcx + 0.0 * gcy) - normalization);
            double interp = 0;
            for (int p = 0; p < 4; p++)
                interp += s.ig_weight[4 * g + p] * I[s.ig_index[4 * g + p]];
            err += std::abs((exact - interp) / exact);
            count++;
        }
        err /= count;
        if (err > maxError)
        {
            sigma -= std::pow(10, -refinement);
            refinement++;
            sigma += std::pow(10, -refinement);
            if (refinement >= 8)
                break;
        }
        else
        {
            lut_insert(s, currentF, sigma, normalization);
            sigma += std::pow(10, -refinement);
        }
    }
}
} // namespace

StencilTables StencilTables::build(int n_order, bool intensity)
{
    StencilTables s;
    s.n = n_order;
    s.w.resize(n_order);
    s.phi.resize(n_order);
    s.cx.resize(n_order);
    s.cy.resize(n_order);
    // src/Stencil.cpp:194-200
    for (int d = 0; d < n_order; d++)
    {
        s.w[d] = 1.0 / (double)n_order;
        s.phi[d] = 2.0 * kPi * (d + 0.5) / (double)n_order;
        s.cx[d] = approx_cos(s.phi[d]);
        s.cy[d] = approx_sin(s.phi[d]);
    }
    s.ng = intensity ? 10 * n_order : 3;
    s.ig_index.resize(4 * (size_t)s.ng);
    s.ig_weight.resize(4 * (size_t)s.ng);
    for (int g = 0; g < s.ng; g++)
        cubic_row(s, 2.0 * kPi * g / (double)s.ng, &s.ig_index[4 * g], &s.ig_weight[4 * g]);
    if (intensity)
        build_flux_table(s);
    return s;
}

// LookUpTable::Evaluate (src/DataTypes.hh:672-701)
double StencilTables::lut_eval(const std::vector<double> &out, double x) const
{
    const auto &in = lut_in;
    const size_t size = in.size();
    if (x <= in[0] || size == 1)
        return out[0];
    if (x >= in[size - 1])
        return out[size - 1];
    const size_t hi = (size_t)(std::lower_bound(in.begin(), in.end(), x) - in.begin());
    const size_t lo = hi - 1;
    if (in[lo] == x)
        return out[lo];
    const double t = (x - in[lo]) / (in[hi] - in[lo]);
    return out[lo] + t * (out[hi] - out[lo]);
}

// ------------------------------------------------------------------- metric
void MetricArrays::metric_function(double x, double y, double *gl) const
{
    // src/Spacetimes.cpp:21-24 (Minkowski), 48-64 (SchwarzSchild), 87-112 (KerrSchild)
    static const double eta[9] = {-1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(gl, eta, sizeof(eta));
    if (kind == GRLBM_SCHWARZSCHILD)
    {
        const double rs = 2.0 * m;
        const double r2 = x * x + y * y;
        const double r = std::sqrt(r2);
        if (r > 2.0 * m)
        {
            gl[0] = -1.0 + rs / r;
            gl[4] = x * x / (r2 - rs * r) + y * y / r2;
            gl[8] = x * x / r2 + y * y / (r2 - rs * r);
            gl[5] = gl[7] = rs * x * y / (r2 * (r - rs));
        }
    }
    else if (kind == GRLBM_KERRSCHILD)
    {
        const double a2 = a * a;
        const double R2 = x * x + y * y;
        if (R2 > a2)
        {
            const double r2 = R2 - a2;
            const double r = std::sqrt(r2);
            const double rho2 = r2 + a2;
            const double H = m / r;
            const double l[3] = {1, (r * x + a * y) / rho2, (r * y - a * x) / rho2};
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    gl[3 * i + j] = (i == 0 && j == 0) ? -1.0 + 2.0 * H * l[i] * l[j]
                                                       : (double)(i == j) + 2.0 * H * l[i] * l[j];
        }
    }
}

MetricArrays MetricArrays::build(const GridGeom &g, const grlbm_metric_desc &d)
{
    MetricArrays M;
    M.kind = d.kind;
    M.m = d.m;
    M.a = d.a;
    const double rex = d.excision > 0 ? d.excision : 2.1;
    M.excision2 = rex * rex * d.m * d.m;
    M.g = g;
    M.arr.assign((size_t)kMetricArrays * g.nxy, 0.0);
    const int64_t nx = g.nx, ny = g.ny;

    // 4th-order central differences with step 1e-8 (src/Metric.cpp:189-219)
    auto deriv = [&](int axis, double x, double y, bool inverse, double *out) {
        const double h = 1e-8;
        const double ex = (axis == 1), ey = (axis == 2);
        double m2[9], m1[9], p1[9], p2[9], t[9];
        M.metric_function(x - 2 * h * ex, y - 2 * h * ey, m2);
        M.metric_function(x - 1 * h * ex, y - 1 * h * ey, m1);
        M.metric_function(x + 1 * h * ex, y + 1 * h * ey, p1);
        M.metric_function(x + 2 * h * ex, y + 2 * h * ey, p2);
        if (inverse)
            for (double *q : {m2, m1, p1, p2})
            {
                invert3(q, t);
                std::memcpy(q, t, sizeof(t));
            }
        for (int c = 0; c < 9; c++)
            out[c] = (1.0 / 12.0 * m2[c] - 1 / 12.0 * p2[c] - 2.0 / 3.0 * m1[c] + 2.0 / 3.0 * p1[c]) / h;
    };

    static const int kComp[6] = {0, 1, 2, 4, 5, 8}; // 00 01 02 11 12 22
    for (int64_t j = 0; j < ny; j++)
        for (int64_t i = 0; i < nx; i++)
        {
            const int64_t ij = i + j * nx;
            const double x = g.x((double)i), y = g.y((double)j);
            // InitializeMetricOnGrid (src/Metric.cpp:126-150)
            double gl[9], gu[9];
            M.metric_function(x, y, gl);
            invert3(gl, gu);
            for (int c = 0; c < 6; c++)
            {
                M.at(G00L + 2 * c, ij) = gl[kComp[c]];
                M.at(G00U + 2 * c, ij) = gu[kComp[c]];
            }
            // InitializeMetricDerivativesOnGrid (src/Metric.cpp:221-274)
            double dxl[9], dyl[9], dxu[9], dyu[9];
            deriv(1, x, y, false, dxl);
            deriv(2, x, y, false, dyl);
            deriv(1, x, y, true, dxu);
            deriv(2, x, y, true, dyu);
            for (int c = 0; c < 6; c++)
            {
                M.at(D0G00L + 3 * c, ij) = 0.0;
                M.at(D1G00L + 3 * c, ij) = dxl[kComp[c]];
                M.at(D2G00L + 3 * c, ij) = dyl[kComp[c]];
                M.at(D0G00U + 3 * c, ij) = 0.0;
                M.at(D1G00U + 3 * c, ij) = dxu[kComp[c]];
                M.at(D2G00U + 3 * c, ij) = dyu[kComp[c]];
            }
        }

    // InitializeAdmComponentsOnGrid (src/Metric.cpp:276-336)
    for (int64_t ij = 0; ij < g.nxy; ij++)
    {
        const double g00u = M.at(G00U, ij), g01u = M.at(G01U, ij), g02u = M.at(G02U, ij);
        const double al = 1.0 / std::sqrt(-g00u);
        const double b1 = al * al * g01u, b2 = al * al * g02u;
        M.at(ALPHA, ij) = al;
        M.at(BETA1U, ij) = b1;
        M.at(BETA2U, ij) = b2;
        M.at(BETA1L, ij) = M.at(G01L, ij);
        M.at(BETA2L, ij) = M.at(G02L, ij);
        M.at(GAM11L, ij) = M.at(G11L, ij);
        M.at(GAM12L, ij) = M.at(G12L, ij);
        M.at(GAM22L, ij) = M.at(G22L, ij);
        M.at(GAM11U, ij) = M.at(G11U, ij) + b1 * b1 / (al * al);
        M.at(GAM12U, ij) = M.at(G12U, ij) + b1 * b2 / (al * al);
        M.at(GAM22U, ij) = M.at(G22U, ij) + b2 * b2 / (al * al);
        const double da[3] = {0, M.at(D1G00U, ij) / (2.0 * std::pow(-g00u, 3.0 / 2.0)),
                              M.at(D2G00U, ij) / (2.0 * std::pow(-g00u, 3.0 / 2.0))};
        M.at(D1ALPHA, ij) = da[1];
        M.at(D2ALPHA, ij) = da[2];
        // db[b][c] = d_b beta^c
        double db[3][3] = {};
        for (int b = 1; b < 3; b++)
        {
            db[b][1] = al * al * M.at(b == 1 ? D1G01U : D2G01U, ij) + 2.0 * g01u * al * da[b];
            db[b][2] = al * al * M.at(b == 1 ? D1G02U : D2G02U, ij) + 2.0 * g02u * al * da[b];
        }
        M.at(D1BETA1LU, ij) = db[1][1];
        M.at(D1BETA2LU, ij) = db[1][2];
        M.at(D2BETA1LU, ij) = db[2][1];
        M.at(D2BETA2LU, ij) = db[2][2];
        M.at(D1BETA1LL, ij) = M.at(D1G01L, ij);
        M.at(D1BETA2LL, ij) = M.at(D1G02L, ij);
        M.at(D2BETA1LL, ij) = M.at(D2G01L, ij);
        M.at(D2BETA2LL, ij) = M.at(D2G02L, ij);
        M.at(D1GAM11LLL, ij) = M.at(D1G11L, ij);
        M.at(D2GAM11LLL, ij) = M.at(D2G11L, ij);
        M.at(D1GAM12LLL, ij) = M.at(D1G12L, ij);
        M.at(D2GAM12LLL, ij) = M.at(D2G12L, ij);
        M.at(D1GAM22LLL, ij) = M.at(D1G22L, ij);
        M.at(D2GAM22LLL, ij) = M.at(D2G22L, ij);
        const double a3 = std::pow(al, 3);
        const double beta[3] = {0, b1, b2};
        // d_k gamma^{pq} = d_k g^{pq} + (d_k b^p b^q + b^p d_k b^q)/a^2 - 2 b^p b^q d_k a / a^3
        struct
        {
            int out, gu, p, q;
        } const comps[6] = {{D1GAM11LUU, D1G11U, 1, 1}, {D1GAM12LUU, D1G12U, 1, 2}, {D1GAM22LUU, D1G22U, 2, 2},
                            {D2GAM11LUU, D2G11U, 1, 1}, {D2GAM12LUU, D2G12U, 1, 2}, {D2GAM22LUU, D2G22U, 2, 2}};
        for (int c = 0; c < 6; c++)
        {
            const int k = c < 3 ? 1 : 2;
            const int p = comps[c].p, q = comps[c].q;
            M.at(comps[c].out, ij) = M.at(comps[c].gu, ij) + (db[k][p] * beta[q] + beta[p] * db[k][q]) / (al * al) -
                                     2.0 * beta[p] * beta[q] * da[k] / a3;
        }
        // extrinsic curvature with a static 3-metric
        const double gam[3][3] = {{0, 0, 0}, {0, M.at(GAM11L, ij), M.at(GAM12L, ij)}, {0, M.at(GAM12L, ij), M.at(GAM22L, ij)}};
        double dg[3][3][3] = {}; // [c][a][b] = d_c gamma_ab
        dg[1][1][1] = M.at(D1GAM11LLL, ij);
        dg[1][1][2] = dg[1][2][1] = M.at(D1GAM12LLL, ij);
        dg[1][2][2] = M.at(D1GAM22LLL, ij);
        dg[2][1][1] = M.at(D2GAM11LLL, ij);
        dg[2][1][2] = dg[2][2][1] = M.at(D2GAM12LLL, ij);
        dg[2][2][2] = M.at(D2GAM22LLL, ij);
        double K[3][3];
        for (int a_ = 1; a_ < 3; a_++)
            for (int b = 1; b < 3; b++)
            {
                K[a_][b] = -0.0;
                for (int c = 1; c < 3; c++)
                    K[a_][b] += 2.0 * gam[a_][c] * db[b][c] + dg[c][a_][b] * beta[c];
                K[a_][b] /= 2.0 * al;
            }
        M.at(K11L, ij) = K[1][1];
        M.at(K12L, ij) = K[1][2];
        M.at(K22L, ij) = K[2][2];
    }

    // InitializeBoostedTetradOnGrid (src/Metric.cpp:152-187)
    for (int64_t ij = 0; ij < g.nxy; ij++)
    {
        const double s = 1.0 / std::sqrt(M.at(GAM11U, ij));
        const double b = s * s * M.at(GAM12U, ij);
        const double g2 = 1.0 * M.at(GAM22L, ij) * 1.0;
        const double al = M.at(ALPHA, ij);
        const double t[9] = {1.0 / al, 0, 0, -M.at(BETA1U, ij) / al, 1 / s, 0, -M.at(BETA2U, ij) / al, b / s, 1 / std::sqrt(g2)};
        double ti[9];
        invert3(t, ti);
        for (int q = 0; q < 9; q++)
        {
            M.at(TET00 + q, ij) = t[q];
            M.at(ITET00 + q, ij) = ti[q];
        }
    }
    return M;
}

// ------------------------------------------------------------------ sources
Sources build_sources(const MetricArrays &M, const StencilTables &st, int initial_data_type,
                      const uint8_t *is_initial, const double *initial_I, const double *E,
                      const double *Fx, const double *Fy, const double *Pxx, const double *Pxy,
                      const double *Pyy, bool adaptive, const double *flux_angle)
{
    Sources S;
    const int nd = st.n;
    for (int64_t ij = 0; ij < M.g.nxy; ij++)
    {
        if (!is_initial || !is_initial[ij])
            continue;
        S.nodes.push_back(ij);
        const size_t base = S.intensities.size();
        S.intensities.resize(base + nd);
        double *I = &S.intensities[base];
        if (initial_data_type == GRLBM_INTENSITIES)
        {
            for (int d = 0; d < nd; d++)
                I[d] = initial_I ? initial_I[ij * nd + d] : 0.0;
            if (adaptive)
            {
                // rotationAngle[ij] = initialFluxAngle_IF[ij] (src/Radiation.cpp:177)
                S.angle_nodes.push_back(ij);
                S.angles.push_back(flux_angle ? flux_angle[ij] : 0.0);
            }
            continue;
        }
        // InitialDataLFtoIF (src/Radiation.cpp:103-127): E from the boosted
        // tensor, the flux taken from the lab-frame tensor as the reference does
        const double T[9] = {E[ij], Fx[ij], Fy[ij], Fx[ij], Pxx[ij], Pxy[ij], Fy[ij], Pxy[ij], Pyy[ij]};
        double e[9], ie[9];
        for (int q = 0; q < 9; q++)
            e[q] = M.at(TET00 + q, ij);
        invert3(e, ie);
        double e00 = 0.0;
        for (int A = 0; A < 3; A++)
            for (int B = 0; B < 3; B++)
                e00 += T[3 * A + B] * ie[A] * ie[B];
        double fx = T[1], fy = T[2];
        const double f0 = std::sqrt(fx * fx + fy * fy);
        if (f0 > e00)
        {
            fx *= e00 / f0;
            fy *= e00 / f0;
        }
        // LoadInitialData, InitialDataType::Moments (src/Radiation.cpp:150-174)
        const double f = std::sqrt(fx * fx + fy * fy);
        const double rel = f / e00;
        double dir1 = adaptive ? 1.0 : fx / f, dir2 = adaptive ? 0.0 : fy / f;
        if (f < 1e-16)
        {
            dir1 = 1;
            dir2 = 0;
        }
        if (adaptive && !(f < 1e-16))
        {
            // rotationAngle[ij] (src/Radiation.cpp:170-171)
            S.angle_nodes.push_back(ij);
            S.angles.push_back(std::fmod(approx_atan2(fy, fx) + 2.0 * kPi, 2.0 * kPi));
        }
        const double sigma = st.lut_eval(st.lut_sigma, rel);
        const double norm = st.lut_eval(st.lut_norm, rel);
        for (int d = 0; d < nd; d++)
            I[d] = e00 * std::exp(sigma * (dir1 * st.cx[d] + dir2 * st.cy[d]) - norm);
    }
    return S;
}
} // namespace grlbm
