// Host-side set-up of one radiation problem: grid geometry, stencil tables,
// metric arrays and source intensities.  These are the tables the reference
// builds in its constructors (src/Grid.cpp, src/Stencil.cpp, src/Metric.cpp,
// src/Spacetimes.cpp) and in Radiation::LoadInitialData; the device kernels
// consume them unchanged.  Everything here is FP64 with the reference's
// association order, built without floating-point contraction, so the arrays
// are bit-identical to the reference's IEEE build.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/grlbm.h"

namespace grlbm
{
constexpr int kMetricArrays = 102;

// Indices of the metric arrays in the member order of src/Metric.h:19-65.
enum MetricIndex : int
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
    K11L, K12L, K22L,
    TET00, TET01, TET02, TET10, TET11, TET12, TET20, TET21, TET22,
    ITET00, ITET01, ITET02, ITET10, ITET11, ITET12, ITET20, ITET21, ITET22,
    kMetricIndexEnd
};
static_assert(kMetricIndexEnd == kMetricArrays, "metric array count");

// Grid(nx_, ny_, start, end, halo=1) + SetCFL (src/Grid.cpp:4-37)
struct GridGeom
{
    int64_t nx = 0, ny = 0, nxy = 0;
    double dx = 0, dy = 0, dt = 0, cfl = 1;
    double startx = 0, starty = 0, endx = 0, endy = 0;

    static GridGeom from(const grlbm_grid_desc &d);
    double x(double i) const { return startx + i * dx; }
    double y(double j) const { return starty + j * dy; }
    double fi(double xx) const { return (xx - startx) / dx; }
    double fj(double yy) const { return (yy - starty) / dy; }
    bool outside(double xx, double yy) const { return xx > endx || xx < startx || yy > endy || yy < starty; }
};

// Stencil(nOrder, 0, isIntensity) with its cubic InterpolationGrid and the
// flux -> sigma / normalization look-up tables (src/Stencil.cpp:4-455).
struct StencilTables
{
    int n = 0;
    std::vector<double> w, phi, cx, cy;
    int ng = 0;                      // interpolation grid rows (10 n)
    std::vector<int64_t> ig_index;   // 4 per row
    std::vector<double> ig_weight;   // 4 per row
    std::vector<double> lut_in, lut_sigma, lut_norm;

    static StencilTables build(int n_order, bool intensity);
    double lut_eval(const std::vector<double> &out, double x) const;
};

// The Metric class arrays (src/Metric.cpp:126-336) for one spacetime.
struct MetricArrays
{
    int kind = 0;
    double m = 1, a = 0, excision2 = 0;
    GridGeom g;
    std::vector<double> arr; // kMetricArrays * nxy

    static MetricArrays build(const GridGeom &g, const grlbm_metric_desc &d);
    double &at(int k, int64_t ij) { return arr[(size_t)k * g.nxy + ij]; }
    double at(int k, int64_t ij) const { return arr[(size_t)k * g.nxy + ij]; }
    bool inside_bh(double x, double y) const { return kind != GRLBM_MINKOWSKI && x * x + y * y <= excision2; }
    void metric_function(double x, double y, double *g_ll) const;
};

// Row-major 3x3 inverse, adjugate over determinant, fixed operation order.
void invert3(const double *m, double *r);

// Source intensities of Radiation::LoadInitialData for every flagged node
// (src/Radiation.cpp:103-182, fixed streaming): returns the node indices and
// their nDir intensities.
struct Sources
{
    std::vector<int64_t> nodes;
    std::vector<double> intensities; // nodes.size() * nDir, node-major
    // adaptive streaming: the rotation angles LoadInitialData sets
    std::vector<int64_t> angle_nodes;
    std::vector<double> angles;
};
// adaptive: the adaptive streaming types (von Mises distributions around
// direction (1, 0), angles from the flux or from flux_angle (nx*ny; NULL: 0)).
Sources build_sources(const MetricArrays &M, const StencilTables &st, int initial_data_type,
                      const uint8_t *is_initial, const double *initial_I, const double *E,
                      const double *Fx, const double *Fy, const double *Pxx, const double *Pxy,
                      const double *Pyy, bool adaptive = false, const double *flux_angle = nullptr);

// Fourier basis of src/FourierHarmonics.cpp:5-14 (libm cos/sin).
double fourier_basis(int k, double phi);
} // namespace grlbm
