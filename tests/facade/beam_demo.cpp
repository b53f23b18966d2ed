// User code of the reference's beam examples (exe/main.cpp:246-343
// BeamCrossing, :538-598 CurvedBeam) at a reduced size, written once as a
// template and run on the reference's own Radiation and on RadiationB200:
// the facade is a drop-in for that code.  Test infrastructure only, built
// by oracle/Makefile (target `facade`) from the reference's sources.
//
//   beam_demo nogpu               construct a RadiationB200; exit 0 when the
//                                 constructor throws (prints the message)
//   beam_demo flat|curved <dir> [precision]
//                                 run both classes in <dir> (RadiationB200 in
//                                 the given arithmetic form, default the
//                                 plain one); print one line per compared
//                                 buffer: name max|a-b| max|a|
#include "RadiationB200.h"

#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace
{
struct Case
{
    bool curved;
    size_t nx, ny;
    Coord start, end;
    double cfl, sim_time;
    int n_dir, n_fourier;
};

Case make_case(bool curved)
{
    if (curved)
        return Case{true, 61, 49, Coord(0, 0), Coord(5, 4), 0.9, 1.5, 24, 5};
    return Case{false, 81, 41, Coord(-0.5, -0.25), Coord(0.5, 0.25), 0.9, 0.4, 40, 5};
}

Config make_config(const Case &c, const std::string &name, StreamingType type)
{
    Config config;
    config.name = name;
    config.t0 = 0;
    config.simTime = c.sim_time;
    config.writePeriod = c.sim_time / 2;
    config.updateFourierHarmonics = false;
    config.keepSourceNodesActive = true;
    config.writeData = true;
    config.printSetup = false;
    config.printProgress = false;
    config.printResults = false;
    config.saveInitialData = true;
    config.streamingType = type;
    config.initialDataType = c.curved ? InitialDataType::Moments : InitialDataType::Intensities;
    return config;
}

// The set-up of BeamCrossing (two beams, intensities) or CurvedBeam (one
// beam entering at the left edge, moments), identical for both classes.
template <class R>
void set_up(R &radiation, const Case &c, Grid &grid, Metric &metric, Stencil &stencil)
{
    Tensor2 dir0 = Tensor2(0.3, 0.1).EuklNormalized();
    Tensor2 dir1 = Tensor2(0.3, -0.1).EuklNormalized();
    int d0 = -1, d1 = -1;
    float dist0 = 1e10, dist1 = 1e10;
    for (int d = 0; d < (int)stencil.nDir; d++)
    {
        float dist = (dir0 - stencil.C(d)).EuklNorm();
        if (dist < dist0)
            dist0 = dist, d0 = d;
        dist = (dir1 - stencil.C(d)).EuklNorm();
        if (dist < dist1)
            dist1 = dist, d1 = d;
    }
    for (size_t j = 0; j < grid.ny; j++)
        for (size_t i = 0; i < grid.nx; i++)
        {
            const size_t ij = grid.Index(i, j);
            const Coord xy = grid.xy(i, j);
            const double x = xy[1], y = xy[2];
            radiation.kappa0[ij] = radiation.kappa1[ij] = radiation.kappaA[ij] = radiation.eta[ij] = 0;
            if (c.curved)
            {
                if (3.0 < y && y < 3.5 && i <= 1)
                {
                    Tensor3 uLF(1, 1, 0);
                    uLF = NullNormalize(uLF, metric.GetMetric_ll(ij));
                    Tensor2 vLF = Vec2ObservedByEulObs<LF, LF>(uLF, xy, metric);
                    radiation.isInitialGridPoint[ij] = true;
                    radiation.initialE_LF[ij] = 1;
                    radiation.initialFx_LF[ij] = 10 * vLF[1];
                    radiation.initialFy_LF[ij] = 10 * vLF[2];
                }
                continue;
            }
            if (-0.45 - grid.dx < x && x <= -0.45 && -0.20 < y && y < -0.15)
            {
                radiation.isInitialGridPoint[ij] = true;
                radiation.initialE_LF[ij] = 1;
                radiation.initialFx_LF[ij] = dir0[1];
                radiation.initialFy_LF[ij] = dir0[2];
                radiation.initialI[radiation.Index(ij, d0)] = 1.0 / stencil.W(d0);
            }
            if (-0.45 - grid.dx < x && x <= -0.45 && 0.15 < y && y < 0.20)
            {
                radiation.isInitialGridPoint[ij] = true;
                radiation.initialE_LF[ij] = 1;
                radiation.initialFx_LF[ij] = dir1[1];
                radiation.initialFy_LF[ij] = dir1[2];
                radiation.initialI[radiation.Index(ij, d1)] = 1.0 / stencil.W(d1);
            }
        }
}

// name, max |a - b|, max |a|; then where the largest difference is
void compare(const char *name, const DoubleBuffer &a, const DoubleBuffer &b)
{
    double diff = 0, mag = 0;
    size_t at = 0;
    for (size_t k = 0; k < a.size(); k++)
    {
        if (std::fabs(a[k] - b[k]) > diff)
            diff = std::fabs(a[k] - b[k]), at = k;
        mag = std::max(mag, std::fabs(a[k]));
    }
    std::printf("%s %.17g %.17g\n", name, diff, mag);
    if (diff > 0)
        std::fprintf(stderr, "  %s: largest difference at element %zu of %zu: %.17g vs %.17g\n", name, at, a.size(),
                     a[at], b[at]);
}

int run_nogpu()
{
    const Case c = make_case(false);
    Grid grid(c.nx, c.ny, c.start, c.end);
    grid.SetCFL(c.cfl);
    Minkowski metric(grid, 1.0, 0.0);
    Stencil stencil(c.n_dir, 0);
    Stencil streaming(c.n_fourier, 0, false);
    try
    {
        RadiationB200 r(metric, stencil, streaming, make_config(c, "nogpu", StreamingType::FlatFixed));
    }
    catch (const std::runtime_error &e)
    {
        std::printf("refused: %s\n", e.what());
        return 0;
    }
    std::printf("constructed\n");
    return 3;
}

int run_pair(bool curved, int precision)
{
    const Case c = make_case(curved);
    Grid grid(c.nx, c.ny, c.start, c.end);
    grid.SetCFL(c.cfl);
    Metric *metric = curved ? (Metric *)new SchwarzSchild(grid, 1.0, 0.0) : (Metric *)new Minkowski(grid, 1.0, 0.0);
    Stencil stencil(c.n_dir, 0);
    Stencil streaming(c.n_fourier, 0, false);
    const StreamingType type = curved ? StreamingType::CurvedFixed : StreamingType::FlatFixed;

    Radiation ref(*metric, stencil, streaming, make_config(c, "ref", type));
    set_up(ref, c, grid, *metric, stencil);
    ref.RunSimulation();

    RadiationB200 gpu(*metric, stencil, streaming, make_config(c, "b200", type), precision);
    set_up(gpu, c, grid, *metric, stencil);
    gpu.RunSimulation();

    compare("I", ref.I, gpu.I);
    compare("E", ref.E, gpu.E);
    compare("Fx", ref.Fx, gpu.Fx);
    compare("Fy", ref.Fy, gpu.Fy);
    compare("Pxx", ref.Pxx, gpu.Pxx);
    compare("E_LF", ref.E_LF, gpu.E_LF);
    compare("F_LF", ref.F_LF, gpu.F_LF);
    compare("coefficientsS", ref.coefficientsS, gpu.coefficientsS);
    compare("coefficientsX", ref.coefficientsX, gpu.coefficientsX);
    std::printf("maxItterationCount %d %d\n", ref.maxItterationCount, gpu.maxItterationCount);
    std::printf("averageItterationCount %.17g %.17g\n", ref.averageItterationCount, gpu.averageItterationCount);
    std::printf("timeSteps %d %d\n", ref.logger.timeSteps, gpu.logger.timeSteps);
    delete metric;
    return 0;
}
} // namespace

int main(int argc, char **argv)
{
    if (argc >= 2 && std::strcmp(argv[1], "nogpu") == 0)
        return run_nogpu();
    if (argc >= 3 && (std::strcmp(argv[1], "flat") == 0 || std::strcmp(argv[1], "curved") == 0))
    {
        if (chdir(argv[2]) != 0)
        {
            std::perror("chdir");
            return 2;
        }
        try
        {
            return run_pair(std::strcmp(argv[1], "curved") == 0, argc >= 4 ? std::atoi(argv[3]) : GRLBM_PLAIN_FP64);
        }
        catch (const std::exception &e)
        {
            std::printf("error: %s\n", e.what());
            return 4;
        }
    }
    std::fprintf(stderr, "usage: beam_demo nogpu | flat <dir> [precision] | curved <dir> [precision]\n");
    return 2;
}
