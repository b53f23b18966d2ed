// Driver that runs the reference implementation (Tom-Olsen/2dRadiation,
// compiled from its own unmodified sources by oracle/Makefile) behind the
// ref_run() entry point declared in oracle/ref_api.h.
//
// Test infrastructure only: it pins the oracle restatement and provides the
// timed CPU baseline.  It is never linked into the product library.
//
// Two deviations from the shipped constants are reachable without touching the
// reference sources:
//   * the excision radius: a subclass overrides the virtual InsideBH()
//     (reference: r <= 2.1 m, src/Spacetimes.cpp:42,81);
//   * the RK45 tolerance maxTE: ref_geodesic_tu.cpp compiles the reference's
//     src/GeodesicEquationSolver.cpp with `constexpr` defined away, which turns
//     `constexpr double maxTE = 1e-4;` (line 79) into a plain global that this
//     driver assigns before each run.
#include "Radiation.h"
#include "ref_api.h"
#include <chrono>
#include <cstring>
#include <omp.h>
#include <unistd.h>

extern double maxTE; // from ref_geodesic_tu.cpp

namespace
{
// Frame output of RunSimulation (ref_set_frames): off unless a directory is set.
double g_frame_period = 1e300;
std::string g_frame_workdir;

using MetricArray = DoubleBuffer Metric::*;
// Member order of src/Metric.h:19-65.
const MetricArray kMetricArrays[GRLBM_N_METRIC_ARRAYS] = {
    &Metric::g00_ll, &Metric::g00_uu, &Metric::g01_ll, &Metric::g01_uu, &Metric::g02_ll, &Metric::g02_uu,
    &Metric::g11_ll, &Metric::g11_uu, &Metric::g12_ll, &Metric::g12_uu, &Metric::g22_ll, &Metric::g22_uu,
    &Metric::d0_g00_lll, &Metric::d1_g00_lll, &Metric::d2_g00_lll,
    &Metric::d0_g01_lll, &Metric::d1_g01_lll, &Metric::d2_g01_lll,
    &Metric::d0_g02_lll, &Metric::d1_g02_lll, &Metric::d2_g02_lll,
    &Metric::d0_g11_lll, &Metric::d1_g11_lll, &Metric::d2_g11_lll,
    &Metric::d0_g12_lll, &Metric::d1_g12_lll, &Metric::d2_g12_lll,
    &Metric::d0_g22_lll, &Metric::d1_g22_lll, &Metric::d2_g22_lll,
    &Metric::d0_g00_luu, &Metric::d1_g00_luu, &Metric::d2_g00_luu,
    &Metric::d0_g01_luu, &Metric::d1_g01_luu, &Metric::d2_g01_luu,
    &Metric::d0_g02_luu, &Metric::d1_g02_luu, &Metric::d2_g02_luu,
    &Metric::d0_g11_luu, &Metric::d1_g11_luu, &Metric::d2_g11_luu,
    &Metric::d0_g12_luu, &Metric::d1_g12_luu, &Metric::d2_g12_luu,
    &Metric::d0_g22_luu, &Metric::d1_g22_luu, &Metric::d2_g22_luu,
    &Metric::alpha, &Metric::beta1_u, &Metric::beta1_l, &Metric::beta2_u, &Metric::beta2_l,
    &Metric::gamma11_ll, &Metric::gamma11_uu, &Metric::gamma12_ll, &Metric::gamma12_uu,
    &Metric::gamma22_ll, &Metric::gamma22_uu,
    &Metric::d1_alpha_l, &Metric::d2_alpha_l,
    &Metric::d1_beta1_lu, &Metric::d1_beta2_lu, &Metric::d2_beta1_lu, &Metric::d2_beta2_lu,
    &Metric::d1_beta1_ll, &Metric::d1_beta2_ll, &Metric::d2_beta1_ll, &Metric::d2_beta2_ll,
    &Metric::d1_gamma11_lll, &Metric::d2_gamma11_lll, &Metric::d1_gamma12_lll, &Metric::d2_gamma12_lll,
    &Metric::d1_gamma22_lll, &Metric::d2_gamma22_lll,
    &Metric::d1_gamma11_luu, &Metric::d2_gamma11_luu, &Metric::d1_gamma12_luu, &Metric::d2_gamma12_luu,
    &Metric::d1_gamma22_luu, &Metric::d2_gamma22_luu,
    &Metric::K11_ll, &Metric::K12_ll, &Metric::K22_ll,
    &Metric::tetrad00_ul, &Metric::tetrad01_ul, &Metric::tetrad02_ul,
    &Metric::tetrad10_ul, &Metric::tetrad11_ul, &Metric::tetrad12_ul,
    &Metric::tetrad20_ul, &Metric::tetrad21_ul, &Metric::tetrad22_ul,
    &Metric::tetrad00_lu, &Metric::tetrad01_lu, &Metric::tetrad02_lu,
    &Metric::tetrad10_lu, &Metric::tetrad11_lu, &Metric::tetrad12_lu,
    &Metric::tetrad20_lu, &Metric::tetrad21_lu, &Metric::tetrad22_lu,
};

template <class Base>
struct Excised : Base
{
    double r2;
    Excised(Grid &g, double m, double a, double rex) : Base(g, m, a), r2(rex * rex * m * m) {}
    bool InsideBH(const Coord &xy) override { return xy.EuklNormSquared() <= r2; }
};

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void copy_out(double *dst, const DoubleBuffer &src)
{
    if (dst)
        std::memcpy(dst, src.data(), src.size() * sizeof(double));
}
} // namespace

extern "C" int ref_run(const grlbm_ref_params *p, const grlbm_ref_inputs *in, grlbm_ref_outputs *out)
{
    if (p->n_threads > 0)
        omp_set_num_threads(p->n_threads);
    maxTE = p->rk_tol;

    Grid grid(p->nx_, p->ny_, Coord(p->startx, p->starty), Coord(p->endx, p->endy));
    grid.SetCFL(p->cfl);

    Metric *metric = nullptr;
    const bool excise = p->excision > 0;
    switch (p->metric_kind)
    {
    case 0:
        metric = new Minkowski(grid, p->m, p->a);
        break;
    case 1:
        metric = excise ? (Metric *)new Excised<SchwarzSchild>(grid, p->m, p->a, p->excision)
                        : (Metric *)new SchwarzSchild(grid, p->m, p->a);
        break;
    case 2:
        metric = excise ? (Metric *)new Excised<KerrSchild>(grid, p->m, p->a, p->excision)
                        : (Metric *)new KerrSchild(grid, p->m, p->a);
        break;
    default:
        return -1;
    }
    const size_t nxy = grid.nxy;
    for (int k = 0; k < GRLBM_N_METRIC_ARRAYS; k++)
    {
        DoubleBuffer &arr = metric->*kMetricArrays[k];
        if (out->metric_arrays)
            std::memcpy(out->metric_arrays + k * nxy, arr.data(), nxy * sizeof(double));
        if (in->metric_override)
            std::memcpy(arr.data(), in->metric_override + k * nxy, nxy * sizeof(double));
    }

    Stencil stencil(p->n_dir, 0);
    Stencil streamingStencil(p->n_fourier, 0, false);
    const size_t nDir = stencil.nDir;

    Config config = {
        .name = "ref_run",
        .t0 = 0,
        .simTime = (p->n_steps - 0.5) * grid.dt,
        .writePeriod = g_frame_workdir.empty() ? 1e300 : g_frame_period,
        .updateFourierHarmonics = p->update_tables_each_step != 0,
        .keepSourceNodesActive = p->keep_source_nodes_active != 0,
        .writeData = !g_frame_workdir.empty(),
        .printSetup = false,
        .printProgress = false,
        .printResults = false,
        .saveInitialData = !g_frame_workdir.empty(),
        .streamingType = (StreamingType)p->streaming_type,
        .initialDataType = (InitialDataType)p->initial_data_type,
    };
    Radiation *rad = new Radiation(*metric, stencil, streamingStencil, config);
    Radiation &r = *rad;
    for (size_t ij = 0; ij < nxy; ij++)
    {
        r.kappa0[ij] = in->kappa0[ij];
        r.kappa1[ij] = in->kappa1[ij];
        r.kappaA[ij] = in->kappaA[ij];
        r.eta[ij] = in->eta[ij];
        r.ux[ij] = in->ux[ij];
        r.uy[ij] = in->uy[ij];
        r.isInitialGridPoint[ij] = in->is_initial[ij] != 0;
        r.initialE_LF[ij] = in->initial_E_LF[ij];
        r.initialFx_LF[ij] = in->initial_Fx_LF[ij];
        r.initialFy_LF[ij] = in->initial_Fy_LF[ij];
        r.initialPxx_LF[ij] = in->initial_Pxx_LF[ij];
        r.initialPxy_LF[ij] = in->initial_Pxy_LF[ij];
        r.initialPyy_LF[ij] = in->initial_Pyy_LF[ij];
    }
    std::memcpy(r.initialI.data(), in->initial_I, nxy * nDir * sizeof(double));

    if (p->use_run_simulation)
    {
        // with frames on, the reference writes under ../output/<name>/ relative
        // to the working directory: run it from <workdir>/run
        char cwd[4096] = {0};
        const bool frames = !g_frame_workdir.empty();
        if (frames)
        {
            if (!getcwd(cwd, sizeof cwd) || chdir(g_frame_workdir.c_str()) != 0)
                return -2;
        }
        r.RunSimulation();
        if (frames && chdir(cwd) != 0)
            return -2;
        out->computation_time_s = r.logger.ComputationTime();
        out->table_time_s = Profiler::Session::Get().GetTotalTime("void Radiation::UpdateFourierCoefficients()");
        out->max_iterations = r.logger.maxItterationCount;
        out->average_iterations = r.logger.averageItterationCount;
    }
    else
    {
        // src/Radiation.cpp:745-832 with the file output, progress printing
        // and profiler session left out.
        r.LoadInitialData();
        auto t0 = std::chrono::steady_clock::now();
        r.UpdateFourierCoefficients();
        out->table_time_s = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        for (int n = 0; n < p->n_steps; n++)
        {
            auto ts = std::chrono::steady_clock::now();
            // src/Radiation.cpp:790-793
            if (config.updateFourierHarmonics)
                r.UpdateFourierCoefficients();
            if (config.keepSourceNodesActive)
                r.LoadInitialData();
            switch (config.streamingType)
            {
            case StreamingType::FlatFixed:
                r.StreamFlatFixed();
                break;
            case StreamingType::CurvedFixed:
                r.StreamCurvedFixed();
                break;
            case StreamingType::FlatAdaptive:
                r.UpdateRotationMatrizes();
                r.StreamFlatAdaptive();
                break;
            case StreamingType::CurvedAdaptive:
                r.UpdateRotationMatrizes();
                r.StreamCurvedAdaptive();
                break;
            default:
                return -2;
            }
            r.ComputeMomentsIF();
            r.Collide();
            if (out->step_times)
                out->step_times[n] = seconds_since(ts);
        }
        out->computation_time_s = seconds_since(t0);
        out->max_iterations = r.maxItterationCount;
        out->average_iterations =
            r.averageItterationCount / ((double)p->n_steps * (grid.nx - 2) * (grid.ny - 2));
    }

    copy_out(out->E, r.E);
    copy_out(out->Fx, r.Fx);
    copy_out(out->Fy, r.Fy);
    copy_out(out->Pxx, r.Pxx);
    copy_out(out->Pxy, r.Pxy);
    copy_out(out->Pyy, r.Pyy);
    copy_out(out->I, r.I);
    copy_out(out->coefS, r.coefficientsS);
    copy_out(out->coefX, r.coefficientsX);
    copy_out(out->coefY, r.coefficientsY);
    copy_out(out->coefCx, r.coefficientsCx);
    copy_out(out->coefCy, r.coefficientsCy);
    r.ComputeMomentsLF();
    copy_out(out->E_LF, r.E_LF);
    copy_out(out->Fx_LF, r.Fx_LF);
    copy_out(out->Fy_LF, r.Fy_LF);
    copy_out(out->Pxx_LF, r.Pxx_LF);
    copy_out(out->Pxy_LF, r.Pxy_LF);
    copy_out(out->Pyy_LF, r.Pyy_LF);
    copy_out(out->F_LF, r.F_LF);

    for (size_t d = 0; d < nDir; d++)
    {
        if (out->st_w)
            out->st_w[d] = stencil.W(d);
        if (out->st_phi)
            out->st_phi[d] = stencil.Phi(d);
        if (out->st_cx)
            out->st_cx[d] = stencil.Cx(d);
        if (out->st_cy)
            out->st_cy[d] = stencil.Cy(d);
    }
    for (size_t g = 0; g < stencil.interpolationGrid.nGrid; g++)
        for (int k = 0; k < 4; k++)
        {
            if (out->ig_index)
                out->ig_index[4 * g + k] = (int64_t)stencil.interpolationGrid.neighbourIndexesCubic[g][k];
            if (out->ig_weight)
                out->ig_weight[4 * g + k] = stencil.interpolationGrid.neighbourWeightsCubic[g][k];
        }
    for (size_t f = 0; f < streamingStencil.nDir; f++)
    {
        if (out->ss_phi)
            out->ss_phi[f] = streamingStencil.Phi(f);
        if (out->ss_w)
            out->ss_w[f] = streamingStencil.W(f);
    }
    delete rad;
    delete metric;
    return 0;
}

// Frame output for the next RunSimulation runs (use_run_simulation): every
// write_period and at the start and end, into <workdir>/../output/ref_run/
// Moments/; workdir NULL turns it off.
extern "C" void ref_set_frames(double write_period, const char *workdir)
{
    g_frame_period = write_period;
    g_frame_workdir = workdir ? workdir : "";
}

// Grid::WriteFrametoCsv of a grid built like ref_run's, for host arrays.
extern "C" int ref_write_frame(const grlbm_ref_params *p, float time, const double *r, const double *g,
                               const double *b, const double *a, const char *directory, const char *name)
{
    Grid grid(p->nx_, p->ny_, Coord(p->startx, p->starty), Coord(p->endx, p->endy));
    grid.SetCFL(p->cfl);
    DoubleBuffer R(grid.nxy), G(grid.nxy), B(grid.nxy), A(grid.nxy);
    std::memcpy(R.data(), r, grid.nxy * sizeof(double));
    std::memcpy(G.data(), g, grid.nxy * sizeof(double));
    std::memcpy(B.data(), b, grid.nxy * sizeof(double));
    std::memcpy(A.data(), a, grid.nxy * sizeof(double));
    grid.WriteFrametoCsv(time, R, G, B, A, directory, name ? name : "");
    return 0;
}
