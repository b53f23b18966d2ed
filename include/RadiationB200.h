/* RadiationB200: the reference's Radiation class (src/Radiation.h) with its
 * set-up, table build and time loop run on the GPU through libgrlbm.  User
 * code written against Radiation -- construct it from a Metric, two Stencils
 * and a Config, write kappa0 ... uy and the initial data, call
 * RunSimulation(), read the moments -- compiles and runs unchanged against
 * RadiationB200.
 *
 * Build it with the reference's own include directory (src/) ahead of this
 * one and link libgrlbm.so together with the reference's sources:
 *     g++ -std=c++20 -I<reference>/src -Iinclude app.cpp <reference>/src/*.cpp \
 *         -L2dradiation_b200 -lgrlbm
 *
 * Radiation's methods are not virtual, so a RadiationB200 must never be used
 * through a Radiation reference: that would run the reference's CPU methods
 * on buffers this class does not keep current.  The inheritance is private
 * for that reason -- binding a RadiationB200 to a Radiation& does not compile
 * -- and the reference's public data members and helpers are re-exported by
 * name.
 *
 * Supported: the metrics Minkowski, SchwarzSchild and KerrSchild (derived
 * classes of them count as their base), intensity stencils Stencil(n, 0) and
 * streaming stencils Stencil(n, 0, false), all five streaming types except
 * GeodesicFixed.  Anything else throws std::runtime_error from the
 * constructor, as does a failed grlbm_create (no GPU, for instance). */
#pragma once

#include "Radiation.h"
#include "Spacetimes.h"
#include "grlbm.h"

#include <cmath>
#include <stdexcept>
#include <string>

class RadiationB200 : private Radiation
{
public:
    // The reference's public members (src/Radiation.h:20-84).
    using Radiation::averageItterationCount;
    using Radiation::coefficientsCx;
    using Radiation::coefficientsCy;
    using Radiation::coefficientsS;
    using Radiation::coefficientsX;
    using Radiation::coefficientsY;
    using Radiation::config;
    using Radiation::E;
    using Radiation::E_LF;
    using Radiation::eta;
    using Radiation::F_LF;
    using Radiation::Fx;
    using Radiation::Fx_LF;
    using Radiation::Fy;
    using Radiation::Fy_LF;
    using Radiation::grid;
    using Radiation::HarmonicIndex;
    using Radiation::I;
    using Radiation::Index;
    using Radiation::initialE_LF;
    using Radiation::initialFluxAngle_IF;
    using Radiation::initialFx_LF;
    using Radiation::initialFy_LF;
    using Radiation::initialI;
    using Radiation::initialPxx_LF;
    using Radiation::initialPxy_LF;
    using Radiation::initialPyy_LF;
    using Radiation::isInitialGridPoint;
    using Radiation::kappa0;
    using Radiation::kappa1;
    using Radiation::kappaA;
    using Radiation::logger;
    using Radiation::maxItterationCount;
    using Radiation::metric;
    using Radiation::Pxx;
    using Radiation::Pxx_LF;
    using Radiation::Pxy;
    using Radiation::Pxy_LF;
    using Radiation::Pyy;
    using Radiation::Pyy_LF;
    using Radiation::stencil;
    using Radiation::streamingStencil;
    using Radiation::ux;
    using Radiation::uy;

    // precision: GRLBM_PLAIN_FP64 (the reference's arithmetic),
    // GRLBM_PRECISION_FP32 or GRLBM_FAST_FP64; device < 0 selects the current
    // CUDA device.
    RadiationB200(Metric &metric, Stencil &stencil, Stencil &streamingStencil, Config config,
                  int precision = GRLBM_PLAIN_FP64, int device = -1)
        : Radiation(metric, stencil, streamingStencil, config)
    {
        if (stencil.nGhost != 0 || streamingStencil.nGhost != 0)
            throw std::runtime_error("RadiationB200: stencils with ghost directions are not supported");
        if (config.streamingType == StreamingType::GeodesicFixed)
            throw std::runtime_error("RadiationB200: GeodesicFixed streaming is not supported");
        Grid &g = metric.grid;
        // Grid(nx_, ny_, start, end) keeps one halo cell on each side
        // (src/Grid.cpp:13-22); the descriptor takes the caller's values,
        // recovered so that the library's grid is this one bit for bit.
        double sx, ex, sy, ey;
        if (!RecoverInterval(g.startx, g.endx, g.dx, (int64_t)g.nx - 2, sx, ex) ||
            !RecoverInterval(g.starty, g.endy, g.dy, (int64_t)g.ny - 2, sy, ey))
            throw std::runtime_error("RadiationB200: the grid's start and end cannot be recovered exactly");
        const grlbm_grid_desc gd{(int64_t)g.nx - 2, (int64_t)g.ny - 2, sx, sy, ex, ey, g.GetCFL()};
        const grlbm_metric_desc md{MetricKind(metric), metric.m, metric.a, 0.0};
        const grlbm_run_desc rd{(int32_t)stencil.nDir,
                                (int32_t)streamingStencil.nDir,
                                (int32_t)config.streamingType,
                                (int32_t)precision,
                                config.keepSourceNodesActive ? 1 : 0,
                                (int32_t)config.initialDataType};
        Check(grlbm_create(&gd, &md, &rd, device, &ctx_), nullptr);
    }
    ~RadiationB200() { grlbm_destroy(ctx_); }
    RadiationB200(const RadiationB200 &) = delete;
    RadiationB200 &operator=(const RadiationB200 &) = delete;

    // Radiation::LoadInitialData (src/Radiation.cpp:128-182): uploads the
    // fluid fields and initial data the caller wrote, then sets the source
    // intensities on the GPU.
    void LoadInitialData()
    {
        const bool adaptive = config.streamingType == StreamingType::FlatAdaptive ||
                              config.streamingType == StreamingType::CurvedAdaptive;
        Check(grlbm_set_fields(ctx_, kappa0.data(), kappa1.data(), kappaA.data(), eta.data(), ux.data(), uy.data()));
        if (adaptive)
            Check(grlbm_set_initial_flux_angle(ctx_, initialFluxAngle_IF.data()));
        static_assert(sizeof(bool) == sizeof(uint8_t), "isInitialGridPoint is passed as bytes");
        Check(grlbm_set_initial_data(ctx_, reinterpret_cast<const uint8_t *>(isInitialGridPoint), initialI.data(),
                                     initialE_LF.data(), initialFx_LF.data(), initialFy_LF.data(),
                                     initialPxx_LF.data(), initialPxy_LF.data(), initialPyy_LF.data()));
        Check(grlbm_load_initial_data(ctx_));
    }

    // Radiation::UpdateFourierCoefficients (src/Radiation.cpp:191-237) with
    // the reference's RK45 tolerance; the coefficient buffers are read back.
    void UpdateFourierCoefficients()
    {
        Check(grlbm_update_fourier_coefficients(ctx_, 1e-4, 0));
        Check(grlbm_get_fourier_coefficients(ctx_, coefficientsS.data(), coefficientsX.data(), coefficientsY.data(),
                                             coefficientsCx.data(), coefficientsCy.data()));
    }

    // Radiation::ComputeMomentsIF / ComputeMomentsLF (src/Radiation.cpp:
    // 239-301): the inertial-frame moments of the last step, and the
    // lab-frame moments derived from them.
    void ComputeMomentsIF()
    {
        Check(grlbm_get_moments_if(ctx_, E.data(), Fx.data(), Fy.data(), Pxx.data(), Pxy.data(), Pyy.data()));
    }
    void ComputeMomentsLF()
    {
        Check(grlbm_compute_moments_lf(ctx_, E_LF.data(), Fx_LF.data(), Fy_LF.data(), Pxx_LF.data(), Pxy_LF.data(),
                                       Pyy_LF.data(), F_LF.data()));
    }

    // n iterations of RunSimulation's loop body (src/Radiation.cpp:789-822);
    // I and the moment buffers are not refreshed (see SyncIntensity).
    void Step(int n) { Check(grlbm_step(ctx_, n)); }
    // Copies the current intensities into I.
    void SyncIntensity() { Check(grlbm_get_intensity(ctx_, I.data())); }

    // Radiation::RunSimulation (src/Radiation.cpp:735-884) without its
    // console output: set-up, the time loop with its frames under
    // config.writeData, the profile session's trace and Log.txt, then the
    // iteration counts, I, the inertial-frame moments and (when frames were
    // written) the lab-frame moments in the public buffers, as the
    // reference leaves them.
    void RunSimulation()
    {
        Check(grlbm_trace_begin(ctx_, ("output/" + config.name + "/profileResults.json").c_str()));
        int rc = GRLBM_OK;
        std::string out;
        try
        {
            LoadInitialData();
            UpdateFourierCoefficients();
            const int time_steps = (int)std::ceil(config.simTime / grid.dt);
            config.simTime = time_steps * grid.dt;
            logger.SetValues(config.name, config.simTime);
            out = logger.directoryPath;
            const std::string frames = out + "/Moments/";
            int64_t steps = 0;
            rc = grlbm_run_simulation(ctx_, config.t0, config.simTime, config.writePeriod,
                                      config.saveInitialData ? 1 : 0, config.writeData ? frames.c_str() : nullptr,
                                      &steps);
            if (rc == GRLBM_OK && steps != logger.timeSteps)
                throw std::runtime_error("RadiationB200: the library ran " + std::to_string(steps) +
                                         " steps, the reference's loop " + std::to_string(logger.timeSteps));
        }
        catch (...)
        {
            grlbm_trace_end(ctx_); // the session closes whatever failed
            throw;
        }
        Check(grlbm_trace_end(ctx_));
        Check(rc);
        grlbm_stats st{};
        Check(grlbm_get_stats(ctx_, &st));
        maxItterationCount = st.max_iterations;
        averageItterationCount = st.average_iterations;
        logger.maxItterationCount = maxItterationCount;
        logger.averageItterationCount = averageItterationCount;
        SyncIntensity();
        ComputeMomentsIF();
        if (config.writeData)
        {
            ComputeMomentsLF();
            Check(grlbm_write_log(ctx_, out.c_str()));
        }
    }

    grlbm_ctx *Context() { return ctx_; }

private:
    grlbm_ctx *ctx_ = nullptr;

    void Check(int rc) { Check(rc, ctx_); }
    // The start and end a Grid was built from, given its startx = start - d,
    // endx = end + d and d = (end - start) / (n_ - 1) (src/Grid.cpp:16-22):
    // start = startx + d to within rounding, searched over a few ulps for
    // the values that give back the grid's own startx, endx and d exactly.
    static bool RecoverInterval(double lo, double hi, double d, int64_t n_, double &start, double &end)
    {
        auto nudge = [](double x, int k) {
            for (int u = 0; u < (k < 0 ? -k : k); u++)
                x = std::nextafter(x, k < 0 ? -INFINITY : INFINITY);
            return x;
        };
        for (int i = -4; i <= 4; i++)
            for (int k = -4; k <= 4; k++)
            {
                const double s = nudge(lo + d, i), e = nudge(hi - d, k);
                const double dd = (e - s) / ((double)(n_ + 2) - 1.0 - 2.0);
                if (dd == d && s - dd == lo && e + dd == hi)
                {
                    start = s, end = e;
                    return true;
                }
            }
        return false;
    }
    static void Check(int rc, grlbm_ctx *c)
    {
        if (rc != GRLBM_OK)
            throw std::runtime_error(std::string("libgrlbm: ") + grlbm_last_error(c));
    }
    // The metric classes of src/Spacetimes.h; an unknown Metric subclass is
    // refused rather than guessed.
    static int32_t MetricKind(Metric &m)
    {
        if (dynamic_cast<KerrSchild *>(&m))
            return GRLBM_KERRSCHILD;
        if (dynamic_cast<SchwarzSchild *>(&m))
            return GRLBM_SCHWARZSCHILD;
        if (dynamic_cast<Minkowski *>(&m))
            return GRLBM_MINKOWSKI;
        throw std::runtime_error("RadiationB200: metric " + m.Name() + " is not Minkowski, SchwarzSchild or KerrSchild");
    }
};
