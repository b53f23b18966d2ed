/* Shared parameter block for the two CPU checkers in oracle/:
 *   - oracle_run()  in grlbm_oracle.c   (the C restatement, liboracle.so)
 *   - ref_run()     in ref_driver.cpp   (the reference itself, compiled from
 *                                        its own sources into oracle/_ref/)
 * Both take the same inputs and fill the same outputs so that the tests can
 * compare them field by field.  This header is test infrastructure only.
 *
 * Array conventions follow the reference (src/Radiation.h:28-79):
 *   per-node arrays have nx*ny entries, ij = i + j*nx (src/Grid.cpp:44-47),
 *   where nx = nx_ + 2*halo (src/Grid.cpp:14);
 *   intensities are cell-major: I[ij*nDir + d] (src/Radiation.cpp:89-92);
 *   Fourier coefficients are [ij*nF + k] (src/Radiation.cpp:98-101). */
#ifndef GRLBM_ORACLE_REF_API_H
#define GRLBM_ORACLE_REF_API_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* number of per-node metric arrays exchanged (order: see metric_names in
 * oracle/oracle.py; it follows the member order of src/Metric.h:19-65) */
#define GRLBM_N_METRIC_ARRAYS 102

typedef struct
{
    /* Grid(nx_, ny_, start, end, halo=1) + SetCFL (src/Grid.cpp:4-37) */
    int64_t nx_, ny_;
    double startx, starty, endx, endy, cfl;
    /* metric: 0 Minkowski, 1 SchwarzSchild, 2 KerrSchild (src/Spacetimes.h) */
    int32_t metric_kind;
    double m, a;
    /* excision radius in units of m; <= 0 keeps the reference value 2.1
     * (src/Spacetimes.cpp:42,81) */
    double excision;
    /* Stencil(nOrder=n_dir, 0) and Stencil(n_fourier, 0, false) */
    int32_t n_dir, n_fourier;
    /* StreamingType: 0 FlatFixed, 2 CurvedFixed (src/Config.hh:5-12) */
    int32_t streaming_type;
    /* InitialDataType: 0 Moments, 1 Intensities (src/Config.hh:38-42) */
    int32_t initial_data_type;
    int32_t keep_source_nodes_active;
    int32_t n_steps;
    /* RK45 truncation-error tolerance (reference: maxTE = 1e-4,
     * src/GeodesicEquationSolver.cpp:79) */
    double rk_tol;
    /* 0: explicit step loop (mirrors src/Radiation.cpp:745-832 without I/O);
     * 1: call Radiation::RunSimulation() itself (timing arm) */
    int32_t use_run_simulation;
    /* OpenMP threads (0 = leave default) */
    int32_t n_threads;
    /* Config::updateFourierHarmonics (src/Config.hh:51): rebuild the geodesic
     * tables at the top of every step (reference driver only) */
    int32_t update_tables_each_step;
} grlbm_ref_params;

typedef struct
{
    /* per-node fluid fields (nx*ny each) */
    const double *kappa0, *kappa1, *kappaA, *eta, *ux, *uy;
    /* initial data */
    const uint8_t *is_initial; /* nx*ny */
    const double *initial_I;   /* nx*ny*nDir, cell-major */
    const double *initial_E_LF, *initial_Fx_LF, *initial_Fy_LF;
    const double *initial_Pxx_LF, *initial_Pxy_LF, *initial_Pyy_LF;
    /* optional: replaces the metric arrays after construction (NULL: keep the
     * ones the metric class computed); GRLBM_N_METRIC_ARRAYS * nx*ny */
    const double *metric_override;
} grlbm_ref_inputs;

typedef struct
{
    /* inertial-frame moments as left by the last step (nx*ny each) */
    double *E, *Fx, *Fy, *Pxx, *Pxy, *Pyy;
    /* lab-frame moments: ComputeMomentsLF() after the last step (nx*ny) */
    double *E_LF, *Fx_LF, *Fy_LF, *Pxx_LF, *Pxy_LF, *Pyy_LF, *F_LF;
    /* final intensities, cell-major (nx*ny*nDir) */
    double *I;
    /* Fourier coefficients of the geodesic tables (nx*ny*nF each) */
    double *coefS, *coefX, *coefY, *coefCx, *coefCy;
    /* the metric arrays as computed by the metric class (before override) */
    double *metric_arrays; /* GRLBM_N_METRIC_ARRAYS * nx*ny, may be NULL */
    /* stencil tables: w, phi, cx, cy (nDir each) */
    double *st_w, *st_phi, *st_cx, *st_cy;
    /* interpolation grid: nGrid = 10*nDir rows of 4 indices and 4 weights */
    int64_t *ig_index;
    double *ig_weight;
    /* streaming stencil phi, w (nF each) */
    double *ss_phi, *ss_w;
    /* lambda-iteration statistics and timing */
    int32_t max_iterations;
    double average_iterations;
    double computation_time_s; /* the step loop only (Logger::ComputationTime) */
    double table_time_s;       /* UpdateFourierCoefficients */
    /* optional: wall time of each step of the loop (n_steps entries) */
    double *step_times;
} grlbm_ref_outputs;

int ref_run(const grlbm_ref_params *p, const grlbm_ref_inputs *in, grlbm_ref_outputs *out);
int oracle_run(const grlbm_ref_params *p, const grlbm_ref_inputs *in, grlbm_ref_outputs *out);

#ifdef __cplusplus
}
#endif
#endif
