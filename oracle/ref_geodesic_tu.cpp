// Compiles the reference's own src/GeodesicEquationSolver.cpp unchanged, with
// one preprocessor definition: `constexpr` expands to nothing inside that file
// only (every header it includes is pulled in first, so their include guards
// keep them untouched).  Its file-scope `constexpr double maxTE = 1e-4;`
// (src/GeodesicEquationSolver.cpp:79) thereby becomes an assignable global,
// which oracle/ref_driver.cpp sets to the run's RK45 tolerance.
// Test infrastructure only (see oracle/Makefile).
#include "Radiation.h"
#define constexpr
#include "GeodesicEquationSolver.cpp"
#undef constexpr
