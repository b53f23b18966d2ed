// Frame output in the reference's CSV format (see frames.cpp).
#pragma once
#include <string>

#include "host_setup.hpp"

namespace grlbm
{
// Format(n, precision) of src/Utility.hh:511-541 with its default flags.
std::string format_fixed(double n, int precision);
// Grid::WriteFrametoCsv (src/Grid.cpp:110-137): the file
// directory + name + Format(time, 3) + "t " + nx + "x " + ny + "y.csv" with the
// node coordinates and four per-node arrays (nx * ny each); the directory is
// created if needed.
bool write_frame_csv(const GridGeom &G, float time, const double *r, const double *g, const double *b,
                     const double *a, const std::string &directory, const std::string &name, std::string &err);
} // namespace grlbm
