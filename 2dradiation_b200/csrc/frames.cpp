// Frame output of the radiation step in the reference's CSV format
// (src/Grid.cpp:110-137) and its number formatting (src/Utility.hh:511-541),
// so that files written here and by the reference for the same data are
// byte-identical.
#include "frames.hpp"

#include <cmath>
#include <filesystem>
#include <fstream>
#include <sstream>

namespace grlbm
{
std::string format_fixed(double n, int precision)
{
    // a leading space for non-negative values (none for -0), then fixed
    // notation with `precision` decimals (Format with its default flags)
    std::string out;
    if (n == 0)
        out = std::signbit(n) ? "" : " ";
    else
        out = n >= 0 ? " " : "";
    std::ostringstream ss;
    ss.precision(precision);
    ss << std::fixed << n;
    return out + ss.str();
}

bool write_frame_csv(const GridGeom &G, float time, const double *r, const double *g, const double *b,
                     const double *a, const std::string &directory, const std::string &name, std::string &err)
{
    std::error_code ec;
    if (!directory.empty())
        std::filesystem::create_directories(directory, ec);
    const std::string stem = name.empty() ? "data" : name;
    const std::string path = directory + stem + format_fixed(time, 3) + "t " + std::to_string(G.nx) + "x " +
                             std::to_string(G.ny) + "y" + ".csv";
    std::ofstream out(path);
    if (!out)
    {
        err = "cannot open " + path;
        return false;
    }
    out << "#nx=" << G.nx << "\n";
    out << "#ny=" << G.ny << "\n";
    out << "#startx=" << G.startx << "\n";
    out << "#starty=" << G.starty << "\n";
    out << "#endx=" << G.endx << "\n";
    out << "#endy=" << G.endy << "\n";
    out << "#t=" << time << "\n";
    out << "#x,y,r,g,b,a\n";
    for (int64_t j = 0; j < G.ny; j++)
        for (int64_t i = 0; i < G.nx; i++)
        {
            const int64_t ij = i + j * G.nx;
            out << G.x((double)i) << "," << G.y((double)j) << ",";
            out << r[ij] << "," << g[ij] << "," << b[ij] << "," << a[ij] << "\n";
        }
    out.close();
    if (!out)
    {
        err = "cannot write " + path;
        return false;
    }
    return true;
}
} // namespace grlbm
