// The run's log file (Logger::Write, src/Logger.hh:48-97) and profile trace
// (Profiler::Session's Chrome-trace JSON, src/Profiler.hh:104-141) in the
// reference's formats, so that tools reading the reference's output files
// read these too.  Numbers are written with the iostream defaults the
// reference uses.
#include "runlog.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <sstream>

namespace grlbm
{
const char *const kFrameWriterName = "void Grid::WriteFrametoCsv(float, const DoubleBuffer&, const DoubleBuffer&, "
                                     "const DoubleBuffer&, const DoubleBuffer&, std::string, std::string)";

std::string log_date_now()
{
    const std::time_t t = std::time(nullptr);
    std::tm tm{};
    localtime_r(&t, &tm);
    std::ostringstream oss;
    oss << std::put_time(&tm, "%H.%M.%S - %d.%m.%Y");
    return oss.str();
}

const char *metric_name(int kind)
{
    switch (kind)
    {
    case 0:
        return "Minkowski";
    case 1:
        return "SchwarzSchild";
    case 2:
        return "KerrSchild";
    default:
        return "";
    }
}

namespace
{
// mkdir -p of the directory part of a path
bool make_dirs(const std::string &dir, std::string &err)
{
    std::string cur;
    for (size_t k = 0; k <= dir.size(); k++)
    {
        if (k == dir.size() || dir[k] == '/')
        {
            if (!cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
            {
                err = "cannot create directory " + cur + ": " + std::strerror(errno);
                return false;
            }
        }
        if (k < dir.size())
            cur += dir[k];
    }
    return true;
}

double time_of(const RunLog &log, const char *name)
{
    for (const auto &t : log.times)
        if (t.first == name)
            return t.second;
    return 0.0;
}
} // namespace

bool write_log_txt(const std::string &directory, const GridGeom &G, int metric_kind, double m, double a,
                   const StencilTables &intensity, const StencilTables &streaming, const RunLog &log,
                   std::string &err)
{
    if (!make_dirs(directory, err))
        return false;
    const std::string path = directory + "/Log.txt";
    std::ofstream file(path);
    if (!file)
    {
        err = "cannot open " + path;
        return false;
    }
    file << "Creation Date: " << log.date << std::endl << std::endl;

    file << "Spacetime: " << metric_name(metric_kind) << std::endl;
    file << "Black Hole  Mass,   M = " << m << std::endl;
    file << "Black Hole  Spin,   a = " << a << std::endl << std::endl;

    file << "Grid Structure:" << std::endl;
    file << "Simulation Time = " << log.sim_time << std::endl;
    file << "(startx,starty) = (" << G.startx << "," << G.starty << ")" << std::endl;
    file << "(endx  ,  endy) = (" << G.endx << "," << G.endy << ")" << std::endl;
    file << "(Nx    ,    Ny) = (" << G.nx << "," << G.ny << ")" << std::endl;
    file << "Nt         = " << log.time_steps << std::endl;
    file << "dx         = " << G.dx << std::endl;
    file << "dy         = " << G.dy << std::endl;
    file << "dt         = " << G.dt << std::endl;
    file << "cfl        = " << G.cfl << std::endl << std::endl;

    // Stencil(n, 0): nDir = nOrder = nCoefficients = n; the flux table's last
    // entries are sigmaMax and relativeFluxMax (src/Stencil.cpp:177-297)
    const double sigma_max = intensity.lut_sigma.empty() ? 0.0 : intensity.lut_sigma.back();
    const double flux_max = intensity.lut_in.empty() ? 0.0 : intensity.lut_in.back();
    const double max_interpolation_error = 0.01; // Stencil::maxInterpolationError (src/Stencil.h:64)
    file << "Stencil Properties:" << std::endl;
    file << "Intensity Stencil: nDir          = " << intensity.n << std::endl;
    file << "Intensity Stencil: nOrder        = " << intensity.n << std::endl;
    file << "Intensity Stencil: nCoefficients = " << intensity.n << std::endl;
    file << "Intensity Stencil: max Interpolation Error = " << 100 * max_interpolation_error << "%" << std::endl;
    file << "Intensity Stencil: sigma max               = " << sigma_max << std::endl;
    file << "Intensity Stencil: relative flux max       = " << flux_max << std::endl;
    file << "Streaming Stencil: nDir          = " << streaming.n << std::endl;
    file << "Streaming Stencil: nOrder        = " << streaming.n << std::endl;
    file << "Streaming Stencil: nCoefficients = " << streaming.n << std::endl << std::endl;

    file << "Lambda Itteration:" << std::endl;
    file << "Max Lambda Itteration Count     = " << log.max_iterations << std::endl;
    file << "Average Lambda Itteration Count = " << log.average_iterations << std::endl << std::endl;

    file << "Time measurements:" << std::endl;
    for (const auto &t : log.times)
        file << t.first << ": " << t.second << "s" << std::endl;
    const double computation = time_of(log, "Total Time") - time_of(log, kFrameWriterName);
    file << "Computation Time: " << computation << "s" << std::endl;
    file << "Benchmark: " << G.nxy * log.time_steps / (1e6 * computation) << " MLUPS" << std::endl;
    if (!file)
    {
        err = "writing " + path + " failed";
        return false;
    }
    return true;
}

long long trace_now_us()
{
    // the profiler's clock and unit (src/Profiler.hh:28-56)
    return std::chrono::time_point_cast<std::chrono::microseconds>(std::chrono::high_resolution_clock::now())
        .time_since_epoch()
        .count();
}

// The profiler records omp_get_thread_num(), 0 on the thread that calls the
// library outside parallel regions.
uint32_t trace_thread_id() { return 0u; }

bool write_trace_json(const std::string &path, const std::vector<TraceEvent> &events, std::string &err)
{
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && !make_dirs(path.substr(0, slash), err))
        return false;
    std::ofstream out(path);
    if (!out)
    {
        err = "cannot open " + path;
        return false;
    }
    out << "{\n";
    out << "\t\"otherData\": {},\n";
    out << "\t\"traceEvents\":\n";
    out << "\t[\n";
    for (size_t k = 0; k < events.size(); k++)
    {
        const TraceEvent &e = events[k];
        if (k > 0)
            out << ",\n";
        std::string name = e.name;
        std::replace(name.begin(), name.end(), '"', '\'');
        out << "\t\t{\n";
        out << "\t\t\t\"cat\":\"function\",\n";
        out << "\t\t\t\"dur\":" << (e.end_us - e.start_us) << ",\n";
        out << "\t\t\t\"name\":\"" << name << "\",\n";
        out << "\t\t\t\"ph\":\"X\",\n";
        out << "\t\t\t\"pid\":0,\n";
        out << "\t\t\t\"tid\":" << e.thread_id << ",\n";
        out << "\t\t\t\"ts\":" << e.start_us << "\n";
        out << "\t\t}";
    }
    out << "\n\t]\n";
    out << "}";
    out.flush();
    if (!out)
    {
        err = "writing " + path + " failed";
        return false;
    }
    return true;
}
} // namespace grlbm
