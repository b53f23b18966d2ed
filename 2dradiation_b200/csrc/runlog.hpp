// The run's log file and profile trace in the reference's formats (see
// runlog.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "host_setup.hpp"

namespace grlbm
{
// What Logger::Write reports about a run (src/Logger.hh:48-97): the creation
// date (Logger::SetValues' "%H.%M.%S - %d.%m.%Y"), the time steps and
// simulated time, the lambda-iteration statistics and the named time
// measurements in seconds ("Total Time" and the frame writer's name among
// them: the computation time is the first minus the second).
struct RunLog
{
    std::string date;
    int64_t time_steps = 0;
    double sim_time = 0;
    int32_t max_iterations = 0;
    double average_iterations = 0;
    std::vector<std::pair<std::string, double>> times;
    bool valid = false;
};

// The profiler's name of Grid::WriteFrametoCsv (the frame writer), which
// ComputationTime subtracts from "Total Time" (src/Logger.hh:117-126).
extern const char *const kFrameWriterName;

// Logger::SetValues' creation date of the current local time.
std::string log_date_now();

// Metric::Name of the metric kinds (src/Spacetimes.cpp:16-85).
const char *metric_name(int kind);

// Writes directory + "/Log.txt" in Logger::Write's format (creating the
// directory); the stencil properties come from the stencils' tables.
bool write_log_txt(const std::string &directory, const GridGeom &G, int metric_kind, double m, double a,
                   const StencilTables &intensity, const StencilTables &streaming, const RunLog &log,
                   std::string &err);

// One event of a profile session (Profiler.hh's Result): microseconds since
// the steady clock's epoch, and the thread's id hash.
struct TraceEvent
{
    std::string name;
    long long start_us = 0, end_us = 0;
    uint32_t thread_id = 0;
};

long long trace_now_us();
uint32_t trace_thread_id();

// Writes a session's events in the profiler's Chrome-trace JSON
// (src/Profiler.hh:104-141).
bool write_trace_json(const std::string &path, const std::vector<TraceEvent> &events, std::string &err);
} // namespace grlbm
