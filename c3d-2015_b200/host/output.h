// Output files of the reference (src/output.cpp:19-110) and a checkpoint of (u, alpha).
#pragma once
#include "solver.h"

#include <string>
#include <vector>

namespace c3d_host {

// The reference's closure statistics as outputData writes them (src/output.cpp:98-105;
// accumulated in src/update.cpp:79-97, 156-176).
struct OutputStats {
    long long maxIter = 0, maxIterGamma = 0, numDualSolves = 0;
    double iterMean = 0.0, iterGammaMean = 0.0;
    std::vector<long long> regHist; // NUM_REGULARIZATIONS entries
};

// <dir>/out_<time>.master and <dir>/out_<time>_0.pn; u holds all cells (ghosts included).
bool write_output_data(const std::string &dir, double time, const Config &c, int nm,
                       const double *u, const OutputStats &st, std::string &err);

// outputTimings (src/output.cpp:116-178): <dir>/times.master and <dir>/times_0.dat with 8
// seconds per update (per RK stage: ghost fill, closure, flux, Euler; src/update.cpp:217-262).
bool write_timings(const std::string &dir, int numUpdates, const std::vector<double> &times,
                   std::string &err);

// outputOptStats (src/output.cpp:184-222): <dir>/stats_0.dat, int64 numUpdates, int64 nx, then
// per closure (2 per update) and x-line cell the record {double r; int64 iter; int64 iterGamma;
// double gamma; double normG} (OPTIMIZATION_STATS, src/global.h:53-60). log holds 5 doubles
// per record in that order.
bool write_opt_stats(const std::string &dir, int numUpdates, int nx, const std::vector<double> &log,
                     std::string &err);

// Checkpoint: "C3DCKPT1", int64 nx ny nz nm, double time, u and alpha of all cells.
bool write_checkpoint(const std::string &path, double time, const Config &c, int nm,
                      const double *u, const double *alpha, std::string &err);
bool read_checkpoint(const std::string &path, const Config &c, int nm, double *u, double *alpha,
                     double *time, std::string &err);

} // namespace c3d_host
