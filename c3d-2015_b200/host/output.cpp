// Output files of the reference (src/output.cpp:19-110): the text master file and the
// binary .pn data file of one rank, plus a checkpoint of (u, alpha) that the reference
// does not have. Formats are the reference's, byte for byte, so its readers (plot.py)
// work unchanged.
#include "output.h"

#include <cstdint>
#include <cstdio>

namespace c3d_host {

static bool put_i64(FILE *f, long long v)
{
    int64_t t = (int64_t)v;
    return fwrite(&t, sizeof(t), 1, f) == 1;
}
static bool put_f64(FILE *f, double v) { return fwrite(&v, sizeof(v), 1, f) == 1; }

bool write_output_data(const std::string &dir, double time, const Config &c, int nm,
                       const double *u, const OutputStats &st, std::string &err)
{
    char name[512];
    // master file (rank 0; one rank here)
    snprintf(name, sizeof(name), "%s/out_%.6f.master", dir.c_str(), time);
    FILE *f = fopen(name, "w");
    if (!f) {
        err = std::string("could not open ") + name;
        return false;
    }
    fprintf(f, "%d\n%d\n%d\n", c.nx, c.ny, c.nz);
    fprintf(f, "%f\n%f\n%f\n%f\n%f\n%f\n", c.ax, c.ay, c.az, c.bx, c.by, c.bz);
    fprintf(f, "%d\n", nm);
    fprintf(f, "1\n1\n1\n");
    fprintf(f, "out_%.6f_%d.pn\n", time, 0);
    fclose(f);

    // data file: nx ny nz, the interior moments (i, j, k with k fastest), closure statistics
    snprintf(name, sizeof(name), "%s/out_%.6f_%d.pn", dir.c_str(), time, 0);
    f = fopen(name, "wb");
    if (!f) {
        err = std::string("could not open ") + name;
        return false;
    }
    bool ok = put_i64(f, c.nx) && put_i64(f, c.ny) && put_i64(f, c.nz);
    const long long nyg = c.ny + 4, nzg = c.nz + 4;
    for (int i = 2; ok && i < c.nx + 2; ++i)
        for (int j = 2; ok && j < c.ny + 2; ++j)
            for (int k = 2; ok && k < c.nz + 2; ++k) {
                const long long cell = k + nzg * (j + nyg * (long long)i);
                ok = fwrite(u + cell * nm, sizeof(double), (size_t)nm, f) == (size_t)nm;
            }
    ok = ok && put_i64(f, st.maxIter) && put_i64(f, st.maxIterGamma) &&
         put_f64(f, st.iterMean) && put_f64(f, st.iterGammaMean) && put_i64(f, st.numDualSolves);
    for (size_t r = 0; ok && r < st.regHist.size(); ++r)
        ok = put_i64(f, st.regHist[r]);
    fclose(f);
    if (!ok)
        err = std::string("write failed: ") + name;
    return ok;
}

bool write_timings(const std::string &dir, int numUpdates, const std::vector<double> &times,
                   std::string &err)
{
    char name[512];
    snprintf(name, sizeof(name), "%s/times.master", dir.c_str());
    FILE *f = fopen(name, "w");
    if (!f) {
        err = std::string("could not open ") + name;
        return false;
    }
    fprintf(f, "%d\n1\n1\n1\ntimes_%d.dat\n", numUpdates, 0);
    fclose(f);
    snprintf(name, sizeof(name), "%s/times_%d.dat", dir.c_str(), 0);
    f = fopen(name, "wb");
    if (!f) {
        err = std::string("could not open ") + name;
        return false;
    }
    const size_t n = (size_t)numUpdates * 8;
    bool ok = n <= times.size() && fwrite(times.data(), sizeof(double), n, f) == n;
    fclose(f);
    if (!ok)
        err = std::string("write failed: ") + name;
    return ok;
}

bool write_opt_stats(const std::string &dir, int numUpdates, int nx, const std::vector<double> &log,
                     std::string &err)
{
    char name[512];
    snprintf(name, sizeof(name), "%s/stats_%d.dat", dir.c_str(), 0);
    FILE *f = fopen(name, "wb");
    if (!f) {
        err = std::string("could not open ") + name;
        return false;
    }
    bool ok = put_i64(f, numUpdates) && put_i64(f, nx);
    const size_t recs = (size_t)numUpdates * 2 * nx;
    for (size_t k = 0; ok && k < recs; ++k) {
        const double *r = log.data() + 5 * k;
        const bool have = 5 * k + 5 <= log.size();
        ok = put_f64(f, have ? r[0] : 0.0) && put_i64(f, have ? (long long)r[1] : 0) &&
             put_i64(f, have ? (long long)r[2] : 0) && put_f64(f, have ? r[3] : 0.0) &&
             put_f64(f, have ? r[4] : 0.0);
    }
    fclose(f);
    if (!ok)
        err = std::string("write failed: ") + name;
    return ok;
}

static const char CKPT_MAGIC[8] = {'C', '3', 'D', 'C', 'K', 'P', 'T', '1'};

bool write_checkpoint(const std::string &path, double time, const Config &c, int nm,
                      const double *u, const double *alpha, std::string &err)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) {
        err = "could not open " + path;
        return false;
    }
    const size_t n = (size_t)(c.nx + 4) * (c.ny + 4) * (c.nz + 4) * nm;
    bool ok = fwrite(CKPT_MAGIC, 1, 8, f) == 8 && put_i64(f, c.nx) && put_i64(f, c.ny) &&
              put_i64(f, c.nz) && put_i64(f, nm) && put_f64(f, time) &&
              fwrite(u, sizeof(double), n, f) == n && fwrite(alpha, sizeof(double), n, f) == n;
    fclose(f);
    if (!ok)
        err = "write failed: " + path;
    return ok;
}

bool read_checkpoint(const std::string &path, const Config &c, int nm, double *u, double *alpha,
                     double *time, std::string &err)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) {
        err = "could not open " + path;
        return false;
    }
    char magic[8];
    int64_t hdr[4];
    double t = 0.0;
    bool ok = fread(magic, 1, 8, f) == 8 && fread(hdr, sizeof(int64_t), 4, f) == 4 &&
              fread(&t, sizeof(double), 1, f) == 1;
    if (ok && (std::string(magic, 8) != std::string(CKPT_MAGIC, 8) || hdr[0] != c.nx ||
               hdr[1] != c.ny || hdr[2] != c.nz || hdr[3] != nm)) {
        err = "checkpoint " + path + " does not match this problem";
        fclose(f);
        return false;
    }
    const size_t n = (size_t)(c.nx + 4) * (c.ny + 4) * (c.nz + 4) * nm;
    ok = ok && fread(u, sizeof(double), n, f) == n && fread(alpha, sizeof(double), n, f) == n;
    fclose(f);
    if (!ok) {
        err = "read failed: " + path;
        return false;
    }
    if (time)
        *time = t;
    return true;
}

} // namespace c3d_host
