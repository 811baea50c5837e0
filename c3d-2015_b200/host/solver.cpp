#include "solver.h"
#include "output.h"
#include "../../include/c3d_solver.h"

#include "tables.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <sstream>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace c3d_host {

#define REQUIRE(call, name)                                                                        \
    if (!(call))                                                                                   \
        return std::string("missing or invalid deck key ") + name;

std::string parse_config(const InputDeck &d, Config &c)
{
    REQUIRE(d.get("SOLVER", c.solver), "SOLVER");
    REQUIRE(d.get("TFINAL", c.tFinal), "TFINAL");
    REQUIRE(d.get("OUTDT", c.outDt), "OUTDT");
    REQUIRE(d.get("OUTPUT_DATA", c.outputData), "OUTPUT_DATA");
    REQUIRE(d.get("OUTPUT_OPT_STATS", c.outputOptStats), "OUTPUT_OPT_STATS");
    REQUIRE(d.get("OUTPUT_TIMINGS", c.outputTimings), "OUTPUT_TIMINGS");
    REQUIRE(d.get("MOMENT_ORDER", c.momentOrder), "MOMENT_ORDER");
    REQUIRE(d.get("QUAD_ORDER", c.quadOrder), "QUAD_ORDER");
    REQUIRE(d.get("CFL_FACTOR", c.cfl), "CFL_FACTOR");
    REQUIRE(d.get("CROSS_SECTION", c.crossSection), "CROSS_SECTION");
    REQUIRE(d.get("INIT_FLOOR", c.initFloor), "INIT_FLOOR");
    REQUIRE(d.get("GAUSS_SIGMA", c.gaussSigma), "GAUSS_SIGMA");
    REQUIRE(d.get("INIT_COND", c.initCond), "INIT_COND");
    REQUIRE(d.get("OMP_THREADS", c.ompThreads), "OMP_THREADS");
    REQUIRE(d.get("CUDA_KINETIC", c.cudaKinetic), "CUDA_KINETIC");
    REQUIRE(d.get("CUDA_BATCHED", c.cudaBatched), "CUDA_BATCHED");
    REQUIRE(d.get("CUDA_BATCH_SIZE", c.cudaBatchSize), "CUDA_BATCH_SIZE");
    REQUIRE(d.get("THETA", c.theta), "THETA");
    REQUIRE(d.get("NX", c.nx), "NX");
    REQUIRE(d.get("NY", c.ny), "NY");
    REQUIRE(d.get("NZ", c.nz), "NZ");
    REQUIRE(d.get("MPIX", c.mpix), "MPIX");
    REQUIRE(d.get("MPIY", c.mpiy), "MPIY");
    REQUIRE(d.get("MPIZ", c.mpiz), "MPIZ");
    REQUIRE(d.get("AX", c.ax), "AX");
    REQUIRE(d.get("AY", c.ay), "AY");
    REQUIRE(d.get("AZ", c.az), "AZ");
    REQUIRE(d.get("BX", c.bx), "BX");
    REQUIRE(d.get("BY", c.by), "BY");
    REQUIRE(d.get("BZ", c.bz), "BZ");
    if (c.solver == "pn") {
        REQUIRE(d.get("PN_USE_KINETIC_FLUX", c.pnUseKineticFlux), "PN_USE_KINETIC_FLUX");
    } else if (c.solver == "mn") {
        REQUIRE(d.get("MN_TOL", c.mnTol), "MN_TOL");
        REQUIRE(d.get("MN_COND_H_MAX", c.mnCondHMax), "MN_COND_H_MAX");
        REQUIRE(d.get("MN_MAX_ITER", c.mnMaxIter), "MN_MAX_ITER");
        REQUIRE(d.get("MN_BATCHED", c.mnBatched), "MN_BATCHED");
        REQUIRE(d.get("MN_TOL_GAMMA", c.mnTolGamma), "MN_TOL_GAMMA");
        REQUIRE(d.get("MN_USE_GAUNT_COEF", c.mnUseGaunt), "MN_USE_GAUNT_COEF");
        REQUIRE(d.get("MN_USE_GAUNT_SPARSE", c.mnUseGauntSparse), "MN_USE_GAUNT_SPARSE");
    } else {
        return "Solver type does not exist";
    }
    if (c.initCond != "gaussian" && c.initCond != "smooth" && c.initCond != "funky" &&
        c.initCond != "gaussian_psi")
        return "Initial condition not supported";
    if (c.nx < 1 || c.ny < 1 || c.nz < 1 || c.momentOrder < 0 || c.quadOrder < 1)
        return "invalid grid, moment order or quadrature order";
    // optional keys
    d.get("NSTEPS", c.nsteps);
    std::string lad;
    if (d.get("REG_LADDER", lad)) {
        c.ladder.clear();
        std::stringstream ss(lad);
        std::string tok;
        while (std::getline(ss, tok, ','))
            if (!tok.empty())
                c.ladder.push_back(std::atof(tok.c_str()));
        if (c.ladder.empty() || c.ladder.size() > 16)
            return "REG_LADDER must list 1 to 16 values";
    }
    d.get("MN_REPROJECT", c.mnReproject);
    d.get("MN_GAUNT_ON_DEVICE", c.mnGauntOnDevice);
    d.get("MN_MIXED_PRECISION", c.mnMixed);
    d.get("MN_MIXED_COND_BF16", c.mnMixedCondBf16);
    d.get("MN_MIXED_COND_MAX", c.mnMixedCondMax);
    d.get("MN_MIXED_ITER_MAX", c.mnMixedIterMax);
    d.get("MN_MIXED_POLISH", c.mnMixedPolish);
    d.get("FLUX_AUTOTUNE", c.fluxAutotune);
    d.get("SIGMA_CHECKER_BLOCK", c.checkerBlock);
    d.get("SIGMA_S_HI", c.sigmaSHi);
    d.get("SIGMA_A_HI", c.sigmaAHi);
    return "";
}

// Initial conditions, src/init.cpp:26-67.
static double gaussian_ic(double sigma, double x, double y, double z)
{
    double s2 = sigma * sigma;
    double factor1d = 1.0 / (sigma * sqrt(2.0 * M_PI));
    double factor3d = factor1d * factor1d * factor1d;
    return factor3d * exp(-(x * x + y * y + z * z) / (2.0 * s2));
}
static double smooth_ic(double x, double y, double z)
{
    return 2.0 + cos(2 * M_PI * x) * cos(2 * M_PI * y) * cos(2 * M_PI * z);
}
static double funky_ic(const Config &c, double sigma, double x, double y, double z)
{
    double r = 0.0;
    double wx = c.bx - c.ax, wy = c.by - c.ay, wz = c.bz - c.az;
    for (int i = 1; i < 10; i += 2)
        for (int j = 1; j < 10; j += 2)
            for (int k = 1; k < 10; k += 2)
                r += gaussian_ic(sigma, x - (c.ax + i * wx / 10.0), y - (c.ay + j * wy / 10.0),
                                 z - (c.az + k * wz / 10.0));
    return smooth_ic(x, y, z) + r;
}

Solver::~Solver()
{
    if (ctx_)
        c3d_destroy(ctx_);
}

void Solver::prepare(const Config &cfg)
{
    cfg_ = cfg;
    const Config &c = cfg_;
    // setupLocalMpiInfo, one rank (src/init.cpp:104-121)
    dx_ = (c.bx - c.ax) / c.nx;
    dy_ = (c.by - c.ay) / c.ny;
    dz_ = (c.bz - c.az) / c.nz;
    nq_ = 2 * c.quadOrder * c.quadOrder;
    nm_ = (c.momentOrder + 1) * (c.momentOrder + 1);
    const int nm = nm_, nq = nq_;
    const int nxg = c.nx + 4, nyg = c.ny + 4, nzg = c.nz + 4;
    const long long nall = (long long)nxg * nyg * nzg;

    u.assign(nall * nm, 0.0);
    sigT.assign(nall, 0.0);
    sigS.assign(nall, 0.0);
    // initial condition and cross sections (src/init.cpp:480-506)
    for (int i = 0; i < nxg; i++)
        for (int j = 0; j < nyg; j++)
            for (int k = 0; k < nzg; k++) {
                long long cell = (long long)k + nzg * ((long long)j + (long long)nyg * i);
                double x = c.ax + (i - 2) * dx_ + dx_ / 2.0;
                double y = c.ay + (j - 2) * dy_ + dy_ / 2.0;
                double z = c.az + (k - 2) * dz_ + dz_ / 2.0;
                double ss = c.crossSection, sa = 0.0;
                if (c.checkerBlock > 0) {
                    // periodic block index so ghost cells carry their image's values
                    int ii = ((i - 2) % c.nx + c.nx) % c.nx, jj = ((j - 2) % c.ny + c.ny) % c.ny,
                        kk = ((k - 2) % c.nz + c.nz) % c.nz;
                    int parity = (ii / c.checkerBlock + jj / c.checkerBlock + kk / c.checkerBlock) & 1;
                    if (parity) {
                        ss = c.sigmaSHi;
                        sa = c.sigmaAHi;
                    }
                }
                sigT[cell] = ss + sa;
                sigS[cell] = ss;
                double *uc = &u[cell * nm];
                if (c.initCond == "gaussian") {
                    uc[0] = std::max(c.initFloor, gaussian_ic(c.gaussSigma, x, y, z) * 2.0 * sqrt(M_PI));
                } else if (c.initCond == "gaussian_psi") {
                    double psi = std::max(c.initFloor, gaussian_ic(c.gaussSigma, x, y, z) / (4.0 * M_PI));
                    uc[0] = 2.0 * sqrt(M_PI) * psi;
                } else if (c.initCond == "smooth") {
                    uc[0] = smooth_ic(x, y, z) * 2.0 * sqrt(M_PI);
                    if (nm > 3) {
                        uc[1] = 0.3 * uc[0];
                        uc[2] = 0.3 * uc[0];
                        uc[3] = 0.3 * uc[0];
                    }
                } else {
                    uc[0] = funky_ic(c, c.gaussSigma, x, y, z) * 2.0 * sqrt(M_PI);
                }
            }
    // quadrature (src/init.cpp:509-548)
    M.assign((size_t)nq * nm, 0.0);
    w.assign(nq, 0.0);
    xi.assign(nq, 0.0);
    eta.assign(nq, 0.0);
    mu.assign(nq, 0.0);
    c3d_build_quadrature(c.momentOrder, c.quadOrder, w.data(), xi.data(), eta.data(), mu.data(),
                         M.data(), nullptr);

    c3d_params &P = params_;
    P = c3d_params{};
    P.nx = c.nx;
    P.ny = c.ny;
    P.nz = c.nz;
    P.nm = nm;
    P.nq = nq;
    P.dx = dx_;
    P.dy = dy_;
    P.dz = dz_;
    P.theta = c.theta;
    P.solver = c.solver == "mn" ? 1 : 0;
    P.pnUseKineticFlux = c.pnUseKineticFlux;
    P.mnBatched = c.mnBatched ? 1 : 0;
    P.mnMaxIter = c.mnMaxIter;
    P.mnTol = c.mnTol;
    P.mnTolGamma = c.mnTolGamma;
    P.mnReproject = c.mnReproject ? 1 : 0;
    P.mnCondHMax = c.mnCondHMax;
    P.nreg = (int)c.ladder.size();
    for (size_t i = 0; i < c.ladder.size(); ++i)
        P.reg[i] = c.ladder[i];

    if (c.solver == "pn") {
        // initPn, src/init.cpp:193-238
        pnOps.assign((size_t)6 * nm * nm, 0.0);
        for (int i = 0; i < nm; i++)
            for (int j = 0; j < nm; j++) {
                double v[6] = {0, 0, 0, 0, 0, 0};
                for (int q = 0; q < nq; q++) {
                    double mi = M[(size_t)q * nm + i], mj = M[(size_t)q * nm + j];
                    if (xi[q] > 0) v[0] += xi[q] * mi * mj * w[q];
                    else v[1] += xi[q] * mi * mj * w[q];
                    if (eta[q] > 0) v[2] += eta[q] * mi * mj * w[q];
                    else v[3] += eta[q] * mi * mj * w[q];
                    if (mu[q] > 0) v[4] += mu[q] * mi * mj * w[q];
                    else v[5] += mu[q] * mi * mj * w[q];
                }
                for (int k = 0; k < 6; k++)
                    pnOps[(size_t)k * nm * nm + i * nm + j] = v[k];
            }
        maxDt_ = c.cfl * 0.5 * std::min(std::min(dx_, dy_), dz_);
        alpha.clear();
    } else {
        // initMn, src/init.cpp:260-274
        alpha.assign(nall * nm, 0.0);
        for (long long cell = 0; cell < nall; cell++)
            alpha[cell * nm] = sqrt(4.0 * M_PI) * log(u[cell * nm] / sqrt(4.0 * M_PI));
        maxDt_ = c.cfl * (2.0 / (2.0 + c.theta)) / (1.0 / dx_ + 1.0 / dy_ + 1.0 / dz_);
    }
}

c3d_status Solver::prepare_gaunt()
{
    // Gaunt coefficients by least squares over the quadrature (src/init.cpp:287-336)
    const int N = cfg_.momentOrder, nm = nm_, nq = nq_;
    const int nm2 = (2 * N + 1) * (2 * N + 1);
    std::vector<double> w2(nq), xi2(nq), eta2(nq), mu2(nq), M1((size_t)nq * nm);
    M2.assign((size_t)nq * nm2, 0.0);
    c3d_build_quadrature(N, cfg_.quadOrder, w2.data(), xi2.data(), eta2.data(), mu2.data(),
                         M1.data(), M2.data());
    double thr = cfg_.mnUseGauntSparse ? 1e-13 : 0.0;
    if (cfg_.mnGauntOnDevice) {
        // the same least-squares tables built on the device (values agree to rounding)
        const long long cap = (long long)nm * nm * nm2;
        betaRow.assign((size_t)nm * nm + 1, 0);
        betaCol.assign((size_t)cap, 0);
        betaVal.assign((size_t)cap, 0.0);
        long long nnz = 0;
        c3d_status s = c3d_gaunt_build(nm, nm2, nq, M2.data(), thr, nullptr, betaRow.data(), cap,
                                       betaCol.data(), betaVal.data(), &nnz);
        if (s != C3D_OK)
            return s;
        betaCol.resize(nnz > 0 ? (size_t)nnz : 1);
        betaVal.resize(nnz > 0 ? (size_t)nnz : 1);
        nm2_ = nm2;
        return C3D_OK;
    }
    std::vector<double> beta((size_t)nm * nm * nm2);
    c3d_gaunt_dense(nm, nm2, nq, M2.data(), beta.data());
    int nnz = c3d_gaunt_csr_threshold(nm, nm2, beta.data(), thr, nullptr, nullptr, nullptr);
    betaRow.assign((size_t)nm * nm + 1, 0);
    betaCol.assign(nnz > 0 ? nnz : 1, 0);
    betaVal.assign(nnz > 0 ? nnz : 1, 0.0);
    c3d_gaunt_csr_threshold(nm, nm2, beta.data(), thr, betaVal.data(), betaCol.data(),
                            betaRow.data());
    nm2_ = nm2;
    return C3D_OK;
}

c3d_status Solver::init(const Config &cfg, void *stream)
{
    prepare(cfg);
    c3d_status s = c3d_create(&params_, M.data(), w.data(), xi.data(), eta.data(), mu.data(),
                              pnOps.empty() ? nullptr : pnOps.data(), stream, &ctx_);
    if (s != C3D_OK)
        return s;
    if (cfg_.solver == "mn" && cfg_.mnUseGaunt) {
        if (nm_ > 64) {
            fprintf(stderr, "[c3d_b200] MN_USE_GAUNT_COEF: Gaunt form provided for N <= 7; the "
                            "closure forms H by direct quadrature (same H up to rounding)\n");
        } else {
            if ((s = prepare_gaunt()) != C3D_OK)
                return s;
            s = c3d_set_gaunt(ctx_, nm2_, M2.data(), betaRow.data(), betaCol.data(),
                              betaVal.data());
            if (s != C3D_OK)
                return s;
        }
    }
    if (cfg_.solver == "mn" && cfg_.mnMixed &&
        (s = c3d_set_precision(ctx_, 1, cfg_.mnMixedCondBf16, cfg_.mnMixedCondMax,
                               cfg_.mnMixedIterMax, cfg_.mnMixedPolish)) != C3D_OK)
        return s;
    if (cfg_.outputTimings && (s = c3d_timing_enable(ctx_, 1)) != C3D_OK)
        return s;
    if (cfg_.outputOptStats && cfg_.solver == "mn") {
        // room for every closure of the run (the reference sizes g_optStats from TFINAL,
        // src/init.cpp:558-568)
        long long steps = cfg_.nsteps >= 0 ? cfg_.nsteps
                                           : (long long)std::ceil(cfg_.tFinal / maxDt_) + 2;
        if ((s = c3d_line_stats_enable(ctx_, (int)(2 * steps + 2))) != C3D_OK)
            return s;
    }
    if ((s = push()) != C3D_OK)
        return s;
    if (cfg_.solver == "mn" && cfg_.fluxAutotune && (s = c3d_autotune(ctx_, nullptr, nullptr, nullptr)) != C3D_OK)
        return s;
    return C3D_OK;
}

c3d_status Solver::push()
{
    return c3d_set_state(ctx_, u.data(), alpha.empty() ? nullptr : alpha.data(), sigT.data(),
                         sigS.data(), 0);
}

c3d_status Solver::pull()
{
    return c3d_get_state(ctx_, u.data(), alpha.empty() ? nullptr : alpha.data(), 0);
}

c3d_status Solver::update(double dt)
{
    c3d_status s = c3d_step(ctx_, dt);
    if (s != C3D_OK)
        return s;
    ++numUpdates_;
    return cfg_.outputTimings ? record_update_times() : C3D_OK;
}

// The 8 timers of one update (src/update.cpp:217-262): per RK stage communicateBoundaries,
// solveOptimization (0 for P_N), the flux and the Euler stage, in seconds, from the
// context's stage events (synchronises).
c3d_status Solver::record_update_times()
{
    std::vector<int> kinds(64);
    std::vector<double> ms(64);
    int n = c3d_timing_events(ctx_, kinds.data(), ms.data(), (int)kinds.size());
    if (n < 0)
        return C3D_ERR_CUDA;
    double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int stage = 0;
    static const int slot[4] = {1, 2, 0, 3}; // kind: closure, flux, ghost fill, Euler
    for (int e = 0; e < n; ++e) {
        if (kinds[e] < 0 || kinds[e] > 3)
            continue;
        t[4 * stage + slot[kinds[e]]] += 1e-3 * ms[e];
        if (kinds[e] == 3 && stage == 0)
            stage = 1; // the first Euler stage ends RK stage 1
    }
    updateTimes_.insert(updateTimes_.end(), t, t + 8);
    return c3d_timing_enable(ctx_, 1); // clears the events for the next update
}

c3d_status Solver::outputTimings(const std::string &dir)
{
    std::string err;
    if (!write_timings(dir, numUpdates_, updateTimes_, err)) {
        fprintf(stderr, "[c3d_b200] outputTimings: %s\n", err.c_str());
        return C3D_ERR_INVALID;
    }
    return C3D_OK;
}

c3d_status Solver::outputOptStats(const std::string &dir)
{
    std::vector<double> log;
    if (ctx_ && cfg_.solver == "mn") {
        int count = 0;
        c3d_status s = c3d_line_stats_get(ctx_, nullptr, &count);
        if (s != C3D_OK)
            return s;
        log.resize((size_t)count * cfg_.nx * 5);
        if ((s = c3d_line_stats_get(ctx_, log.data(), &count)) != C3D_OK)
            return s;
    }
    std::string err;
    if (!write_opt_stats(dir, numUpdates_, cfg_.nx, log, err)) {
        fprintf(stderr, "[c3d_b200] outputOptStats: %s\n", err.c_str());
        return C3D_ERR_INVALID;
    }
    return C3D_OK;
}

c3d_status Solver::outputData(double time, const std::string &dir)
{
    OutputStats st;
    st.regHist.assign(cfg_.ladder.size(), 0);
    if (ctx_) {
        c3d_status s = pull();
        if (s != C3D_OK)
            return s;
        if (cfg_.solver == "mn") {
            c3d_closure_stats cs;
            if ((s = c3d_closure_stats_get(ctx_, &cs)) != C3D_OK)
                return s;
            st.maxIter = cs.maxIter;
            st.maxIterGamma = cs.maxIterGamma;
            st.numDualSolves = cs.cells;
            st.iterMean = cs.cells ? (double)cs.totalIters / (double)cs.cells : 0.0;
            st.iterGammaMean = cs.cells ? (double)cs.totalIterGamma / (double)cs.cells : 0.0;
            for (size_t r = 0; r < st.regHist.size() && r < 16; ++r)
                st.regHist[r] = cs.regHist[r];
        }
    }
    std::string err;
    if (!write_output_data(dir, time, cfg_, nm_, u.data(), st, err)) {
        fprintf(stderr, "[c3d_b200] outputData: %s\n", err.c_str());
        return C3D_ERR_INVALID;
    }
    return C3D_OK;
}

c3d_status Solver::checkpoint(const std::string &path, double time)
{
    if (ctx_) {
        c3d_status s = pull();
        if (s != C3D_OK)
            return s;
    }
    std::string err;
    if (!write_checkpoint(path, time, cfg_, nm_, u.data(), alpha.data(), err)) {
        fprintf(stderr, "[c3d_b200] checkpoint: %s\n", err.c_str());
        return C3D_ERR_INVALID;
    }
    return C3D_OK;
}

c3d_status Solver::restore(const std::string &path, double *time)
{
    std::string err;
    if (!read_checkpoint(path, cfg_, nm_, u.data(), alpha.data(), time, err)) {
        fprintf(stderr, "[c3d_b200] restore: %s\n", err.c_str());
        return C3D_ERR_INVALID;
    }
    return ctx_ ? push() : C3D_OK;
}

// The time loop of src/main.cpp:57-76 (or NSTEPS steps of dt_max): step(dt) for each update,
// out(t) at each output time; stops at the first status that is not C3D_OK. A positive OUTDT
// is required with TFINAL (the reference's loop never ends otherwise).
c3d_status Solver::walk(const std::function<c3d_status(double)> &step,
                        const std::function<c3d_status(double)> &out) const
{
    c3d_status s;
    if (cfg_.nsteps >= 0) {
        for (int n = 0; n < cfg_.nsteps; ++n)
            if ((s = step(maxDt_)) != C3D_OK)
                return s;
        return out(cfg_.nsteps * maxDt_);
    }
    if (!(cfg_.outDt > 0.0))
        return C3D_ERR_INVALID;
    double t = 0.0, dt;
    const double tFinal = cfg_.tFinal;
    for (double tOut = std::min(t + cfg_.outDt, tFinal); tOut <= tFinal;
         tOut = std::min(tOut + cfg_.outDt, tFinal)) {
        dt = maxDt_;
        while (t < tOut - 1e-14 * tOut) {
            t += dt;
            if (t > tOut) {
                dt = tOut - (t - dt);
                t = tOut;
            }
            if ((s = step(dt)) != C3D_OK)
                return s;
        }
        if ((s = out(t)) != C3D_OK)
            return s;
        if (tOut > tFinal - 1e-14 * tFinal)
            break;
    }
    return C3D_OK;
}

c3d_status Solver::plan(std::vector<double> &dts) const
{
    dts.clear();
    return walk(
        [&](double dt) {
            dts.push_back(dt);
            return C3D_OK;
        },
        [](double) { return C3D_OK; });
}

c3d_status Solver::run(int *stepsTaken)
{
    int steps = 0;
    c3d_status s = C3D_OK;
    if (cfg_.outputData && (s = outputData(0.0, "output")) != C3D_OK)
        return s;
    s = walk(
        [&](double dt) {
            c3d_status e = update(dt);
            if (e == C3D_OK)
                ++steps;
            return e;
        },
        [&](double t) { return cfg_.outputData ? outputData(t, "output") : C3D_OK; });
    if (s != C3D_OK)
        return s;
    if (stepsTaken)
        *stepsTaken = steps;
    if ((s = c3d_sync(ctx_)) != C3D_OK)
        return s;
    // src/main.cpp:98-103
    if (cfg_.outputTimings && (s = outputTimings("output")) != C3D_OK)
        return s;
    if (cfg_.outputOptStats && (s = outputOptStats("output")) != C3D_OK)
        return s;
    return C3D_OK;
}

} // namespace c3d_host

// ---------------------------------------------------------------- C ABI of the host solver
using c3d_host::Solver;

struct c3d_solver {
    Solver s;
};

extern "C" {

/* Reads a deck and runs init() (tables, IC, multipliers, dt) on the current device. */
c3d_status c3d_solver_create(const char *deckPath, void *stream, c3d_solver **out)
{
    if (!deckPath || !out)
        return C3D_ERR_INVALID;
    c3d_host::InputDeck deck;
    if (!deck.read(deckPath))
        return C3D_ERR_INVALID;
    c3d_host::Config cfg;
    std::string err = c3d_host::parse_config(deck, cfg);
    if (!err.empty()) {
        fprintf(stderr, "[c3d_b200] %s: %s\n", deckPath, err.c_str());
        return C3D_ERR_INVALID;
    }
    std::unique_ptr<c3d_solver> s(new c3d_solver());
    c3d_status st = s->s.init(cfg, stream);
    if (st != C3D_OK)
        return st;
    *out = s.release();
    return C3D_OK;
}

/* Host-only init(): parses the deck and builds tables, initial state, cross
 * sections, multipliers and dt_max without touching a GPU. errbuf receives the
 * first missing or invalid key. */
c3d_status c3d_solver_prepare(const char *deckPath, c3d_solver **out, char *errbuf, int errlen)
{
    if (!deckPath || !out)
        return C3D_ERR_INVALID;
    c3d_host::InputDeck deck;
    std::string err;
    if (!deck.read(deckPath))
        err = "Could not open file.";
    c3d_host::Config cfg;
    if (err.empty())
        err = c3d_host::parse_config(deck, cfg);
    if (!err.empty()) {
        if (errbuf && errlen > 0)
            snprintf(errbuf, errlen, "%s", err.c_str());
        return C3D_ERR_INVALID;
    }
    c3d_solver *s = new c3d_solver();
    s->s.prepare(cfg);
    *out = s;
    return C3D_OK;
}

void c3d_solver_destroy(c3d_solver *s) { delete s; }

c3d_status c3d_solver_update(c3d_solver *s, double dt) { return s ? s->s.update(dt) : C3D_ERR_INVALID; }
c3d_status c3d_solver_run(c3d_solver *s, int *steps) { return s ? s->s.run(steps) : C3D_ERR_INVALID; }
c3d_status c3d_solver_pull(c3d_solver *s) { return s ? s->s.pull() : C3D_ERR_INVALID; }
c3d_status c3d_solver_push(c3d_solver *s) { return s ? s->s.push() : C3D_ERR_INVALID; }
c3d_ctx *c3d_solver_context(c3d_solver *s) { return s ? s->s.ctx() : nullptr; }

c3d_status c3d_solver_output_data(c3d_solver *s, double time, const char *dir)
{
    return (s && dir) ? s->s.outputData(time, dir) : C3D_ERR_INVALID;
}

c3d_status c3d_solver_checkpoint(c3d_solver *s, double time, const char *path)
{
    return (s && path) ? s->s.checkpoint(path, time) : C3D_ERR_INVALID;
}

c3d_status c3d_solver_restore(c3d_solver *s, const char *path, double *time)
{
    return (s && path) ? s->s.restore(path, time) : C3D_ERR_INVALID;
}

c3d_status c3d_solver_output_timings(c3d_solver *s, const char *dir)
{
    return (s && dir) ? s->s.outputTimings(dir) : C3D_ERR_INVALID;
}

c3d_status c3d_solver_output_opt_stats(c3d_solver *s, const char *dir)
{
    return (s && dir) ? s->s.outputOptStats(dir) : C3D_ERR_INVALID;
}

/* iv: nx ny nz nm nq solver(0 pn/1 mn) nsteps ; dv: dx dy dz maxDt theta tFinal */
void c3d_solver_info(c3d_solver *s, int *iv, double *dv)
{
    const c3d_host::Config &c = s->s.config();
    iv[0] = c.nx; iv[1] = c.ny; iv[2] = c.nz; iv[3] = s->s.nm(); iv[4] = s->s.nq();
    iv[5] = c.solver == "mn" ? 1 : 0; iv[6] = c.nsteps; iv[7] = (int)c.ladder.size();
    dv[0] = s->s.dx(); dv[1] = s->s.dy(); dv[2] = s->s.dz(); dv[3] = s->s.maxDt();
    dv[4] = c.theta; dv[5] = c.tFinal;
}

/* Host mirrors (valid after c3d_solver_pull): 0 u, 1 alpha, 2 sigT, 3 sigS, 4 M, 5 w, 6 xi,
 * 7 eta, 8 mu, 9 P_N operators. */
double *c3d_solver_host_array(c3d_solver *s, int which)
{
    Solver &v = s->s;
    std::vector<double> *a[] = {&v.u, &v.alpha, &v.sigT, &v.sigS, &v.M, &v.w, &v.xi, &v.eta, &v.mu, &v.pnOps};
    if (which < 0 || which > 9 || a[which]->empty())
        return nullptr;
    return a[which]->data();
}

} // extern "C"
