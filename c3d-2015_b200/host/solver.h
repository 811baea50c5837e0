// C++ host of the B200 M_N / P_N solver: the counterpart of the reference's
// init() (src/init.cpp:344-576), update() (src/update.cpp:185-275) and time
// loop (src/main.cpp:57-97), running every stage on one GPU through the C ABI
// of include/c3d_b200.h.
//
// Deck keys are the reference's (all mandatory, src/init.cpp:364-381,
// :195, :252-258). Optional keys, ignored by the reference, describe the
// synthetic workloads the benchmark configurations need:
//   NSTEPS n                 run exactly n steps of dt = dt_max (instead of TFINAL)
//   REG_LADDER a,b,...       regularisation ladder (default 0,1e-3,1e-2,1e-1,5e-1)
//   INIT_COND gaussian_psi   isotropic psi = max(INIT_FLOOR, G(x)/(4 pi)), u0 = 2 sqrt(pi) psi
//   SIGMA_CHECKER_BLOCK b    sigma_s/sigma_a checkerboard over b^3-cell blocks:
//   SIGMA_S_HI, SIGMA_A_HI     the odd blocks get sigma_s = SIGMA_S_HI, sigma_a = SIGMA_A_HI,
//                              the even blocks sigma_s = CROSS_SECTION, sigma_a = 0;
//                              sigma_t = sigma_s + sigma_a.
//   MN_REPROJECT true        after each closure set u = <m e^{alpha.m}> keeping u_0 (the
//                              robustness note of the reference's readme.txt)
//   MN_MIXED_PRECISION true  mixed-precision closure (c3d_set_precision mode 1; needs
//                              MN_USE_GAUNT_COEF true and N <= 6), thresholds
//                              MN_MIXED_COND_BF16, MN_MIXED_COND_MAX, MN_MIXED_ITER_MAX,
//                              MN_MIXED_POLISH
//   FLUX_AUTOTUNE true       time the kinetic flux per direction chunk and z run length at
//                              set-up and keep the fastest (c3d_autotune)
#pragma once
#include "../../include/c3d_b200.h"
#include "deck.h"

#include <functional>
#include <string>
#include <vector>

namespace c3d_host {

struct Config {
    std::string solver = "mn", initCond = "gaussian";
    double tFinal = 0, outDt = 0;
    bool outputData = false, outputOptStats = false, outputTimings = false;
    int nx = 0, ny = 0, nz = 0, mpix = 1, mpiy = 1, mpiz = 1;
    double ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
    int momentOrder = 0, quadOrder = 0;
    double cfl = 0, crossSection = 0, initFloor = 0, gaussSigma = 0, theta = 2.0;
    int ompThreads = 1;
    bool cudaKinetic = false, cudaBatched = false;
    int cudaBatchSize = 0;
    int pnUseKineticFlux = 0;
    double mnTol = 0, mnTolGamma = 0, mnCondHMax = 0;
    int mnMaxIter = 0;
    bool mnBatched = true, mnUseGaunt = false, mnUseGauntSparse = false;
    bool mnReproject = false; // optional MN_REPROJECT (readme.txt robustness note)
    bool mnGauntOnDevice = false; // optional MN_GAUNT_ON_DEVICE: beta from c3d_gaunt_build
    bool mnMixed = false;     // optional MN_MIXED_PRECISION
    double mnMixedCondBf16 = 0.0, mnMixedCondMax = 0.0;
    int mnMixedIterMax = 0;
    double mnMixedPolish = 0.0;
    bool fluxAutotune = false; // optional FLUX_AUTOTUNE: c3d_autotune after the state upload
    // optional keys
    int nsteps = -1;
    std::vector<double> ladder{0.0, 1e-3, 1e-2, 1e-1, 5e-1};
    int checkerBlock = 0;
    double sigmaSHi = 0, sigmaAHi = 0;
};

// Parses a deck; returns "" on success or the first missing/invalid key.
std::string parse_config(const InputDeck &deck, Config &cfg);

class Solver {
public:
    ~Solver();
    // Host half of init(): tables, initial condition, cross sections, multipliers, dt_max.
    void prepare(const Config &cfg);
    // init(): prepare() plus the device context and upload.
    // stream: cudaStream_t for the device work (NULL: the context's own stream).
    c3d_status init(const Config &cfg, void *stream = nullptr);
    // update(dt): one SSP-RK2 step on the device (no host synchronisation).
    c3d_status update(double dt);
    // The time loop of src/main.cpp:57-76 (or NSTEPS steps); returns the steps taken.
    c3d_status run(int *stepsTaken);
    // The dt of each update run() makes, in order (C3D_ERR_INVALID for TFINAL with OUTDT <= 0).
    c3d_status plan(std::vector<double> &dts) const;
    // Copies device state to the host arrays (u, alpha).
    c3d_status pull();
    // Copies the host arrays to the device (u, alpha, sigma_t, sigma_s).
    c3d_status push();
    // outputData(time) of src/output.cpp:19-110 into dir (the reference uses "output"): the
    // current state (pulled from the device when there is one) and closure statistics.
    c3d_status outputData(double time, const std::string &dir);
    // Checkpoint of (u, alpha) and the time; restore() loads it and pushes it to the device.
    c3d_status checkpoint(const std::string &path, double time);
    c3d_status restore(const std::string &path, double *time);
    // outputTimings / outputOptStats of src/output.cpp:116-222 for the updates run so far
    // (the per-update timers and x-line statistics are recorded when the deck sets
    // OUTPUT_TIMINGS / OUTPUT_OPT_STATS).
    c3d_status outputTimings(const std::string &dir);
    c3d_status outputOptStats(const std::string &dir);

    const Config &config() const { return cfg_; }
    c3d_ctx *ctx() { return ctx_; }
    int nm() const { return nm_; }
    // Whether its steps can run as CUDA graphs (c3d_group_step): M_N without re-projection,
    // per-update timers or x-line statistics.
    bool graphable() const
    {
        return cfg_.solver == "mn" && !cfg_.mnReproject && !cfg_.outputTimings &&
               !cfg_.outputOptStats;
    }
    int nq() const { return nq_; }
    long long ncellsAll() const { return (long long)(cfg_.nx + 4) * (cfg_.ny + 4) * (cfg_.nz + 4); }
    double dx() const { return dx_; }
    double dy() const { return dy_; }
    double dz() const { return dz_; }
    double maxDt() const { return maxDt_; }

    // host mirrors of the reference globals g_u, g_mnAlpha, g_sigmaT, g_sigmaS, g_m, g_w, ...
    std::vector<double> u, alpha, sigT, sigS, M, w, xi, eta, mu, pnOps;
    // Gaunt form (MN_USE_GAUNT_COEF): g_m2 and the CSR of g_beta
    std::vector<double> M2, betaVal;
    std::vector<int> betaRow, betaCol;

private:
    c3d_status walk(const std::function<c3d_status(double)> &step,
                    const std::function<c3d_status(double)> &out) const;
    Config cfg_;
    c3d_ctx *ctx_ = nullptr;
    c3d_params params_{};
    int nm_ = 0, nq_ = 0, nm2_ = 0;
    c3d_status prepare_gaunt();
    double dx_ = 0, dy_ = 0, dz_ = 0, maxDt_ = 0;
    int numUpdates_ = 0;
    std::vector<double> updateTimes_; // 8 seconds per update (OUTPUT_TIMINGS)
    c3d_status record_update_times();
};

} // namespace c3d_host
