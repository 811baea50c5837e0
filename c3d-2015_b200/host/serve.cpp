// Serving loop (include/c3d_serve.h): admission of independent problems against a
// device-memory budget, a pool of host threads each driving one problem's context to
// completion, per-request completion latency.
#include "../../include/c3d_serve.h"
#include "deck.h"
#include "solver.h"

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace {

using Clock = std::chrono::steady_clock;

// Device bytes one problem holds at its peak: state (u, alpha, uOld, flux), cross sections,
// per-cell records, the materialised ansatz of one direction chunk (all directions when they
// fit the default 32 GiB budget, as the closure's ansatz hand-off wants), the hand-off's
// refresh list, the closure's work-list state and buffers, tables; 10% and 64 MiB of slack.
long long footprint(const c3d_host::Config &c)
{
    const long long nall = (long long)(c.nx + 4) * (c.ny + 4) * (c.nz + 4);
    const long long nm = (long long)(c.momentOrder + 1) * (c.momentOrder + 1);
    const long long nmp = 8 * ((nm + 7) / 8);
    const long long nq = 2LL * c.quadOrder * c.quadOrder;
    const long long psiCap = (32LL << 30) / 8 / (nall > 0 ? nall : 1);
    const long long psiDirs = nq < psiCap ? nq : psiCap;
    long long b = 4 * nall * nm * 8 + 2 * nall * 8 + 5 * nall * 4 + 2 * nall * 8;
    b += psiDirs * nall * 8 + nall * 4;
    if (c.solver == "mn") {
        const long long batch = nall < (1LL << 20) ? nall : (1LL << 20);
        const long long nm2 = (2LL * c.momentOrder + 1) * (2 * c.momentOrder + 1);
        const long long nm2p = 8 * ((nm2 + 7) / 8);
        const long long per = c.mnUseGaunt ? (c.mnMixed ? nm2p + nmp + 8 : nm2p)
                                           : 64 * ((nmp / 8) * (nmp / 8 + 1) / 2);
        // state, the work lists (four kinds of pass, two generations), the face map
        b += nall * (6 * nmp * 8 + 176) + 9 * nall * 4 + batch * per * 8;
        b += nq * (nm2 + 1) * 8 * 2;
    }
    b += nq * nm * 8 * 4;
    return b + b / 10 + (64LL << 20);
}

bool parse(const char *text, c3d_host::Config &cfg, std::string &err)
{
    if (!text) {
        err = "null deck";
        return false;
    }
    c3d_host::InputDeck deck;
    deck.parse(text);
    err = c3d_host::parse_config(deck, cfg);
    return err.empty();
}

struct Request {
    long long id = 0;
    c3d_host::Config cfg;
    long long bytes = 0;
    Clock::time_point submitted, done;
    bool finished = false;
    c3d_status status = C3D_OK;
    int steps = 0;
    std::vector<double> u; // final interior moments
};

} // namespace

struct c3d_server {
    int device = 0;
    long long budget = 0; // 0: unlimited
    long long inUse = 0, peakBytes = 0;
    int active = 0, peakActive = 0;
    long long nextId = 1;
    bool stopping = false;
    std::mutex m;
    std::condition_variable cv;
    std::deque<Request *> pending;
    std::map<long long, std::unique_ptr<Request>> all;
    std::vector<std::thread> workers;

    void work();
    void run(Request &r);
};

// One problem on its own context: init (tables, initial state, device upload), the time
// loop, the final state back to the host.
void c3d_server::run(Request &r)
{
    cudaSetDevice(device);
    c3d_host::Solver s;
    int steps = 0;
    c3d_status st = s.init(r.cfg, nullptr);
    // launch by launch: capturing CUDA graphs on worker threads while other workers create,
    // free and synchronise their contexts crashed the process in testing (cause not found),
    // so the serving loop's problems do not use the stage and closure graphs
    if (st == C3D_OK && s.ctx())
        st = c3d_set_graphs(s.ctx(), 0);
    if (st == C3D_OK)
        st = s.run(&steps);
    if (st == C3D_OK || st == C3D_ERR_CLOSURE) {
        c3d_status p = s.pull();
        if (p == C3D_OK) {
            const c3d_host::Config &c = r.cfg;
            const int nm = s.nm();
            const long long nyg = c.ny + 4, nzg = c.nz + 4;
            r.u.resize((size_t)c.nx * c.ny * c.nz * nm);
            size_t o = 0;
            for (int i = 2; i < c.nx + 2; ++i)
                for (int j = 2; j < c.ny + 2; ++j)
                    for (int k = 2; k < c.nz + 2; ++k) {
                        const long long cell = k + nzg * (j + nyg * (long long)i);
                        for (int mm = 0; mm < nm; ++mm)
                            r.u[o++] = s.u[(size_t)cell * nm + mm];
                    }
        } else {
            st = p;
        }
    }
    r.status = st;
    r.steps = steps;
}

void c3d_server::work()
{
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&] {
                if (pending.empty())
                    return stopping;
                const long long need = pending.front()->bytes;
                return budget == 0 || inUse == 0 || inUse + need <= budget;
            });
            if (pending.empty())
                return;
            r = pending.front();
            pending.pop_front();
            inUse += r->bytes;
            ++active;
            peakBytes = inUse > peakBytes ? inUse : peakBytes;
            peakActive = active > peakActive ? active : peakActive;
        }
        run(*r);
        {
            std::lock_guard<std::mutex> lk(m);
            r->done = Clock::now();
            r->finished = true;
            inUse -= r->bytes;
            --active;
        }
        cv.notify_all();
    }
}

extern "C" {

c3d_status c3d_server_create(int workers, size_t hbmBudgetBytes, c3d_server **out)
{
    if (!out || workers < 1)
        return C3D_ERR_INVALID;
    std::unique_ptr<c3d_server> s(new c3d_server());
    if (cudaGetDevice(&s->device) != cudaSuccess)
        return C3D_ERR_NO_DEVICE;
    s->budget = (long long)hbmBudgetBytes;
    for (int w = 0; w < workers; ++w)
        s->workers.emplace_back([p = s.get()] { p->work(); });
    *out = s.release();
    return C3D_OK;
}

c3d_status c3d_server_estimate(const char *deckText, long long *bytes)
{
    c3d_host::Config cfg;
    std::string err;
    if (!bytes || !parse(deckText, cfg, err))
        return C3D_ERR_INVALID;
    *bytes = footprint(cfg);
    return C3D_OK;
}

c3d_status c3d_server_submit(c3d_server *s, const char *deckText, long long *id)
{
    if (!s || !id)
        return C3D_ERR_INVALID;
    std::unique_ptr<Request> r(new Request());
    std::string err;
    if (!parse(deckText, r->cfg, err)) {
        fprintf(stderr, "[c3d_b200] c3d_server_submit: %s\n", err.c_str());
        return C3D_ERR_INVALID;
    }
    r->bytes = footprint(r->cfg);
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->budget && r->bytes > s->budget)
            return C3D_ERR_OOM;
        r->id = s->nextId++;
        *id = r->id;
        s->pending.push_back(r.get());
        s->all[r->id] = std::move(r);
    }
    s->cv.notify_all();
    return C3D_OK;
}

c3d_status c3d_server_wait(c3d_server *s, long long id, int *dims, double *u, long long capacity,
                           double *latency, int *steps)
{
    if (!s)
        return C3D_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end())
        return C3D_ERR_INVALID;
    Request &r = *it->second;
    s->cv.wait(lk, [&] { return r.finished; });
    const c3d_host::Config &c = r.cfg;
    if (dims) {
        dims[0] = c.nx;
        dims[1] = c.ny;
        dims[2] = c.nz;
        dims[3] = (c.momentOrder + 1) * (c.momentOrder + 1);
    }
    if (u && capacity >= (long long)r.u.size())
        for (size_t k = 0; k < r.u.size(); ++k)
            u[k] = r.u[k];
    if (latency)
        *latency = std::chrono::duration<double>(r.done - r.submitted).count();
    if (steps)
        *steps = r.steps;
    return r.status;
}

c3d_status c3d_server_stats(c3d_server *s, long long *peakBytes, int *peakActive)
{
    if (!s)
        return C3D_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->m);
    if (peakBytes)
        *peakBytes = s->peakBytes;
    if (peakActive)
        *peakActive = s->peakActive;
    return C3D_OK;
}

void c3d_server_destroy(c3d_server *s)
{
    if (!s)
        return;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stopping = true;
    }
    s->cv.notify_all();
    for (auto &t : s->workers)
        t.join();
    delete s;
}

} // extern "C"
