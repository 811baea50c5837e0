// Serving loop (include/c3d_serve.h): admission of independent problems against a
// device-memory budget, one scheduling thread that steps every admitted problem in one CUDA
// graph launch per pass, per-request completion latency.
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

// An admitted problem: its solver (context on the server's stream), the dt of each step of its
// time loop and the steps taken so far.
struct Active {
    Request *r = nullptr;
    std::unique_ptr<c3d_host::Solver> s;
    std::vector<double> plan;
    size_t next = 0;
};

} // namespace

struct c3d_server {
    int device = 0;
    int slots = 1;        // problems active at once at most
    long long budget = 0; // 0: unlimited
    long long inUse = 0, peakBytes = 0;
    int peakActive = 0;
    long long nextId = 1;
    bool stopping = false;
    cudaStream_t stream = nullptr; // every problem's context
    // scheduler accounting (c3d_server_timing): host seconds in admission (problem set-up),
    // in group creation and step launches (graph builds included), waiting for passes, and
    // finishing problems; passes run and group (re)builds
    double tAdmit = 0, tLaunch = 0, tWait = 0, tFinish = 0;
    long long passes = 0, builds = 0;
    std::mutex m;
    std::condition_variable cv;
    std::deque<Request *> pending;
    std::map<long long, std::unique_ptr<Request>> all;
    std::thread scheduler;

    void schedule();
    void admit(std::vector<std::unique_ptr<Active>> &active);
    void finish(Active &a, c3d_status st);
};

// Admission: requests in arrival order while a slot is free and the budget holds their
// estimated footprint; each gets its solver (tables, initial state, device context on the
// server's stream) and its step plan.
void c3d_server::admit(std::vector<std::unique_ptr<Active>> &active)
{
    for (;;) {
        Request *r = nullptr;
        {
            std::lock_guard<std::mutex> lk(m);
            if (pending.empty() || (int)active.size() >= slots)
                return;
            const long long need = pending.front()->bytes;
            if (!(budget == 0 || inUse == 0 || inUse + need <= budget))
                return;
            r = pending.front();
            pending.pop_front();
            inUse += r->bytes;
            peakBytes = inUse > peakBytes ? inUse : peakBytes;
            const int na = (int)active.size() + 1;
            peakActive = na > peakActive ? na : peakActive;
        }
        std::unique_ptr<Active> a(new Active());
        a->r = r;
        a->s.reset(new c3d_host::Solver());
        c3d_status st = a->s->init(r->cfg, stream);
        if (st == C3D_OK)
            st = a->s->plan(a->plan);
        if (st != C3D_OK || a->plan.empty()) {
            finish(*a, st);
            continue;
        }
        active.push_back(std::move(a));
    }
}

// A problem's end: its status (the closure's failures included), final interior moments,
// completion time; its device memory is released and its budget share returned.
void c3d_server::finish(Active &a, c3d_status st)
{
    Request &r = *a.r;
    if (st == C3D_OK && a.s->ctx())
        st = c3d_sync(a.s->ctx());
    if ((st == C3D_OK || st == C3D_ERR_CLOSURE) && a.s->ctx()) {
        c3d_status p = a.s->pull();
        if (p == C3D_OK) {
            const c3d_host::Config &c = r.cfg;
            const int nm = a.s->nm();
            const long long nyg = c.ny + 4, nzg = c.nz + 4;
            r.u.resize((size_t)c.nx * c.ny * c.nz * nm);
            size_t o = 0;
            for (int i = 2; i < c.nx + 2; ++i)
                for (int j = 2; j < c.ny + 2; ++j)
                    for (int k = 2; k < c.nz + 2; ++k) {
                        const long long cell = k + nzg * (j + nyg * (long long)i);
                        for (int mm = 0; mm < nm; ++mm)
                            r.u[o++] = a.s->u[(size_t)cell * nm + mm];
                    }
        } else {
            st = p;
        }
    }
    a.s.reset(); // frees the context
    {
        std::lock_guard<std::mutex> lk(m);
        r.status = st;
        r.steps = (int)a.next;
        r.done = Clock::now();
        r.finished = true;
        inUse -= r.bytes;
    }
    cv.notify_all();
}

// The scheduling loop (one host thread): every pass admits what fits, then advances every
// active problem by one step -- the M_N problems all in ONE launch, a CUDA graph whose branches
// are their RK steps (c3d_group_step; rebuilt when the set of problems or a dt changes), the
// others (P_N, or options that need launch-by-launch stages) by c3d_step on the same stream --
// and, while the GPU runs the pass, admits the next requests. Problems that took their last
// step, or failed, are finished after the pass.
void c3d_server::schedule()
{
    cudaSetDevice(device);
    std::vector<std::unique_ptr<Active>> active;
    c3d_group *group = nullptr;
    std::vector<c3d_ctx *> members;
    auto now = [] { return Clock::now(); };
    auto secs = [](Clock::time_point a, Clock::time_point b) {
        return std::chrono::duration<double>(b - a).count();
    };
    auto acc = [&](double &x, double v) {
        std::lock_guard<std::mutex> lk(m);
        x += v;
    };
    for (;;) {
        Clock::time_point t0 = now();
        admit(active);
        acc(tAdmit, secs(t0, now()));
        if (active.empty()) {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&] { return stopping || !pending.empty(); });
            if (stopping && pending.empty())
                break;
            continue;
        }
        std::vector<c3d_ctx *> grouped;
        std::vector<double> dts;
        for (auto &a : active)
            if (a->s->graphable()) {
                grouped.push_back(a->s->ctx());
                dts.push_back(a->plan[a->next]);
            }
        c3d_status gs = C3D_OK;
        t0 = now();
        if (grouped != members) {
            if (group)
                c3d_group_destroy(group);
            group = nullptr;
            members = grouped;
            if (!members.empty()) {
                gs = c3d_group_create((int)members.size(), members.data(), &group);
                std::lock_guard<std::mutex> lk(m);
                ++builds;
            }
        }
        if (gs == C3D_OK && group)
            gs = c3d_group_step(group, dts.data());
        std::vector<c3d_status> st(active.size(), C3D_OK);
        for (size_t k = 0; k < active.size(); ++k) {
            Active &a = *active[k];
            st[k] = a.s->graphable() ? gs : a.s->update(a.plan[a.next]);
        }
        Clock::time_point t1 = now();
        {
            std::lock_guard<std::mutex> lk(m);
            ++passes;
            tLaunch += secs(t0, t1);
        }
        admit(active); // overlaps the pass on the GPU; new problems join the next pass
        Clock::time_point t2 = now();
        acc(tAdmit, secs(t1, t2));
        cudaStreamSynchronize(stream);
        Clock::time_point t3 = now();
        acc(tWait, secs(t2, t3));
        // the problems of this pass are active[0 .. st.size()), in order; admitted ones follow
        for (size_t k = 0, j = 0; k < active.size(); ++j) {
            Active &a = *active[k];
            const bool stepped = j < st.size();
            const c3d_status sk = stepped ? st[j] : C3D_OK;
            if (stepped && sk == C3D_OK)
                ++a.next;
            if (sk != C3D_OK || a.next >= a.plan.size()) {
                finish(a, sk);
                active.erase(active.begin() + (long)k);
                continue;
            }
            ++k;
        }
        acc(tFinish, secs(t3, now()));
    }
    if (group)
        c3d_group_destroy(group);
}

extern "C" {

c3d_status c3d_server_create(int workers, size_t hbmBudgetBytes, c3d_server **out)
{
    if (!out || workers < 1)
        return C3D_ERR_INVALID;
    std::unique_ptr<c3d_server> s(new c3d_server());
    if (cudaGetDevice(&s->device) != cudaSuccess)
        return C3D_ERR_NO_DEVICE;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return C3D_ERR_CUDA;
    s->budget = (long long)hbmBudgetBytes;
    s->slots = workers;
    s->scheduler = std::thread([p = s.get()] { p->schedule(); });
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

c3d_status c3d_server_timing(c3d_server *s, double *seconds, long long *counts)
{
    if (!s)
        return C3D_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->m);
    if (seconds) {
        seconds[0] = s->tAdmit;
        seconds[1] = s->tLaunch;
        seconds[2] = s->tWait;
        seconds[3] = s->tFinish;
    }
    if (counts) {
        counts[0] = s->passes;
        counts[1] = s->builds;
    }
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
    s->scheduler.join();
    cudaStreamDestroy(s->stream);
    delete s;
}

} // extern "C"
