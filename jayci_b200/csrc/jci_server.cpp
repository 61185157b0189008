// jci_server.cpp -- request loop with continuous batching on one GPU.
//
// Worker threads ("slots") take requests from one queue.  A request is
// admitted when a slot is free and its estimated device footprint fits in
// what the running solves leave of the HBM budget; later requests that fit
// may pass an earlier one that does not (no head-of-line blocking).  Each
// solve runs the ordinary jci_davidson on its own space handle, whose
// kernels go to that handle's own stream, so solves in different slots
// overlap on the device.  Spaces are cached by their &general values
// (device tables, tuned sigma plans and Davidson buffers are reused by the
// next request on the same space: a geometry scan re-uploads integrals
// only), and a request may start from the Ritz vectors of an earlier one:
// it is not started before that one has finished, so the steps of a scan
// run in order while other scans fill the remaining slots.
//
// Each result depends only on its own request: every kernel sums in a fixed
// order, so a solve returns the same numbers alone and in a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "jci_internal.h"

namespace jci {
jci_status finish_space(jci_space *s);
}

using namespace jci;
using Clock = std::chrono::steady_clock;

namespace {

using Key = std::tuple<int, int, int, int, int, int, int>;

Key key_of(const jci_request &r) {
    return Key{r.electrons, r.orbitals, r.nfrozen, r.ndocc, r.nactive, r.nfrzvirt, r.xlevel};
}

struct Job {
    long long id = 0;
    jci_request req{};
    std::vector<double> m1, m2;
    size_t footprint = 0;
    long long ndets = 0;
    jci_space *fresh = nullptr;   // host-built space, used if no cached one
    bool done = false;
    jci_result res{};
    std::vector<double> civec;    // nroots x ndets
    std::vector<double> restart;  // krymin Ritz vectors, for warm starts
    Clock::time_point t_submit, t_start, t_end;
};

// Device footprint of one solve: Davidson panels, device tables, sigma
// plan scratch (generous: every panel the product kernel may allocate).
size_t estimate_footprint(const jci_space *s, const jci_request &r) {
    long long n = s->ndets, ld = (n + 31) / 32 * 32;
    size_t b = 8ull * ld * (3ull * r.krymax + 2);
    if (r.precision == JCI_MIXED) b += 8ull * ld * std::max(r.krymin, r.nroots);
    b += 12ull * n + 32ull * ld;  // hdiag (FP64+FP32), autotune and streaming scratch
    long long npair = (long long)s->ci_orbs * (s->ci_orbs + 1) / 2;
    for (int sp = 0; sp < 2; sp++) {
        const SpinSpace &x = s->sp[sp];
        b += 4ull * x.istr.size() + 24ull * x.nstr + 26ull * x.sing.size() + 8ull * x.doub.size();
        if (s->sp[0].ngrp == 1 && s->sp[1].ngrp == 1)
            b += 12ull * x.sing.size() + 12ull * npair * x.nstr + 16ull * x.doub.size() +
                 4ull * x.sing.size();
    }
    if (s->sp[0].ngrp == 1 && s->sp[1].ngrp == 1) {
        long long nbp = (s->sp[1].nstr + 63) / 64 * 64;
        long long grid = std::min<long long>(s->sp[0].nstr, 148 * 4);
        b += 12ull * grid * (npair + 1) * nbp;
    }
    b += 16ull * (npair * (npair + 1) / 2 + npair);  // integrals FP64 + FP32
    return b + (64ull << 20);                         // runtime slack
}

}  // namespace

struct jci_server {
    size_t budget = 0, used = 0;
    int slots = 1;
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> queue;
    std::map<long long, std::unique_ptr<Job>> jobs;
    long long next_id = 1;
    bool stopping = false;
    std::vector<std::thread> workers;
    // idle spaces by key (least recently used first); spaces in use are
    // owned by the worker running them
    std::list<std::pair<Key, jci_space *>> idle;
    size_t idle_max = 8;
};

static void run_job(jci_server *srv, Job *job) {
    const jci_request &r = job->req;
    Key k = key_of(r);
    jci_space *s = nullptr;
    {
        std::lock_guard<std::mutex> g(srv->mu);
        for (auto it = srv->idle.begin(); it != srv->idle.end(); ++it)
            if (it->first == k) {
                s = it->second;
                srv->idle.erase(it);
                break;
            }
    }
    if (s) {
        jci_space_destroy(job->fresh);
    } else {
        s = job->fresh;
    }
    job->fresh = nullptr;
    jci_status st = jci_set_integrals(s, job->m1.data(), job->m2.data(), s->ci_orbs, r.nucrep,
                                      r.frzcore);
    std::vector<double> init;
    int warm = 0;
    if (!st && r.warm_from > 0) {
        std::lock_guard<std::mutex> g(srv->mu);
        auto it = srv->jobs.find(r.warm_from);
        if (it != srv->jobs.end() && it->second->done && it->second->ndets == s->ndets &&
            (long long)it->second->restart.size() >= (long long)r.krymin * s->ndets) {
            init.assign(it->second->restart.begin(),
                        it->second->restart.begin() + (size_t)r.krymin * s->ndets);
            warm = 1;
        }
    }
    jci_davidson_opts o;
    jci_davidson_defaults(&o);
    o.maxiter = r.maxiter;
    o.krymin = r.krymin;
    o.krymax = r.krymax;
    o.nroots = r.nroots;
    o.refdim = r.refdim;
    o.restol = r.restol;
    o.precision = r.precision;
    o.switch_tol = r.switch_tol;
    o.block = r.block;
    o.prediagr = warm ? 3 : 1;
    o.init = warm ? init.data() : nullptr;
    jci_davidson_stats stats{};
    std::vector<double> e(r.nroots), civ((size_t)std::max(r.nroots, r.krymin) * s->ndets);
    if (!st) {
        // the solve's first krymin vectors are the Ritz vectors after the
        // final collapse; civec returns nroots <= krymin of them
        jci_davidson_opts o2 = o;
        st = davidson(s, &o2, e.data(), nullptr, &stats);
        if (st == JCI_OK || st == JCI_ERR_NOCONV) {
            jci_status c = davidson_vectors(s, std::max(r.nroots, r.krymin), civ.data());
            if (c) st = c;
        }
    }
    std::lock_guard<std::mutex> g(srv->mu);
    job->t_end = Clock::now();
    job->res.status = st == JCI_ERR_NOCONV ? JCI_OK : st;
    job->res.converged = st == JCI_OK;
    job->res.nroots = r.nroots;
    for (int i = 0; i < r.nroots && i < JCI_MAX_ROOTS; i++) job->res.energies[i] = e[i];
    job->res.iterations = stats.iterations;
    job->res.warm_started = warm;
    job->res.ndets = s->ndets;
    job->res.queue_seconds = std::chrono::duration<double>(job->t_start - job->t_submit).count();
    job->res.solve_seconds = std::chrono::duration<double>(job->t_end - job->t_start).count();
    job->res.sigma_vectors = stats.sigma_vectors;
    job->res.sigma_seconds = stats.sigma_seconds;
    if (st == JCI_OK || st == JCI_ERR_NOCONV) {
        job->civec.assign(civ.begin(), civ.begin() + (size_t)r.nroots * s->ndets);
        job->restart.assign(civ.begin(), civ.begin() + (size_t)r.krymin * s->ndets);
    }
    job->m1.clear();
    job->m1.shrink_to_fit();
    job->m2.clear();
    job->m2.shrink_to_fit();
    job->done = true;
    srv->used -= job->footprint;
    if (st == JCI_ERR_CUDA || st == JCI_ERR_NODEVICE) {
        jci_space_destroy(s);
    } else {
        srv->idle.emplace_back(k, s);
        while (srv->idle.size() > srv->idle_max) {
            jci_space_destroy(srv->idle.front().second);
            srv->idle.pop_front();
        }
    }
    srv->cv_done.notify_all();
    srv->cv_work.notify_all();
}

static void worker(jci_server *srv) {
    cudaSetDevice(srv->device);
    for (;;) {
        Job *job = nullptr;
        {
            std::unique_lock<std::mutex> g(srv->mu);
            for (;;) {
                // first queued request that fits next to the running ones and
                // whose warm-start source (an earlier ticket) has finished
                for (auto it = srv->queue.begin(); it != srv->queue.end(); ++it) {
                    if (!(srv->used == 0 || srv->used + (*it)->footprint <= srv->budget))
                        continue;
                    long long w = (*it)->req.warm_from;
                    if (w > 0) {
                        auto src = srv->jobs.find(w);
                        if (src != srv->jobs.end() && !src->second->done) continue;
                    }
                    job = *it;
                    srv->queue.erase(it);
                    break;
                }
                if (job || (srv->stopping && srv->queue.empty())) break;
                srv->cv_work.wait(g);
            }
            if (!job) return;
            srv->used += job->footprint;
            job->t_start = Clock::now();
        }
        run_job(srv, job);
    }
}

extern "C" {

jci_status jci_server_create(size_t budget, int slots, jci_server **out) {
    if (!out || slots < 1 || slots > 64) return JCI_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return JCI_ERR_NODEVICE;
    }
    jci_server *srv = new (std::nothrow) jci_server();
    if (!srv) return JCI_ERR_NOMEM;
    cudaGetDevice(&srv->device);
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete srv;
            return JCI_ERR_CUDA;
        }
        budget = fr / 10 * 8;
    }
    srv->budget = budget;
    srv->slots = slots;
    for (int i = 0; i < slots; i++) srv->workers.emplace_back(worker, srv);
    *out = srv;
    return JCI_OK;
}

jci_status jci_server_submit(jci_server *srv, const jci_request *req, long long *ticket) {
    if (!srv || !req || !ticket || !req->moints1 || !req->moints2) return JCI_ERR_ARG;
    if (req->nroots < 1 || req->nroots > JCI_MAX_ROOTS || req->krymin < req->nroots ||
        req->krymax < req->krymin || req->maxiter < 1)
        return JCI_ERR_ARG;
    if (req->precision != JCI_FP64 && req->precision != JCI_MIXED) return JCI_ERR_ARG;
    auto job = std::make_unique<Job>();
    job->req = *req;
    job->t_submit = Clock::now();
    jci_status st = jci_space_create(req->electrons, req->orbitals, req->nfrozen, req->ndocc,
                                     req->nactive, req->nfrzvirt, req->xlevel, &job->fresh);
    if (st) return st;
    jci_space *s = job->fresh;
    if (req->krymax > s->ndets) {
        jci_space_destroy(s);
        return JCI_ERR_ARG;
    }
    long long n1 = (long long)s->ci_orbs * (s->ci_orbs + 1) / 2, n2 = n1 * (n1 + 1) / 2;
    job->m1.assign(req->moints1, req->moints1 + n1);
    job->m2.assign(req->moints2, req->moints2 + n2);
    job->req.moints1 = job->req.moints2 = nullptr;
    job->ndets = s->ndets;
    job->footprint = estimate_footprint(s, *req);
    std::lock_guard<std::mutex> g(srv->mu);
    if (job->footprint > srv->budget) {
        jci_space_destroy(s);
        return JCI_ERR_BUSY;
    }
    // a warm start names an earlier ticket that has not been released, so
    // the waits between requests form a chain that always ends
    if (req->warm_from > 0 && srv->jobs.find(req->warm_from) == srv->jobs.end()) {
        jci_space_destroy(s);
        return JCI_ERR_ARG;
    }
    job->id = srv->next_id++;
    *ticket = job->id;
    srv->queue.push_back(job.get());
    srv->jobs[job->id] = std::move(job);
    srv->cv_work.notify_one();
    return JCI_OK;
}

jci_status jci_server_wait(jci_server *srv, long long ticket, double timeout_s,
                           jci_result *out) {
    if (!srv || !out) return JCI_ERR_ARG;
    std::unique_lock<std::mutex> g(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) return JCI_ERR_ARG;
    Job *job = it->second.get();
    auto ready = [&] { return job->done; };
    if (timeout_s < 0) {
        srv->cv_done.wait(g, ready);
    } else if (!srv->cv_done.wait_for(g, std::chrono::duration<double>(timeout_s), ready)) {
        return JCI_ERR_TIMEOUT;
    }
    *out = job->res;
    return JCI_OK;
}

jci_status jci_server_vectors(jci_server *srv, long long ticket, double *civec) {
    if (!srv || !civec) return JCI_ERR_ARG;
    std::lock_guard<std::mutex> g(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) return JCI_ERR_ARG;
    if (!it->second->done) return JCI_ERR_STATE;
    if (it->second->civec.empty()) return JCI_ERR_STATE;
    memcpy(civec, it->second->civec.data(), it->second->civec.size() * sizeof(double));
    return JCI_OK;
}

jci_status jci_server_release(jci_server *srv, long long ticket) {
    if (!srv) return JCI_ERR_ARG;
    std::lock_guard<std::mutex> g(srv->mu);
    auto it = srv->jobs.find(ticket);
    if (it == srv->jobs.end()) return JCI_ERR_ARG;
    if (!it->second->done) return JCI_ERR_STATE;
    srv->jobs.erase(it);
    return JCI_OK;
}

void jci_server_destroy(jci_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> g(srv->mu);
        srv->stopping = true;
    }
    srv->cv_work.notify_all();
    for (auto &t : srv->workers) t.join();
    for (auto &p : srv->idle) jci_space_destroy(p.second);
    for (auto &j : srv->jobs) jci_space_destroy(j.second->fresh);
    delete srv;
}

}  // extern "C"
