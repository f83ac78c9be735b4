// Serving layer (hdd_server_* in include/hdd.h): Poisson solves of uneven
// domains arriving over time, run concurrently on one GPU.
//
// The reference has no counterpart: its GPU demo solves one domain per process
// (GPU/Test_Bench_3D/main.cpp), with one worker thread per GPU draining a
// command queue (GPU/Nodes/Command.h:33-55).  Here a server owns `slots`
// worker threads.  Each resident domain is one Solver: read-only device data
// (layout tables, interface matrices, factors and solve plans) plus a pool of
// solve contexts (PCG vectors, sigma V-cycle buffers and a captured CUDA graph
// of the preconditioner, each on its own stream) holding 1, 2 or 4 systems.
// A worker takes the oldest queued request whose domain is resident and has
// an idle context, or room in the HBM budget for a new one (at most `slots`
// drivers per domain), and becomes a driver: with batching on and more of the
// domain's requests waiting it takes a context of several systems, otherwise
// one of one, and solves requests of that domain continuously, each new one
// joining as soon as a system is free (continuous batching), until none is
// waiting.  Requests on one domain overlap on the device as well as requests
// on different domains.  Every system of every context runs the same kernels
// in the same order, so a request's result does not depend on which context,
// which batch or how many others ran beside it.
// Domains are admitted in arrival order once their estimated device footprint
// fits the HBM budget; their host setup (layout, interface assembly,
// factorisation) runs on a worker with setup_threads OpenMP threads, so
// setups overlap with solves of other domains.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "solver.h"

using hdd::Error;
using hdd::Solver;
using hdd::Work;
using Clock = std::chrono::steady_clock;

namespace {

enum class DomainState { Waiting, Admitted, SettingUp, Resident, Failed };

struct Domain {
    hdd_options opts;
    std::vector<uint32_t> flags;     // freed once set up
    DomainState state = DomainState::Waiting;
    hdd_status status = HDD_OK;      // setup failure status
    std::string error;
    std::unique_ptr<Solver> solver;
    struct Ctx {
        Work* w;
        bool busy;
    };
    std::vector<Ctx> pool;           // solve contexts (the solver's first included)
    std::vector<std::unique_ptr<Work>> owned;  // contexts beyond the solver's first
    long long ctx_bytes[3] = {0, 0, 0};  // device bytes of a further context of 1, 2, 4 systems
    int batch_k = 1;                 // most systems per context (1: batching off)
    long long reserved = 0;          // bytes counted against the budget
    int running = 0;                 // drivers solving its requests
    int capacity = 0;                // systems of the running drivers' contexts
    int held = 0;                    // requests those systems hold
    bool removing = false;
    int queued = 0;                  // requests not yet finished
};

struct Request {
    long long domain = 0;
    std::vector<float> rhs;
    bool done = false;
    hdd_status status = HDD_OK;
    hdd_result result{};
    std::vector<float> x;
    Clock::time_point t_submit, t_done;
};

// Device footprint estimate made before the setup: the dense staging buffer
// (4 B per grid cell), six PCG vectors plus flags over the stored tiles
// (26 B per tile cell, 8 B more for the FP64 iterate of the precision form),
// the V-cycle level flags (about 1.2 B per tile cell) and the interface
// solver's factors and FP64 vectors (56 B per Active cell, an upper estimate
// from the 64^3..256^3 sphere domains).
long long estimate_bytes(const hdd_options& o, const uint32_t* flags) {
    const long long n0 = o.size[0], n1 = o.size[1], n2 = o.size[2];
    const int s = std::max(1, o.sub_size[0]);
    const long long t1 = (n1 + s - 1) / s, t2 = (n2 + s - 1) / s, t0 = (n0 + s - 1) / s;
    std::vector<uint8_t> used((size_t)(t0 * t1 * t2), 0);
    long long active = 0;
    for (long long i = 0; i < n0; ++i)
        for (long long j = 0; j < n1; ++j)
            for (long long k = 0; k < n2; ++k)
                if (flags[(i * n1 + j) * n2 + k] & 0x10000u) {
                    ++active;
                    used[(size_t)(((i / s) * t1 + j / s) * t2 + k / s)] = 1;
                }
    long long tiles = 0;
    for (uint8_t u : used) tiles += u;
    const long long tile_cells = tiles * s * s * s;
    const long long per_tile_cell = o.precision_mode == HDD_PRECISION_MIXED ? 36 : 28;
    return 4 * n0 * n1 * n2 + per_tile_cell * tile_cells + 56 * active + (16ll << 20);
}

}  // namespace

struct hdd_server {
    hdd_server_options opt{};
    long long budget = 0, reserved = 0;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    long long next_id = 1;
    std::map<long long, Domain> domains;
    std::map<long long, Request> requests;
    std::deque<long long> admission;   // domains waiting for budget, in arrival order
    std::deque<long long> setups;      // admitted domains waiting for a worker
    std::deque<long long> queue;       // requests not yet started, in arrival order
    std::vector<std::thread> workers;
    int setting_up = 0;                // setups in progress

    // Moves waiting domains into the setup queue while the budget allows.
    void admit() {
        while (!admission.empty()) {
            Domain& d = domains.at(admission.front());
            if (reserved + d.reserved > budget && reserved > 0) break;
            reserved += d.reserved;
            d.state = DomainState::Admitted;
            setups.push_back(admission.front());
            admission.pop_front();
        }
    }

    void finish(Request& r, hdd_status st) {
        r.done = true;
        r.status = st;
        r.t_done = Clock::now();
        r.rhs.clear();
        r.rhs.shrink_to_fit();
    }

    // Requests of a failed domain complete at once with its status.
    void fail_queued(long long id, Domain& d) {
        for (auto it = queue.begin(); it != queue.end();) {
            Request& r = requests.at(*it);
            if (r.domain == id) {
                finish(r, d.status);
                --d.queued;
                it = queue.erase(it);
            } else {
                ++it;
            }
        }
    }

    void run_setup(long long id, std::unique_lock<std::mutex>& lk) {
        Domain& d = domains.at(id);
        d.state = DomainState::SettingUp;
        ++setting_up;
        hdd_options o = d.opts;
        std::vector<uint32_t> flags;
        flags.swap(d.flags);
        lk.unlock();
        std::unique_ptr<Solver> s;
        hdd_status st = HDD_OK;
        std::string err;
        try {
            s.reset(new Solver(o));
            std::vector<float> zero(flags.size(), 0.0f);
            s->set_domain(flags.data(), zero.data());
            s->initialize();
        } catch (const Error& e) {
            st = e.status;
            err = e.what();
        } catch (const std::bad_alloc&) {
            st = HDD_ERR_OUT_OF_MEMORY;
            err = "host allocation failed";
        } catch (const std::exception& e) {
            st = HDD_ERR_INTERNAL;
            err = e.what();
        }
        if (st != HDD_OK) s.reset();
        lk.lock();
        --setting_up;
        Domain& dd = domains.at(id);
        if (st == HDD_OK) {
            // Count what the solver actually holds from now on.
            const long long actual = (long long)s->device_bytes();
            reserved += actual - dd.reserved;
            dd.reserved = actual;
            dd.solver = std::move(s);
            dd.pool.assign(1, Domain::Ctx{&dd.solver->w0, false});
            dd.batch_k = 1;
            if (opt.batch >= 2) {
                const int kmax = dd.solver->max_batch();
                dd.batch_k = opt.batch >= 4 && kmax >= 4 ? 4 : (kmax >= 2 ? 2 : 1);
            }
            for (int i = 0; i < 3; ++i) dd.ctx_bytes[i] = (long long)dd.solver->work_bytes(1 << i);
            dd.state = DomainState::Resident;
        } else {
            reserved -= dd.reserved;
            dd.reserved = 0;
            dd.state = DomainState::Failed;
            dd.status = st;
            dd.error = err;
            fail_queued(id, dd);
            admit();
        }
    }

    // Requests of domain `dom` in the queue.
    int waiting_for(long long dom) const {
        int n = 0;
        for (long long q : queue)
            if (requests.at(q).domain == dom) ++n;
        return n;
    }

    // Whether a queued request of `d` can start a driver now: more of its
    // requests wait than its running drivers have free systems (those take
    // them at their next iteration), fewer than `slots` drivers on the
    // domain, and an idle context or room in the budget for a new one of one
    // system.
    bool can_run(const Domain& d, long long dom) const {
        if (d.state != DomainState::Resident || d.running >= opt.slots) return false;
        if (d.running > 0 && waiting_for(dom) <= d.capacity - d.held) return false;
        for (const Domain::Ctx& c : d.pool)
            if (!c.busy) return true;
        return reserved + d.ctx_bytes[0] <= budget;
    }

    // Feeds a driver: the request it started with, then every request of its
    // domain that is queued when one of its systems is free.
    struct Feeder : hdd::BatchFeeder {
        hdd_server* srv = nullptr;
        long long dom = 0;
        long long first_id = 0;
        std::vector<float> first_rhs;
        bool first_taken = false;
        std::map<long long, std::vector<float>> rhs;  // kept until the request ends
        bool next(const float** out, long long* id) override {
            if (!first_taken) {
                first_taken = true;
                rhs[first_id] = std::move(first_rhs);
                *out = rhs[first_id].data();
                *id = first_id;
                return true;
            }
            std::lock_guard<std::mutex> lk(srv->mu);
            if (srv->stop) return false;
            for (auto it = srv->queue.begin(); it != srv->queue.end(); ++it) {
                Request& r = srv->requests.at(*it);
                if (r.domain != dom) continue;
                const long long rid = *it;
                srv->queue.erase(it);
                ++srv->domains.at(dom).held;
                std::vector<float>& v = rhs[rid];
                v.swap(r.rhs);
                *out = v.data();
                *id = rid;
                return true;
            }
            return false;
        }
        void done(long long id, hdd_status st, const hdd_result& res, std::vector<float>&& x) override {
            rhs.erase(id);
            std::lock_guard<std::mutex> lk(srv->mu);
            Request& r = srv->requests.at(id);
            r.result = res;
            r.x = std::move(x);
            srv->finish(r, st);
            Domain& d = srv->domains.at(dom);
            --d.queued;
            --d.held;
            srv->cv.notify_all();
        }
    };

    // A driver for request rid's domain: a context sized by how many of the
    // domain's requests wait (several systems when batching is on and more
    // than one waits, else one), then requests solved continuously on it.
    void run_driver(long long rid, std::unique_lock<std::mutex>& lk) {
        Request& r = requests.at(rid);
        const long long dom = r.domain;
        Domain& d = domains.at(dom);
        // Requests this driver is for: this one and those that the running
        // drivers' free systems will not take.
        const int need = 1 + std::max(0, waiting_for(dom) - (d.capacity - d.held));
        int want = 1;
        if (d.batch_k >= 2 && need >= 2) want = (d.batch_k >= 4 && need >= 3) ? 4 : 2;
        auto slot_of = [](int k) { return k == 1 ? 0 : (k == 2 ? 1 : 2); };
        // An idle context of the wanted size, else a new one if the budget
        // allows, else any idle context, else a new one of one system (which
        // can_run guaranteed).
        int pick = -1, make_k = 0;
        for (size_t i = 0; i < d.pool.size() && pick < 0; ++i)
            if (!d.pool[i].busy && d.pool[i].w->k == want) pick = (int)i;
        if (pick < 0 && reserved + d.ctx_bytes[slot_of(want)] <= budget) make_k = want;
        for (size_t i = 0; i < d.pool.size() && pick < 0 && !make_k; ++i)
            if (!d.pool[i].busy) pick = (int)i;
        if (pick < 0 && !make_k) make_k = 1;
        Work* w = nullptr;
        long long mb = 0;
        if (pick >= 0) {
            d.pool[pick].busy = true;
            w = d.pool[pick].w;
        } else {
            mb = d.ctx_bytes[slot_of(make_k)];
            d.reserved += mb;
            reserved += mb;
        }
        ++d.running;
        const int cap = pick >= 0 ? w->k : make_k;
        d.capacity += cap;
        ++d.held;  // the request it starts with
        Solver* s = d.solver.get();
        Feeder feed;
        feed.srv = this;
        feed.dom = dom;
        feed.first_id = rid;
        feed.first_rhs.swap(r.rhs);
        lk.unlock();
        std::unique_ptr<Work> made;
        hdd_status st = HDD_OK;
        try {
            if (!w) {
                made = s->make_work(make_k);
                w = made.get();
            }
            s->solve_batch(*w, feed);
        } catch (const Error& e) {
            st = e.status;
        } catch (const std::bad_alloc&) {
            st = HDD_ERR_OUT_OF_MEMORY;
        } catch (const std::exception&) {
            st = HDD_ERR_INTERNAL;
        }
        lk.lock();
        Domain& dd = domains.at(dom);
        if (made) {
            dd.pool.push_back(Domain::Ctx{made.get(), false});
            dd.owned.push_back(std::move(made));
        } else if (pick >= 0) {
            dd.pool[pick].busy = false;
        } else {
            // The context could not be made: give its reservation back.
            dd.reserved -= mb;
            reserved -= mb;
        }
        // The first request fails with the driver if it never reached a system.
        if (!feed.first_taken) {
            finish(requests.at(rid), st == HDD_OK ? HDD_ERR_INTERNAL : st);
            --dd.queued;
            --dd.held;
        }
        dd.capacity -= cap;
        --dd.running;
    }

    // Index in `queue` of the oldest request whose domain can run now, or -1.
    long long runnable() {
        for (size_t i = 0; i < queue.size(); ++i) {
            const long long dom = requests.at(queue[i]).domain;
            if (can_run(domains.at(dom), dom)) return (long long)i;
        }
        return -1;
    }

    // Solves go first (they hold device state that is already paid for); at
    // most slots - 1 workers set up domains while others could solve.
    bool may_set_up() const {
        return !setups.empty() && (setting_up < std::max(1, opt.slots - 1) || queue.empty());
    }

    void worker() {
        cudaSetDevice(opt.device);
        omp_set_num_threads(opt.setup_threads);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            long long qi = -1;
            cv.wait(lk, [&] {
                qi = runnable();
                return stop || qi >= 0 || may_set_up();
            });
            if (stop) return;
            if (qi >= 0) {
                const long long rid = queue[(size_t)qi];
                queue.erase(queue.begin() + qi);
                run_driver(rid, lk);
            } else {
                const long long id = setups.front();
                setups.pop_front();
                run_setup(id, lk);
            }
            cv.notify_all();
        }
    }
};

namespace {
template <class F>
hdd_status guarded(hdd_server* srv, F&& f) {
    if (!srv) return HDD_ERR_INVALID_ARGUMENT;
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return HDD_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return HDD_ERR_INTERNAL;
    }
}
}  // namespace

extern "C" {

void hdd_server_options_default(hdd_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->slots = 4;
    o->hbm_budget_bytes = 0;
    o->device = 0;
    o->setup_threads = 0;
    o->batch = 0;
}

hdd_status hdd_server_create(const hdd_server_options* o, hdd_server** out) {
    if (!o || !out || o->slots < 1 || o->slots > 64 || o->hbm_budget_bytes < 0 || o->setup_threads < 0 ||
        o->batch < 0 || o->batch > 4)
        return HDD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HDD_ERR_CUDA;
    if (o->device < 0 || o->device >= ndev) return HDD_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(o->device) != cudaSuccess) return HDD_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return HDD_ERR_CUDA;
    hdd_server* srv = new (std::nothrow) hdd_server();
    if (!srv) return HDD_ERR_OUT_OF_MEMORY;
    srv->opt = *o;
    if (srv->opt.setup_threads == 0)
        srv->opt.setup_threads = std::max(1, omp_get_num_procs() / srv->opt.slots);
    srv->budget = o->hbm_budget_bytes > 0 ? o->hbm_budget_bytes : (long long)(0.9 * (double)free_b);
    try {
        for (int i = 0; i < o->slots; ++i) srv->workers.emplace_back([srv] { srv->worker(); });
    } catch (...) {
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->stop = true;
        }
        srv->cv.notify_all();
        for (auto& t : srv->workers) t.join();
        delete srv;
        return HDD_ERR_INTERNAL;
    }
    *out = srv;
    return HDD_OK;
}

hdd_status hdd_server_add_domain(hdd_server* srv, const hdd_options* opts, const uint32_t* flags,
                                 long long* domain_id) {
    if (!opts || !flags || !domain_id) return HDD_ERR_INVALID_ARGUMENT;
    for (int a = 0; a < 3; ++a)
        if (opts->size[a] < 3 || opts->sub_size[a] < 1) return HDD_ERR_INVALID_ARGUMENT;
    return guarded(srv, [&] {
        Domain d;
        d.opts = *opts;
        d.opts.device = srv->opt.device;
        const size_t n = (size_t)opts->size[0] * opts->size[1] * opts->size[2];
        d.flags.assign(flags, flags + n);
        d.reserved = estimate_bytes(d.opts, flags);
        std::lock_guard<std::mutex> lk(srv->mu);
        if (d.reserved > srv->budget) return HDD_ERR_OUT_OF_MEMORY;
        const long long id = srv->next_id++;
        srv->domains.emplace(id, std::move(d));
        srv->admission.push_back(id);
        srv->admit();
        *domain_id = id;
        srv->cv.notify_all();
        return HDD_OK;
    });
}

hdd_status hdd_server_domain_status(hdd_server* srv, long long domain_id, int wait_ms) {
    return guarded(srv, [&] {
        std::unique_lock<std::mutex> lk(srv->mu);
        auto settled = [&] {
            auto it = srv->domains.find(domain_id);
            return it == srv->domains.end() || it->second.state == DomainState::Resident ||
                   it->second.state == DomainState::Failed;
        };
        if (wait_ms < 0) srv->cv.wait(lk, settled);
        else if (wait_ms > 0) srv->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), settled);
        auto it = srv->domains.find(domain_id);
        if (it == srv->domains.end()) return HDD_ERR_NOT_FOUND;
        if (it->second.state == DomainState::Resident) return HDD_OK;
        if (it->second.state == DomainState::Failed) return it->second.status;
        return HDD_ERR_BUSY;
    });
}

hdd_status hdd_server_submit(hdd_server* srv, long long domain_id, const float* rhs, long long* request_id) {
    if (!rhs || !request_id) return HDD_ERR_INVALID_ARGUMENT;
    return guarded(srv, [&] {
        size_t n = 0;
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            auto it = srv->domains.find(domain_id);
            if (it == srv->domains.end() || it->second.removing) return HDD_ERR_NOT_FOUND;
            const int* sz = it->second.opts.size;
            n = (size_t)sz[0] * sz[1] * sz[2];
        }
        Request r;
        r.domain = domain_id;
        r.rhs.assign(rhs, rhs + n);  // copied outside the lock
        r.t_submit = Clock::now();
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->domains.find(domain_id);
        if (it == srv->domains.end() || it->second.removing) return HDD_ERR_NOT_FOUND;
        const long long id = srv->next_id++;
        if (it->second.state == DomainState::Failed) {
            srv->finish(r, it->second.status);
            srv->requests.emplace(id, std::move(r));
        } else {
            ++it->second.queued;
            srv->requests.emplace(id, std::move(r));
            srv->queue.push_back(id);
        }
        *request_id = id;
        srv->cv.notify_all();
        return HDD_OK;
    });
}

hdd_status hdd_server_poll(hdd_server* srv, long long request_id, int wait_ms, hdd_result* result, float* x,
                           double* latency_ms) {
    return guarded(srv, [&] {
        std::unique_lock<std::mutex> lk(srv->mu);
        auto done = [&] {
            auto it = srv->requests.find(request_id);
            return it == srv->requests.end() || it->second.done;
        };
        if (wait_ms < 0) srv->cv.wait(lk, done);
        else if (wait_ms > 0) srv->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), done);
        auto it = srv->requests.find(request_id);
        if (it == srv->requests.end()) return HDD_ERR_NOT_FOUND;
        Request& r = it->second;
        if (!r.done) return HDD_ERR_BUSY;
        if (result) *result = r.result;
        if (x && !r.x.empty()) std::memcpy(x, r.x.data(), r.x.size() * sizeof(float));
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
        const hdd_status st = r.status;
        srv->requests.erase(it);
        return st;
    });
}

hdd_status hdd_server_remove_domain(hdd_server* srv, long long domain_id) {
    return guarded(srv, [&] {
        std::unique_ptr<Solver> s;
        std::vector<std::unique_ptr<Work>> extra;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            auto it = srv->domains.find(domain_id);
            if (it == srv->domains.end() || it->second.removing) return HDD_ERR_NOT_FOUND;
            it->second.removing = true;
            srv->cv.wait(lk, [&] {
                const Domain& d = srv->domains.at(domain_id);
                return srv->stop || (d.queued == 0 && d.running == 0 && d.state != DomainState::SettingUp &&
                                     d.state != DomainState::Admitted);
            });
            if (srv->stop) return HDD_ERR_BUSY;
            Domain& d = srv->domains.at(domain_id);
            if (d.state == DomainState::Waiting) {
                auto a = std::find(srv->admission.begin(), srv->admission.end(), domain_id);
                if (a != srv->admission.end()) srv->admission.erase(a);
            } else {
                srv->reserved -= d.reserved;
            }
            s = std::move(d.solver);
            extra.swap(d.owned);
            srv->domains.erase(domain_id);
            srv->admit();
            srv->cv.notify_all();
        }
        extra.clear();  // device memory freed outside the lock, contexts before the solver they read
        s.reset();
        return HDD_OK;
    });
}

hdd_status hdd_server_memory(hdd_server* srv, long long* reserved, long long* budget) {
    if (!reserved || !budget) return HDD_ERR_INVALID_ARGUMENT;
    return guarded(srv, [&] {
        std::lock_guard<std::mutex> lk(srv->mu);
        *reserved = srv->reserved;
        *budget = srv->budget;
        return HDD_OK;
    });
}

hdd_status hdd_server_domain_error(hdd_server* srv, long long domain_id, char* message, int capacity) {
    if (!message || capacity < 1) return HDD_ERR_INVALID_ARGUMENT;
    return guarded(srv, [&] {
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->domains.find(domain_id);
        if (it == srv->domains.end()) return HDD_ERR_NOT_FOUND;
        std::strncpy(message, it->second.error.c_str(), (size_t)capacity - 1);
        message[capacity - 1] = 0;
        return HDD_OK;
    });
}

void hdd_server_destroy(hdd_server* srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
    }
    srv->cv.notify_all();
    for (auto& t : srv->workers) t.join();
    cudaSetDevice(srv->opt.device);
    delete srv;
}

}  // extern "C"
