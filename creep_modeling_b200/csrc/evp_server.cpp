// evp_server.cpp -- resident request loop over the solver's C ABI.
//
// The reference answers each request with a new solver process
// (utils/run.py:169-196; calibrate.py runs two or three at once,
// calibrate.py:1053-1057).  Here one process keeps a server: requests queue in
// arrival order, a dispatcher thread admits them while the running solves'
// device-memory estimates fit the budget, and every admitted solve runs on its
// own host thread and CUDA stream (the solver creates a non-blocking stream and
// allocates stream-ordered), so solves of different sizes overlap on the GPU.
#include "../../include/evp.h"

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    unsigned long long id = 0;
    std::string fft, out;
    int mix = 1, modal = 0, precision = 0, flags = EVP_WRITE_FILES;
    double deadline_s = 0.0;  // wall-clock budget from admission (0: none)
    int n1 = 0, n2 = 0, n3 = 0;
    unsigned long long foot = 0;
    int state = 0, status = 0, macrosteps = 0;
    long long voxel_iters = 0;
    Clock::time_point t_submit, t_start, t_end;
    std::string error;
};

// Grid size from the deck's first two records (number of phases; nx ny nz).
bool deck_grid(const std::string& fft, int& n1, int& n2, int& n3) {
    std::ifstream f(fft);
    if (!f) return false;
    std::string line;
    if (!std::getline(f, line)) return false;  // nph
    if (!std::getline(f, line)) return false;
    std::istringstream is(line);
    return (bool)(is >> n1 >> n2 >> n3) && n1 > 0 && n2 > 0 && n3 > 0;
}

// Device memory of one solve, from the solver's allocations with the largest
// slip-system count (24) and every optional field present: about 5.3 kB per
// voxel of state, the half spectrum (9 complex values per half-spectrum point),
// the tabulated Green operator of IGAMMA 1 and 2 (81 doubles per half-spectrum
// point), the node coordinates and fixed buffers.
unsigned long long footprint(int n1, int n2, int n3) {
    const unsigned long long N = (unsigned long long)n1 * n2 * n3;
    const unsigned long long per_voxel = 669ull * 8ull;
    const unsigned long long spec = 9ull * 16ull * (unsigned long long)(n1 / 2 + 1) * n2 * n3;
    const unsigned long long goper = 81ull * 8ull * (unsigned long long)(n1 / 2 + 1) * n2 * n3;
    const unsigned long long nodes = 3ull * 8ull * (n1 + 1ull) * (n2 + 1ull) * (n3 + 1ull);
    const unsigned long long partials = 8ull * (200ull * 2048ull + 9ull * ((unsigned long long)n2 * n3 / 2 + 1));
    return N * per_voxel + spec + goper + nodes + partials + (1ull << 20);
}

double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

}  // namespace

struct evp_server {
    std::mutex m;
    std::condition_variable cv;  // any change of queue, admission or completion
    std::deque<unsigned long long> queue;
    std::map<unsigned long long, Request> reqs;
    std::map<unsigned long long, std::thread> workers;
    std::vector<unsigned long long> finished;  // workers to join
    std::thread dispatcher;
    unsigned long long budget = 0, used = 0, next_id = 1, arrivals = 0;
    int max_inflight = 16, inflight = 0, device = 0;
    bool closing = false;

    void run_one(unsigned long long id) {
        Request r;
        {
            std::lock_guard<std::mutex> lk(m);
            r = reqs[id];
        }
        cudaSetDevice(device);
        int rc = 0, macro = 0;
        long long vi = 0;
        std::string err;
        evp_solve* h = nullptr;
        rc = evp_open(r.fft.c_str(), r.out.c_str(), r.mix, r.modal, r.flags, &h);
        if (rc != 0) {
            err = evp_last_error();
        } else {
            if (r.deadline_s > 0.0) evp_set_deadline(h, r.deadline_s - secs(r.t_start, Clock::now()));
            int done = 0;
            while (true) {
                rc = evp_advance(h, 1, &done);
                if (rc != 0) {
                    err = evp_last_error();
                    break;
                }
                if (done == 0) break;
            }
            evp_report rep{};
            evp_stats(h, &rep);
            macro = rep.macrosteps;
            vi = rep.voxel_iters;
            evp_close(h);
        }
        std::lock_guard<std::mutex> lk(m);
        Request& q = reqs[id];
        q.state = 2;
        q.status = rc;
        q.error = err;
        q.macrosteps = macro;
        q.voxel_iters = vi;
        q.t_end = Clock::now();
        used -= q.foot;
        inflight--;
        finished.push_back(id);
        cv.notify_all();
    }

    // join the threads of finished solves (called with the lock held; drops it while joining)
    void reap(std::unique_lock<std::mutex>& lk) {
        if (finished.empty()) return;
        std::vector<std::thread> done;
        for (auto id : finished) {
            auto it = workers.find(id);
            if (it != workers.end()) {
                done.push_back(std::move(it->second));
                workers.erase(it);
            }
        }
        finished.clear();
        lk.unlock();
        for (auto& t : done) t.join();
        lk.lock();
    }

    void dispatch_loop() {
        std::unique_lock<std::mutex> lk(m);
        while (true) {
            reap(lk);
            cv.wait(lk, [&] { return closing || !queue.empty() || !finished.empty(); });
            reap(lk);
            if (queue.empty()) {
                if (closing && inflight == 0) return;
                if (closing) {
                    cv.wait(lk, [&] { return inflight == 0 || !queue.empty() || !finished.empty(); });
                    reap(lk);
                    if (queue.empty() && inflight == 0) return;
                }
                continue;
            }
            // first request in arrival order that fits beside the running ones
            bool admitted = false;
            for (auto it = queue.begin(); it != queue.end() && inflight < max_inflight; ++it) {
                Request& r = reqs[*it];
                if (used + r.foot > budget && inflight > 0) continue;
                // a request larger than the whole budget runs alone
                used += r.foot;
                inflight++;
                r.state = 1;
                r.t_start = Clock::now();
                const unsigned long long id = *it;
                queue.erase(it);
                workers.emplace(id, std::thread([this, id] { run_one(id); }));
                admitted = true;
                break;
            }
            if (!admitted) {  // until a solve ends or another request arrives
                const unsigned long long a0 = arrivals;
                cv.wait(lk, [&] { return !finished.empty() || arrivals != a0; });
            }
        }
    }
};

namespace evp {
void set_last_error(const std::string& m);
}

static int srv_fail(const std::string& m, int code) {
    evp::set_last_error(m);
    return code;
}

extern "C" {

int evp_server_open(unsigned long long hbm_budget_bytes, int max_inflight, const char* tune_cache, evp_server** out) {
    (void)tune_cache;
    if (!out) return srv_fail("evp_server_open: null argument", -7);
    *out = nullptr;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return srv_fail("no CUDA device available", -6);
    evp_server* s = new evp_server();
    cudaGetDevice(&s->device);
    if (hbm_budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete s;
            return srv_fail("cudaMemGetInfo failed", -6);
        }
        hbm_budget_bytes = (unsigned long long)(0.85 * (double)fr);
    }
    s->budget = hbm_budget_bytes;
    s->max_inflight = max_inflight > 0 ? max_inflight : 16;
    s->dispatcher = std::thread([s] { s->dispatch_loop(); });
    *out = s;
    return 0;
}

int evp_submit(evp_server* srv, const char* fft_in, const char* out_dir, int mix, int modal, int precision, int flags,
               unsigned long long* ticket) {
    return evp_submit_deadline(srv, fft_in, out_dir, mix, modal, precision, flags, 0.0, ticket);
}

int evp_submit_deadline(evp_server* srv, const char* fft_in, const char* out_dir, int mix, int modal, int precision,
                        int flags, double deadline_s, unsigned long long* ticket) {
    if (!srv || !fft_in || !ticket) return srv_fail("evp_submit: null argument", -7);
    if (precision != 0 && precision != 1) return srv_fail("evp_submit: precision must be 0 (plain FP64) or 1 (mixed)", -7);
    if ((flags & (EVP_WRITE_FILES | EVP_WRITE_CSV)) == 0) return srv_fail("evp_submit: flags must ask for EVP_WRITE_FILES or EVP_WRITE_CSV", -7);
    Request r;
    r.fft = fft_in;
    r.out = out_dir ? out_dir : "";
    r.mix = mix;
    r.modal = modal;
    r.precision = precision;
    r.flags = (flags & (EVP_WRITE_FILES | EVP_WRITE_CSV | EVP_VERBOSE)) | (precision == 1 ? EVP_MIXED : 0);
    r.deadline_s = deadline_s > 0.0 ? deadline_s : 0.0;
    if (!deck_grid(r.fft, r.n1, r.n2, r.n3)) return srv_fail("evp_submit: cannot read the grid size from " + r.fft, -1);
    r.foot = footprint(r.n1, r.n2, r.n3);
    r.t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(srv->m);
    if (srv->closing) return srv_fail("evp_submit: server is closing", -7);
    r.id = srv->next_id++;
    srv->reqs[r.id] = r;
    srv->queue.push_back(r.id);
    srv->arrivals++;
    *ticket = r.id;
    srv->cv.notify_all();
    return 0;
}

static void fill(const Request& r, evp_status* st) {
    std::memset(st, 0, sizeof(*st));
    st->state = r.state;
    st->status = r.status;
    st->macrosteps = r.macrosteps;
    st->n1 = r.n1;
    st->n2 = r.n2;
    st->n3 = r.n3;
    st->voxel_iters = r.voxel_iters;
    st->footprint_bytes = r.foot;
    const auto now = Clock::now();
    st->queued_s = secs(r.t_submit, r.state >= 1 ? r.t_start : now);
    st->run_s = r.state >= 1 ? secs(r.t_start, r.state == 2 ? r.t_end : now) : 0.0;
    st->latency_s = secs(r.t_submit, r.state == 2 ? r.t_end : now);
    std::strncpy(st->error, r.error.c_str(), sizeof(st->error) - 1);
}

int evp_poll(evp_server* srv, unsigned long long ticket, evp_status* st) {
    if (!srv || !st) return srv_fail("evp_poll: null argument", -7);
    std::lock_guard<std::mutex> lk(srv->m);
    auto it = srv->reqs.find(ticket);
    if (it == srv->reqs.end()) return srv_fail("evp_poll: unknown ticket", -7);
    fill(it->second, st);
    return 0;
}

int evp_wait(evp_server* srv, unsigned long long ticket, double timeout_s, evp_status* st) {
    if (!srv) return srv_fail("evp_wait: null argument", -7);
    std::unique_lock<std::mutex> lk(srv->m);
    auto it = srv->reqs.find(ticket);
    if (it == srv->reqs.end()) return srv_fail("evp_wait: unknown ticket", -7);
    auto done = [&] { return srv->reqs[ticket].state == 2; };
    bool ok = true;
    if (timeout_s < 0) srv->cv.wait(lk, done);
    else ok = srv->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    if (st) fill(srv->reqs[ticket], st);
    return ok ? 0 : 1;
}

int evp_server_close(evp_server* srv) {
    if (!srv) return 0;
    {
        std::lock_guard<std::mutex> lk(srv->m);
        srv->closing = true;
        srv->cv.notify_all();
    }
    if (srv->dispatcher.joinable()) srv->dispatcher.join();
    for (auto& kv : srv->workers)
        if (kv.second.joinable()) kv.second.join();
    delete srv;
    return 0;
}

}  // extern "C"
