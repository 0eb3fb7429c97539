// evp_server.cpp -- resident request loop over a batch of solves (continuous batching).
//
// The reference answers each request with a new solver process
// (utils/run.py:169-196; calibrate.py runs two or three at once,
// calibrate.py:1053-1057).  Here one process keeps a server: requests are parsed on
// the submitting thread and queue; one engine thread owns two Batches (evp_batch.h)
// on the server's GPU.  Between rounds of batched iterations it admits queued requests
// while their device-memory estimates fit the budget (the smallest remaining work
// first: voxels times increments), so requests that arrive while others run join a
// running batch as soon as memory and a slot free up, and their work shares the
// launches of every solve already on the device.  Finished solves (their files
// written) leave the batch at once.  Two batches run side by side: small grids on a
// stream of the highest priority, the others on the lowest, each with its own rounds;
// the second holds a bounded number of voxels, so the shortest large requests run first.
#include "../../include/evp.h"
#include "evp_batch.h"
#include "evp_deck.h"

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <memory>
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
    double work = 0.0;  // voxels x increments of the deck: the admission order
    std::shared_ptr<evp::Deck> deck;
    int state = 0, status = 0, macrosteps = 0;
    long long voxel_iters = 0;
    Clock::time_point t_submit, t_start, t_end;
    std::string error;
};

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

// Solves of at most this many voxels (40^3) run in the small lane: a batch on a stream of the
// device's highest priority, so their short rounds get SMs ahead of the large lane's long ones
// and a small request's latency does not follow the round time of the largest solves.
constexpr long long kSmallLaneVoxels = 40LL * 40 * 40;
// The large lane holds at most this many voxels at once (two 64^3 solves; a larger solve runs
// alone there).  One such solve already fills every launch of an iteration, so admitting more
// would only share the GPU among them (each finishing late) where admitting the least work first
// and few at a time lets the short requests finish early, at the same throughput.
constexpr long long kLargeLaneVoxels = 2LL * 64 * 64 * 64;
static int lane_of(long long voxels) { return voxels <= kSmallLaneVoxels ? 0 : 1; }

struct evp_server {
    std::mutex m;
    std::condition_variable cv;  // any change of queue, admission or completion
    std::deque<unsigned long long> queue;
    std::map<unsigned long long, Request> reqs;
    std::map<std::pair<int, int>, unsigned long long> slot_req;  // (lane, batch slot) -> request
    std::thread engine;
    unsigned long long budget = 0, used = 0, next_id = 1;
    int max_inflight = 16, inflight = 0, device = 0;
    long long lane_vox[2] = {0, 0};  // voxels of the solves running in each lane
    bool closing = false;
    std::string fatal;  // a CUDA failure of the engine: every later request fails with it

    void complete(Request& q, int status, const std::string& err, int macro, long long vi) {
        q.state = 2;
        q.status = status;
        q.error = err;
        q.macrosteps = macro;
        q.voxel_iters = vi;
        q.t_end = Clock::now();
        q.deck.reset();
    }

    // called with the lock held; returns the queued request to admit next, or 0
    unsigned long long pick() {
        unsigned long long best = 0;
        double best_work = 0.0;
        for (auto id : queue) {
            const Request& r = reqs[id];
            if (used + r.foot > budget && inflight > 0) continue;  // a request larger than the budget runs alone
            const long long vox = (long long)r.n1 * r.n2 * r.n3;
            if (lane_of(vox) == 1 && lane_vox[1] > 0 && lane_vox[1] + vox > kLargeLaneVoxels) continue;
            if (best == 0 || r.work < best_work) {
                best = id;
                best_work = r.work;
            }
        }
        return best;
    }

    void engine_loop() {
        cudaSetDevice(device);
        using BatchPtr = std::unique_ptr<evp::Batch, void (*)(evp::Batch*)>;
        BatchPtr lane[2] = {BatchPtr(nullptr, evp::batch_destroy), BatchPtr(nullptr, evp::batch_destroy)};
        try {
            int lowest = 0;
            const int highest = evp::batch_priority_range(&lowest);
            lane[0].reset(evp::batch_create(highest));
            lane[1].reset(evp::batch_create(lowest));
        } catch (std::exception& e) {
            std::lock_guard<std::mutex> lk(m);
            fatal = e.what();
        }
        const bool ok = lane[0] && lane[1];
        bool pending[2] = {false, false};
        std::unique_lock<std::mutex> lk(m);
        while (true) {
            // admission: smallest remaining work first, while slots and memory allow
            while (ok && inflight < max_inflight && !queue.empty()) {
                const unsigned long long id = pick();
                if (id == 0) break;
                for (auto it = queue.begin(); it != queue.end(); ++it)
                    if (*it == id) {
                        queue.erase(it);
                        break;
                    }
                Request& r = reqs[id];
                used += r.foot;
                inflight++;
                r.state = 1;
                r.t_start = Clock::now();
                std::shared_ptr<evp::Deck> dk = r.deck;
                const std::string fft = r.fft, out = r.out;
                const int mix = r.mix, modal = r.modal, flags = r.flags;
                const double dl = r.deadline_s;
                const long long vox = (long long)r.n1 * r.n2 * r.n3;
                const int l = lane_of(vox);
                lane_vox[l] += vox;
                lk.unlock();
                std::string err;
                int slot = -1;
                try {
                    slot = evp::batch_add(lane[l].get(), std::move(*dk), fft, out, mix, modal, flags, dl, err);
                } catch (std::exception& e) {
                    err = e.what();
                }
                lk.lock();
                Request& q = reqs[id];
                int status = 0;
                evp_report rep{};
                const int st = slot >= 0 ? evp::batch_slot(lane[l].get(), slot, &status, &rep, &err) : 1;
                if (slot < 0) status = -6;
                if (st == 1) {  // failed at start-up (or a deck without steps)
                    complete(q, status, err, rep.macrosteps, rep.voxel_iters);
                    if (slot >= 0) evp::batch_remove(lane[l].get(), slot);
                    used -= q.foot;
                    lane_vox[l] -= vox;
                    inflight--;
                    cv.notify_all();
                } else {
                    slot_req[{l, slot}] = id;
                }
            }
            if (!ok) {  // no device: fail what is queued
                for (auto id : queue) complete(reqs[id], -6, fatal, 0, 0);
                queue.clear();
                cv.notify_all();
                if (closing) return;
                cv.wait(lk, [&] { return closing || !queue.empty(); });
                continue;
            }
            if (inflight == 0) {
                if (closing && queue.empty()) break;
                cv.wait(lk, [&] { return closing || !queue.empty(); });
                continue;
            }
            lk.unlock();
            // keep a round queued on each lane that has members; finish whichever is done first
            std::string step_err;
            try {
                for (int l = 0; l < 2; l++)
                    if (!pending[l]) pending[l] = evp::batch_launch(lane[l].get());
                bool any = false;
                while (!any && (pending[0] || pending[1])) {
                    for (int l = 0; l < 2; l++)
                        if (pending[l] && evp::batch_ready(lane[l].get())) {
                            evp::batch_finish(lane[l].get());
                            pending[l] = false;
                            any = true;
                        }
                    if (!any) std::this_thread::sleep_for(std::chrono::microseconds(20));
                }
            } catch (std::exception& e) {
                step_err = e.what();
                pending[0] = pending[1] = false;
            }
            lk.lock();
            for (auto it = slot_req.begin(); it != slot_req.end();) {
                int status = 0;
                evp_report rep{};
                std::string err;
                evp::Batch* b = lane[it->first.first].get();
                const int st = evp::batch_slot(b, it->first.second, &status, &rep, &err);
                if (st == 1 || !step_err.empty()) {
                    Request& q = reqs[it->second];
                    if (st != 1) {
                        status = -6;
                        err = step_err;
                    }
                    complete(q, status, err, rep.macrosteps, rep.voxel_iters);
                    if (st == 1 || !pending[it->first.first]) evp::batch_remove(b, it->first.second);
                    used -= q.foot;
                    lane_vox[it->first.first] -= (long long)q.n1 * q.n2 * q.n3;
                    inflight--;
                    it = slot_req.erase(it);
                } else {
                    ++it;
                }
            }
            cv.notify_all();
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
    if (!out) return srv_fail("evp_server_open: null argument", -7);
    if (tune_cache && tune_cache[0] && evp_tune_cache(tune_cache) != 0) return -7;
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
    s->engine = std::thread([s] { s->engine_loop(); });
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
    r.t_submit = Clock::now();
    // the deck is read here, on the submitting thread, so that admission only does device work
    std::string perr;
    int pcode = 0;
    try {
        r.deck = std::make_shared<evp::Deck>(evp::parse_deck(r.fft));
        r.n1 = r.deck->n1;
        r.n2 = r.deck->n2;
        r.n3 = r.deck->n3;
        long long steps = 0;
        for (auto& p : r.deck->process) steps += p.nsteps;
        r.work = (double)r.deck->nvox() * (double)(steps > 0 ? steps : 1);
    } catch (evp::DeckError& e) {
        perr = e.what();
        pcode = e.code;
    } catch (std::exception& e) {
        perr = e.what();
        pcode = -1;
    }
    r.foot = footprint(r.n1 > 0 ? r.n1 : 1, r.n2 > 0 ? r.n2 : 1, r.n3 > 0 ? r.n3 : 1);
    std::lock_guard<std::mutex> lk(srv->m);
    if (srv->closing) return srv_fail("evp_submit: server is closing", -7);
    r.id = srv->next_id++;
    *ticket = r.id;
    if (pcode != 0) {  // a deck error: the request is done at once with the parser's status
        srv->complete(r, pcode, perr, 0, 0);
        srv->reqs[r.id] = r;
    } else {
        srv->reqs[r.id] = r;
        srv->queue.push_back(r.id);
    }
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
    if (srv->engine.joinable()) srv->engine.join();
    delete srv;
    return 0;
}

}  // extern "C"
