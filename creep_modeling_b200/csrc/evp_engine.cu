// evp_engine.cu -- batched equilibrium iterations over one or many solves (see evp_engine.h).
#include "evp_engine.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

namespace evp {

#define ECK(x)                                                                                             \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess) throw SolveError(std::string("CUDA error: ") + cudaGetErrorString(e_), -6); \
    } while (0)

cudaMemPool_t solver_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw SolveError("cudaGetDevice failed", -6);
    static std::mutex m;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(m);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    ECK(cudaMemPoolCreate(&pool, &props));
    unsigned long long keep = ~0ull;
    ECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools.emplace(dev, pool);
    return pool;
}

static const char* kind_name(int k) {
    static const char* names[BK_N] = {"k_fft_x_fwd", "k_fft_y_fwd", "k_fft_z_green", "k_fft_y_inv",
                                      "k_fft_x_inv", "k_corr", "k_newton"};
    return (k >= 0 && k < BK_N) ? names[k] : "k_batched";
}
static bool fft_kind(int k) { return k == BK_XFWD || k == BK_YFWD || k == BK_ZGREEN || k == BK_YINV || k == BK_XINV; }

Engine::~Engine() {
    drop_graph();
    if (dE_) cudaFreeAsync(dE_, st_);
    if (dEv_) cudaFreeAsync(dEv_, st_);
    if (hEv_) cudaFreeHost(hEv_);
}

void Engine::drop_graph() {
    for (auto& g : graphs_)
        if (g) cudaGraphExecDestroy(g);
    graphs_.clear();
}

template <class T>
T* Engine::grow(T* p, size_t& cap, size_t n) {
    if (n <= cap && p) return p;
    size_t c = std::max<size_t>(n, 2 * cap);
    if (p) ECK(cudaFreeAsync(p, st_));
    void* q = nullptr;
    ECK(cudaMallocFromPoolAsync(&q, c * sizeof(T), solver_pool(), st_));
    cap = c;
    drop_graph();  // the captured launches hold the old pointers
    return (T*)q;
}

void Engine::set_members(const std::vector<Member>& m) {
    members_ = m;
    const int n = (int)m.size();
    std::vector<MemberJobs> mj(n);
    for (int i = 0; i < n; i++) {
        std::memset(&mj[i], 0, sizeof(MemberJobs));
        member_jobs_voxel(m[i].e.d, m[i].modal, mj[i]);
        member_jobs_fft(m[i].e.d, m[i].e.pl1, m[i].e.pl2, m[i].e.pl3, m[i].prec, mj[i]);
    }
    // one launch per pass, spectral precision and kernel variant (and per kBatchChunk members),
    // members in membership order
    plan_.clear();
    for (int k = 0; k < BK_N; k++) {
        for (int w = 0; w < (fft_kind(k) ? 2 : 1); w++) {
            std::map<int, std::vector<int>> byvar;
            for (int i = 0; i < n; i++) {
                if (w == 1 && !mj[i].has32) continue;
                byvar[mj[i].variant[w][k]].push_back(i);
            }
            for (auto& kv : byvar) {
                for (size_t c0 = 0; c0 < kv.second.size(); c0 += kBatchChunk) {
                    plan_.emplace_back();
                    Launch& ln = plan_.back();
                    std::memset(&ln.P, 0, sizeof(BatchParams));
                    ln.L = BatchLaunch{};
                    ln.L.kind = k;
                    ln.L.variant = kv.first;
                    long long blocks = 0;
                    for (size_t c = c0; c < std::min(kv.second.size(), c0 + (size_t)kBatchChunk); c++) {
                        const int i = kv.second[c];
                        const int q = ln.P.njobs++;
                        Job j = mj[i].job[w][k];
                        j.solve = q;
                        j.blk0 = (int)blocks;
                        blocks += (long long)j.gx * j.gy * j.gz;
                        ln.P.jobs[q] = j;
                        ln.P.E[q] = m[i].e;
                        ln.members.push_back(i);
                        ln.L.threads = std::max(ln.L.threads, mj[i].threads[w][k]);
                        ln.L.smem = std::max(ln.L.smem, mj[i].smem[w][k]);
                    }
                    if (blocks >= (1LL << 31)) throw SolveError("batched launch larger than the grid limit", -7);
                    ln.L.blocks = (int)blocks;
                    ln.L.njobs = ln.P.njobs;
                }
            }
        }
    }
    drop_graph();
    if (n == 0) return;
    dE_ = grow(dE_, capE_, (size_t)n);
    dEv_ = grow(dEv_, capEv_, (size_t)n);
    std::vector<BatchSolve> E(n);
    for (int i = 0; i < n; i++) E[i] = m[i].e;
    ECK(cudaMemcpyAsync(dE_, E.data(), n * sizeof(BatchSolve), cudaMemcpyHostToDevice, st_));
    if (hEv_) cudaFreeHost(hEv_);
    hEv_ = nullptr;
    ECK(cudaMallocHost(&hEv_, n * sizeof(int)));
}

void Engine::update_entry(int i, const BatchSolve& e) {
    if (std::memcmp(&members_[i].e, &e, sizeof(BatchSolve)) == 0) return;
    members_[i].e = e;
    for (Launch& ln : plan_)
        for (size_t q = 0; q < ln.members.size(); q++)
            if (ln.members[q] == i) ln.P.E[q] = e;
    ECK(cudaMemcpyAsync(dE_ + i, &members_[i].e, sizeof(BatchSolve), cudaMemcpyHostToDevice, st_));
    drop_graph();  // the captured launches carry the old descriptor
}

void Engine::launch_one_iteration(const Timer* timer) {
    for (const Launch& ln : plan_) {
        if (ln.L.blocks == 0) continue;
        auto f = [&] {
            if (fft_kind(ln.L.kind)) launch_batched_fft(ln.L, ln.P, st_);
            else launch_batched_voxel(ln.L, ln.P, st_);
        };
        if (timer) (*timer)(kind_name(ln.L.kind), f);
        else f();
    }
    auto c = [&] { launch_control(dE_, (int)members_.size(), dEv_, st_); };
    if (timer) (*timer)("k_control", c);
    else c();
}

void Engine::launch(int k, const Timer* timer) {
    if (members_.empty() || k <= 0) return;
    if (timer) {
        for (int i = 0; i < k; i++) launch_one_iteration(timer);
        ECK(cudaGetLastError());
        return;
    }
    if ((int)graphs_.size() <= k) graphs_.resize(k + 1, nullptr);
    cudaGraphExec_t& graph_ = graphs_[k];
    if (!graph_) {
        cudaGraph_t g = nullptr;
        ECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < k; i++) launch_one_iteration(nullptr);
        const cudaError_t e1 = cudaGetLastError();
        const cudaError_t e2 = cudaStreamEndCapture(st_, &g);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            throw SolveError(std::string("CUDA graph capture failed: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2), -6);
        }
        const cudaError_t e3 = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            graph_ = nullptr;
            throw SolveError(std::string("CUDA graph instantiation failed: ") + cudaGetErrorString(e3), -6);
        }
    }
    ECK(cudaGraphLaunch(graph_, st_));
}

const int* Engine::read_events() {
    const int n = (int)members_.size();
    if (n == 0) return hEv_;
    ECK(cudaMemcpyAsync(hEv_, dEv_, n * sizeof(int), cudaMemcpyDeviceToHost, st_));
    ECK(cudaStreamSynchronize(st_));
    return hEv_;
}

}  // namespace evp
