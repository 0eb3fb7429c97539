// evp_engine.h -- the equilibrium-iteration engine: one or many solves advanced by batched launches.
//
// Per equilibrium iteration (LS-EVPFFT.f90:233-359) the engine queues, for all its
// members at once, one launch per pass of the iteration (stress average, the five
// spectral passes, correction, local Newton) and per kernel variant those members
// need (radix set, FP64 / FP32 spectrum, Newton kernel), then k_control, which does
// every member's serial tail on the device.  Each member's blocks run the body of
// its single-solve kernel on its own grid and tile, so a solve gives the same bits
// alone and in a batch.  Without a per-kernel timer the iterations are captured
// once in a CUDA graph and replayed; the host reads the members' event codes only
// every few iterations.
#pragma once
#include "evp_dev.cuh"

#include <cuda_runtime.h>

#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

namespace evp {

// A failed solve: the message and the status code the C ABI returns (include/evp.h).
struct SolveError : std::runtime_error {
    int code;
    SolveError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

// The library's device memory pool of the current device (stream-ordered allocations that
// stay with the process instead of going back to the driver at every synchronisation).
cudaMemPool_t solver_pool();

class Engine {
public:
    struct Member {
        BatchSolve e;
        int modal;  // modified augmented Lagrangian (selects the Newton kernel)
        int prec;   // 1: the member may run FP32 spectra (mixed precision)
    };
    using Timer = std::function<void(const char*, const std::function<void()>&)>;

    explicit Engine(cudaStream_t st) : st_(st) {}
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // New membership: member shapes, job tables and descriptors are rebuilt and uploaded.
    void set_members(const std::vector<Member>& m);
    // A member's descriptor changed (its Dev: the Green-operator table flag of a new process).
    void update_entry(int i, const BatchSolve& e);
    // Queue k iterations of every member that is iterating.  timer (may be null) wraps each
    // launch, for per-kernel device times; without it the k iterations run as one CUDA graph
    // (one graph per k, captured at its first use).
    void launch(int k, const Timer* timer);
    // The members' event codes (EV_RUNNING, EV_CONVERGED, EV_ACCEPTED, EV_HOST or a status
    // code) after the queued work; synchronises the stream.
    const int* read_events();
    int size() const { return (int)members_.size(); }
    // kernels one iteration launches (batched passes and the controller)
    int launches_per_iteration() const { return (int)plan_.size() + 1; }
    // device pointer of a member's event code (k_control writes it)
    cudaStream_t stream() const { return st_; }

private:
    void launch_one_iteration(const Timer* timer);
    void drop_graph();
    template <class T>
    T* grow(T* p, size_t& cap, size_t n);

    struct Launch {
        BatchLaunch L;
        BatchParams P;             // the launch's members (kernel parameter)
        std::vector<int> members;  // their indices in the membership
    };
    cudaStream_t st_;
    std::vector<Member> members_;
    std::vector<Launch> plan_;
    BatchSolve* dE_ = nullptr;  // every member's descriptor, for k_control
    int* dEv_ = nullptr;
    int* hEv_ = nullptr;
    size_t capE_ = 0, capEv_ = 0;
    std::vector<cudaGraphExec_t> graphs_;  // graphs_[k]: k iterations captured (null until first used)
};

}  // namespace evp
