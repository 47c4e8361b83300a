// CUDA-graph capture of repeated operator applications.
//
// Solver loops call the same operator on the same buffers every iteration
// (CG: A(p) -> Ap; split Bregman: (A + mu lap)(p); NAG: grad(y), loss(x)), a
// fixed sequence of 5-20 kernel launches.  GraphedOp runs the first call for a
// given (input, output) pointer pair eagerly (so lazily created buffers and plans
// exist before any capture), records the second with thread-local stream capture
// (concurrent requests on other host threads cannot break it) and replays the
// recorded graph with one cudaGraphLaunch from then on.
#pragma once

#include <map>
#include <set>
#include <utility>

#include "common.cuh"
#include "solvers.cuh"

namespace lamino {

class GraphedOp {
  public:
    explicit GraphedOp(OpFn f, bool enabled = true) : f_(std::move(f)), enabled_(enabled) {}
    ~GraphedOp() {
        for (auto &kv : graphs_) {
            cudaGraphExecDestroy(kv.second.exec);
            cudaGraphDestroy(kv.second.graph);
        }
    }
    GraphedOp(const GraphedOp &) = delete;
    GraphedOp &operator=(const GraphedOp &) = delete;

    void operator()(const float *x, float *y, cudaStream_t s) {
        ++calls_;
        if (!enabled_ || s == nullptr) {  // the legacy default stream cannot be captured
            f_(x, y, s);
            return;
        }
        auto key = std::make_pair(x, (const float *)y);
        auto it = graphs_.find(key);
        if (it == graphs_.end() && seen_.insert(key).second) {
            f_(x, y, s);
            return;
        }
        if (it == graphs_.end()) {
            Entry e{};
            LAMINO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                f_(x, y, s);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            LAMINO_CUDA(cudaStreamEndCapture(s, &e.graph));
            LAMINO_CUDA(cudaGraphInstantiate(&e.exec, e.graph, 0));
            it = graphs_.emplace(key, e).first;
        }
        LAMINO_CUDA(cudaGraphLaunch(it->second.exec, s));
        ++launches_;
    }
    OpFn as_fn() {
        return [this](const float *x, float *y, cudaStream_t s) { (*this)(x, y, s); };
    }
    int graphs() const { return (int)graphs_.size(); }
    long launches() const { return launches_; }
    long calls() const { return calls_; }

  private:
    struct Entry {
        cudaGraph_t graph;
        cudaGraphExec_t exec;
    };
    OpFn f_;
    bool enabled_;
    std::map<std::pair<const float *, const float *>, Entry> graphs_;
    std::set<std::pair<const float *, const float *>> seen_;
    long launches_ = 0, calls_ = 0;
};

}  // namespace lamino
