// The batched form of MBIR3 (src/mbir3.cpp:47-135 per request): many
// reconstructions of uneven size run through one pipeline on one GPU.
//
// Preparer threads take the requests largest first (by estimated footprint),
// each while the sum of the estimated footprints of the prepared and running
// requests fits in the HBM budget, and run their setup (normalisation, padding, setup adjoints,
// Toeplitz operators, Lipschitz constant) on low-priority streams.  One solver
// thread drives every prepared request's NAG solve: each request keeps one
// line-search step in flight on its own high-priority stream (graph replays
// of the gradient and the loss, plus the asynchronous read of the step's
// reductions); the thread polls the streams, decides a step as soon as its
// read has landed and queues the next one at once.  The GPU works on all
// requests' steps while the host decides, setup kernels fill the gaps, and a
// finished request releases its memory at once, which admits the next one.
#pragma once

#include <array>
#include <vector>

#include "mbir.cuh"

namespace lamino {

struct BatchRequest {
    // inputs (host, valid for the whole call)
    std::vector<const float *> projs;  // (nproj, nrows, ncols) each
    std::vector<std::array<int64_t, 3>> pdims;
    std::vector<const float *> angles;  // nproj each
    std::vector<float> gammas;
    Dims3 recon{};
    ReconParams prm;
    float *out = nullptr;  // host, 3 * recon voxels
    // results
    MbirPhases phases;
    int iterations = 0;
    double t_ready = 0, t_done = 0;  // seconds after the call started: prepared, finished
};

struct BatchStats {
    int64_t peak_in_use = 0;  // estimated device bytes held at once
    int peak_live = 0;        // requests solving at once
    int64_t steps = 0;        // line-search steps decided by the solver thread
    double wall_s = 0;
};

// Runs every request (MBIR3) to completion.  budget: device bytes the
// prepared and running requests may hold together (estimated footprints);
// threads: preparer threads.  Throws on the first failure (the requests
// already running are finished or released first).
void mbir3_batch(std::vector<BatchRequest> &reqs, int64_t budget, int threads, BatchStats *stats);

}  // namespace lamino
