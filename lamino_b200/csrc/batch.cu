// The batched form of MBIR3 (see batch.cuh).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>

#include "batch.cuh"

namespace lamino {

namespace {

double clock_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One request on the device: its streams, inputs, output and job.  Members are
// destroyed in reverse order: the job (its buffers, freed on the streams they
// were allocated on), the inputs and output, then the streams.
struct Slot {
    struct Streams {
        cudaStream_t prep = nullptr, solve = nullptr;
        ~Streams() {
            if (prep) cudaStreamDestroy(prep);
            if (solve) cudaStreamDestroy(solve);
        }
    } st;
    size_t idx = 0;
    int64_t footprint = 0;
    std::vector<DevBuf<float>> proj;
    DevBuf<float> out;
    std::unique_ptr<MbirJob> job;
    bool inflight = false;  // a line-search step is queued and not yet decided
    ~Slot() {
        // the job's last work ran on the solve stream; let it drain before the
        // buffers go back to the pool on their own streams
        if (st.solve) cudaStreamSynchronize(st.solve);
    }
};

}  // namespace

void mbir3_batch(std::vector<BatchRequest> &reqs, int64_t budget, int threads, BatchStats *stats) {
    if (budget <= 0) throw Error(ERR_ARG, "batch budget must be positive");
    if (threads <= 0 || threads > 64) throw Error(ERR_ARG, "batch preparer threads must be 1..64");
    const size_t N = reqs.size();
    std::vector<int64_t> fp(N);
    for (size_t i = 0; i < N; ++i) {
        const BatchRequest &r = reqs[i];
        if (r.projs.empty() || r.projs.size() != r.pdims.size() || r.projs.size() != r.angles.size() ||
            r.projs.size() != r.gammas.size())
            throw Error(ERR_ARG, "batch request " + std::to_string(i) + ": inconsistent dataset lists");
        if (!r.out) throw Error(ERR_ARG, "batch request " + std::to_string(i) + ": null output");
        fp[i] = mbir_footprint(3, r.pdims, r.recon, r.prm);
        if (fp[i] > budget)
            throw Error(ERR_OOM, "batch request " + std::to_string(i) + " needs an estimated " +
                                     std::to_string(fp[i]) + " device bytes, more than the budget of " +
                                     std::to_string(budget));
    }
    BatchStats st;
    const double t0 = clock_s();
    if (N == 0) {
        if (stats) *stats = st;
        return;
    }
    int dev = 0, least = 0, greatest = 0;
    LAMINO_CUDA(cudaGetDevice(&dev));
    LAMINO_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    // keep up to the budget cached in the stream-ordered pool while the batch
    // runs (a finished request's memory serves the next setup without going
    // back to the driver); the previous threshold comes back at the end
    struct PoolKeep {
        cudaMemPool_t pool = nullptr;
        uint64_t old = 0;
        PoolKeep(int dev, int64_t keep) {
            if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
                cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &old) != cudaSuccess) {
                pool = nullptr;
                cudaGetLastError();
                return;
            }
            uint64_t k = (uint64_t)keep;
            if (k > old) cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &k);
        }
        ~PoolKeep() {
            if (pool) cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &old);
        }
    } pool_keep(dev, budget);

    std::mutex mu;
    std::condition_variable cv;
    // largest first (estimated footprint, which grows with the volume and the
    // projections): the big requests start early instead of running alone at
    // the end of the batch
    std::vector<size_t> order(N);
    for (size_t i = 0; i < N; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return fp[a] > fp[b]; });
    size_t next = 0;       // position in `order` of the next request to prepare
    int64_t in_use = 0;    // footprints of prepared and running requests
    bool abort = false;
    std::exception_ptr err;
    std::deque<std::unique_ptr<Slot>> ready;

    auto fail = [&](std::exception_ptr e) {
        std::lock_guard<std::mutex> lk(mu);
        if (!err) err = e;
        abort = true;
        cv.notify_all();
    };

    auto preparer = [&]() {
        cudaSetDevice(dev);
        for (;;) {
            std::unique_ptr<Slot> sl(new Slot);
            {
                std::unique_lock<std::mutex> lk(mu);
                // in that order; a request waits until it fits beside the others
                // (always admitted when nothing is held)
                cv.wait(lk, [&] { return abort || next == N || in_use == 0 || in_use + fp[order[next]] <= budget; });
                if (abort || next == N) return;
                sl->idx = order[next++];
                sl->footprint = fp[sl->idx];
                in_use += sl->footprint;
                st.peak_in_use = std::max(st.peak_in_use, in_use);
            }
            try {
                BatchRequest &r = reqs[sl->idx];
                LAMINO_CUDA(cudaStreamCreateWithPriority(&sl->st.prep, cudaStreamNonBlocking, least));
                LAMINO_CUDA(cudaStreamCreateWithPriority(&sl->st.solve, cudaStreamNonBlocking, greatest));
                AllocStreamScope scope(sl->st.prep);
                std::vector<Dataset> data;
                sl->proj.resize(r.projs.size());
                for (size_t i = 0; i < r.projs.size(); ++i) {
                    const int64_t cnt = r.pdims[i][0] * r.pdims[i][1] * r.pdims[i][2];
                    if (cnt <= 0 || !r.projs[i] || !r.angles[i])
                        throw Error(ERR_ARG, "batch request " + std::to_string(sl->idx) + ": empty dataset");
                    sl->proj[i].alloc((size_t)cnt);
                    LAMINO_CUDA(cudaMemcpyAsync(sl->proj[i].p, r.projs[i], cnt * 4, cudaMemcpyHostToDevice,
                                                sl->st.prep));
                    data.push_back(Dataset{sl->proj[i].p, r.pdims[i][0], r.pdims[i][1], r.pdims[i][2], r.angles[i],
                                           r.gammas[i]});
                }
                sl->out.alloc((size_t)(3 * r.recon.size()));
                sl->job.reset(new MbirJob(3, data, r.recon, r.prm, sl->out.p, sl->st.prep, sl->st.solve));
                sl->job->prepare();
                r.t_ready = clock_s() - t0;
            } catch (...) {
                fail(std::current_exception());
                std::lock_guard<std::mutex> lk(mu);
                in_use -= sl->footprint;
                return;
            }
            std::lock_guard<std::mutex> lk(mu);
            ready.push_back(std::move(sl));
            cv.notify_all();
        }
    };

    std::vector<std::thread> pool;
    for (int i = 0; i < std::min<int>(threads, (int)N); ++i) pool.emplace_back(preparer);

    // solver: every prepared request keeps one line-search step in flight; a
    // step is decided as soon as its stream has passed the step's read, and the
    // next one is queued at once
    std::vector<std::unique_ptr<Slot>> live;
    size_t finished = 0;
    auto retire = [&](std::unique_ptr<Slot> &sl) {
        BatchRequest &r = reqs[sl->idx];
        sl->job->finish();
        r.phases = last_mbir_phases();
        r.iterations = sl->job->nag()->iterations();
        LAMINO_CUDA(cudaMemcpyAsync(r.out, sl->out.p, sl->out.bytes(), cudaMemcpyDeviceToHost, sl->st.solve));
        LAMINO_CUDA(cudaStreamSynchronize(sl->st.solve));
        r.t_done = clock_s() - t0;
        const int64_t f = sl->footprint;
        sl.reset();
        ++finished;
        std::lock_guard<std::mutex> lk(mu);
        in_use -= f;
        cv.notify_all();
    };
    try {
        while (finished < N) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (live.empty()) cv.wait(lk, [&] { return abort || !ready.empty(); });
                if (abort) break;
                while (!ready.empty()) {
                    live.push_back(std::move(ready.front()));
                    ready.pop_front();
                }
                st.peak_live = std::max(st.peak_live, (int)live.size());
            }
            bool progressed = false;
            for (auto &sl : live) {
                NagSolve *ng = sl->job->nag();
                if (sl->inflight) {
                    const cudaError_t q = cudaStreamQuery(sl->st.solve);
                    if (q == cudaErrorNotReady) continue;
                    LAMINO_CUDA(q);
                    sl->inflight = false;
                    ng->finish();
                    ++st.steps;
                }
                progressed = true;
                if (!ng->done()) {
                    AllocStreamScope scope(sl->st.solve);
                    ng->enqueue();
                    sl->inflight = true;
                } else {
                    retire(sl);
                }
            }
            live.erase(std::remove_if(live.begin(), live.end(), [](const std::unique_ptr<Slot> &p) { return !p; }),
                       live.end());
            if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(10));
        }
    } catch (...) {
        fail(std::current_exception());
    }
    for (auto &t : pool) t.join();
    live.clear();
    ready.clear();
    st.wall_s = clock_s() - t0;
    if (stats) *stats = st;
    if (err) std::rethrow_exception(err);
}

}  // namespace lamino
