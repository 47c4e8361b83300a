// Continuous-batching reconstruction server (see server.cuh).
#include <chrono>

#include "server.cuh"

namespace lamino {

double Server::now() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

Server::Server(int64_t budget, int slots, bool dry_run, double dry_run_ms)
    : budget_(budget), slots_(slots), dry_(dry_run), dry_ms_(dry_run_ms) {
    if (budget <= 0) throw Error(ERR_ARG, "server budget must be positive");
    if (slots <= 0 || slots > 256) throw Error(ERR_ARG, "server slots must be 1..256");
    int dev = 0;
    if (!dry_) {
        LAMINO_CUDA(cudaGetDevice(&dev));
        // keep up to the budget cached in the stream-ordered pool between requests
        // (the previous threshold comes back when the server is destroyed: the
        // pool is the whole process's)
        LAMINO_CUDA(cudaDeviceGetDefaultMemPool(&pool_, dev));
        LAMINO_CUDA(cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &old_threshold_));
        uint64_t keep = (uint64_t)budget;
        LAMINO_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    for (int i = 0; i < slots; ++i)
        workers_.emplace_back([this, dev, i]() {
            if (!dry_) cudaSetDevice(dev);
            worker(i);
        });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
        for (int64_t id : queue_) {  // never started: fail them so their waiters return
            ServeRequest *r = reqs_[id].get();
            r->status = ERR_STATE;
            r->err = "server shut down before the request started";
            r->t_start = r->t_done = now();
            r->done = true;
            ++failed_;
        }
        queue_.clear();
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();  // running requests finish first
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return users_ == 0; });
    if (pool_) {
        cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &old_threshold_);
        cudaGetLastError();
    }
}

Server::Use::Use(Server &sv) : s(sv) {
    std::lock_guard<std::mutex> lk(s.mu_);
    if (s.stop_) throw Error(ERR_STATE, "server is shutting down");
    ++s.users_;
}

Server::Use::~Use() {
    // notify under the lock: once it is released the destructor may free `s`
    std::lock_guard<std::mutex> lk(s.mu_);
    --s.users_;
    s.cv_.notify_all();
}

int64_t Server::submit(std::unique_ptr<ServeRequest> r) {
    if (r->footprint > budget_)
        throw Error(ERR_OOM, "request needs an estimated " + std::to_string(r->footprint) +
                                 " device bytes, more than the server budget of " + std::to_string(budget_));
    std::lock_guard<std::mutex> lk(mu_);
    if (stop_) throw Error(ERR_STATE, "server is shutting down");
    r->id = next_id_++;
    if (r->t_submit == 0) r->t_submit = now();
    const int64_t id = r->id;
    reqs_[id] = std::move(r);
    queue_.push_back(id);
    ++submitted_;
    cv_.notify_all();
    return id;
}

void Server::worker(int wid) {
    (void)wid;
    // setup on a low-priority stream, the solve on a high-priority one: the
    // block scheduler gives a running solve's small kernels the SMs ahead of
    // another request's setup kernels
    cudaStream_t s = nullptr, ss = nullptr;
    if (!dry_) {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
            cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, least) != cudaSuccess ||
            cudaStreamCreateWithPriority(&ss, cudaStreamNonBlocking, greatest) != cudaSuccess) {
            if (s) cudaStreamDestroy(s);
            if (ss) cudaStreamDestroy(ss);
            s = ss = nullptr;
        }
    }
    for (;;) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] {
            if (stop_) return true;
            if (queue_.empty()) return false;
            const ServeRequest *h = reqs_[queue_.front()].get();
            return in_use_ + h->footprint <= budget_;  // FIFO: only the head is admitted
        });
        if (stop_) break;
        const int64_t id = queue_.front();
        queue_.pop_front();
        ServeRequest *r = reqs_[id].get();
        in_use_ += r->footprint;
        peak_ = std::max(peak_, in_use_);
        ++active_;
        peak_active_ = std::max(peak_active_, active_);
        r->t_start = now();
        lk.unlock();
        cv_.notify_all();  // another head may fit as well

        int status = OK;
        std::string err;
        const int64_t nv = 3 * r->recon.size();
        try {
            if (dry_) {
                std::this_thread::sleep_for(std::chrono::duration<double, std::milli>(dry_ms_));
                r->result.assign((size_t)nv, 0.f);
            } else {
                if (!s) throw Error(ERR_CUDA, "worker stream creation failed");
                std::vector<DevBuf<float>> dp(r->projs.size());
                std::vector<Dataset> data;
                DevBuf<float> out;
                std::unique_ptr<MbirJob> job;
                // destroyed first, also when a step throws: the solve stream has
                // drained before any buffer goes back to the pool
                struct Drain {
                    cudaStream_t st;
                    ~Drain() { cudaStreamSynchronize(st); }
                } drain{ss};
                {
                    AllocStreamScope scope(s);
                    for (size_t i = 0; i < r->projs.size(); ++i) {
                        dp[i].alloc(r->projs[i].size());
                        LAMINO_CUDA(cudaMemcpyAsync(dp[i].p, r->projs[i].data(), r->projs[i].size() * 4,
                                                    cudaMemcpyHostToDevice, s));
                        data.push_back(Dataset{dp[i].p, r->pdims[i][0], r->pdims[i][1], r->pdims[i][2],
                                               r->angles[i].data(), r->gammas[i]});
                    }
                    out.alloc(nv);
                    job.reset(new MbirJob(r->method, data, r->recon, r->prm, out.p, s, ss));
                    job->prepare();
                }
                {
                    AllocStreamScope scope(ss);  // solver buffers live on the solve stream
                    job->solve();
                    job->finish();  // synchronises ss
                }
                r->phases = last_mbir_phases();
                r->result.resize((size_t)nv);
                LAMINO_CUDA(cudaMemcpyAsync(r->result.data(), out.p, nv * 4, cudaMemcpyDeviceToHost, ss));
                LAMINO_CUDA(cudaStreamSynchronize(ss));
                job.reset();
            }
        } catch (const Error &e) {
            status = e.code;
            err = e.what();
        } catch (const std::exception &e) {
            status = ERR_STATE;
            err = e.what();
        }
        lk.lock();
        in_use_ -= r->footprint;
        --active_;
        r->status = status;
        r->err = err;
        r->t_done = now();
        r->done = true;
        if (status == OK) ++completed_;
        else ++failed_;
        lk.unlock();
        cv_.notify_all();
    }
    if (s) cudaStreamDestroy(s);
    if (ss) cudaStreamDestroy(ss);
}

bool Server::wait(int64_t id, double timeout_s, ServeRequest **out) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) throw Error(ERR_ARG, "unknown request id");
    ServeRequest *r = it->second.get();
    auto pred = [&] { return r->done; };
    if (timeout_s < 0) cv_.wait(lk, pred);
    else if (!cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return false;
    *out = r;
    return true;
}

void Server::release(int64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it != reqs_.end() && it->second->done) reqs_.erase(it);
}

ServerStats Server::stats() {
    std::lock_guard<std::mutex> lk(mu_);
    ServerStats st;
    st.submitted = submitted_;
    st.completed = completed_;
    st.failed = failed_;
    st.in_use = in_use_;
    st.peak_in_use = peak_;
    st.budget = budget_;
    st.active = active_;
    st.peak_active = peak_active_;
    st.queued = (int)queue_.size();
    st.slots = slots_;
    return st;
}

}  // namespace lamino
