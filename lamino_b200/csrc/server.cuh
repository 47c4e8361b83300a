// Continuous-batching reconstruction server.
//
// Requests (MBIR1/2/3 problems of any size) arrive at any time.  A request is
// admitted, in arrival order, as soon as a worker slot is free and its
// estimated peak device footprint fits in the HBM budget next to the requests
// already running; each slot runs on its own CUDA stream, so admitted
// reconstructions overlap on the GPU and their iterates stay in device memory
// until they finish.  Finished requests release their memory and slot at once,
// which admits the next ones.
#pragma once

#include <array>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mbir.cuh"

namespace lamino {

struct ServeRequest {
    int64_t id = 0;
    int method = 2;
    Dims3 recon{};
    ReconParams prm;
    std::vector<std::vector<float>> projs;  // host copies
    std::vector<std::array<int64_t, 3>> pdims;
    std::vector<std::vector<float>> angles;
    std::vector<float> gammas;
    int64_t footprint = 0;
    std::vector<float> result;  // 3 * recon voxels, host
    double t_submit = 0, t_start = 0, t_done = 0;
    MbirPhases phases;
    int status = 0;
    std::string err;
    bool done = false;
};

struct ServerStats {
    int64_t submitted = 0, completed = 0, failed = 0;
    int64_t in_use = 0, peak_in_use = 0, budget = 0;
    int active = 0, peak_active = 0, queued = 0, slots = 0;
};

class Server {
  public:
    // budget: device bytes the admitted requests may hold together; slots: requests
    // running at once; dry_run: workers skip the GPU and hold each request for
    // dry_run_ms milliseconds (tests of the admission logic without a device).
    Server(int64_t budget, int slots, bool dry_run = false, double dry_run_ms = 0.0);
    ~Server();
    Server(const Server &) = delete;
    Server &operator=(const Server &) = delete;

    // r->t_submit, when already set, is kept (the caller's arrival time)
    int64_t submit(std::unique_ptr<ServeRequest> r);
    // Marks an API call in progress on this server: the destructor waits for it to
    // end (a thread blocked in wait() for a request that the shutdown drops wakes
    // with that request failed), so destroying the server never frees state that a
    // concurrent call still reads.  Throws ERR_STATE once shutdown has begun.
    struct Use {
        Server &s;
        explicit Use(Server &sv);
        ~Use();
        Use(const Use &) = delete;
        Use &operator=(const Use &) = delete;
    };
    // blocks until the request finished (or timeout_s elapsed: returns false)
    bool wait(int64_t id, double timeout_s, ServeRequest **out);
    void release(int64_t id);  // forget a finished request
    ServerStats stats();

    static double now();  // steady-clock seconds

  private:
    void worker(int wid);

    int64_t budget_;
    int slots_;
    bool dry_;
    cudaMemPool_t pool_ = nullptr;  // the device's default pool and its release threshold before the server
    uint64_t old_threshold_ = 0;
    double dry_ms_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<int64_t> queue_;
    std::map<int64_t, std::unique_ptr<ServeRequest>> reqs_;
    int64_t next_id_ = 1, in_use_ = 0, peak_ = 0, submitted_ = 0, completed_ = 0, failed_ = 0;
    int active_ = 0, peak_active_ = 0;
    bool stop_ = false;
    int users_ = 0;
    std::vector<std::thread> workers_;
};

}  // namespace lamino
