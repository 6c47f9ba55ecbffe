// Serving engine: a request loop over independent FE regressions (OLS, IV / 2SLS, logit,
// Poisson) on one GPU. The reference estimates one model per call from its orchestration thread
// (api.rs:198-210: one handle, one thread); serving multiplexes such calls inside the library.
//
// * Admission by HBM budget: every request carries an estimate of the device memory its session
//   holds (request_bytes). Requests are admitted in arrival order (FIFO, no overtaking) while the
//   admitted requests' estimates fit the budget; a request larger than the whole budget is
//   rejected at submission (909, the reference's OutOfMemory code).
// * Continuous batching: `workers` threads each run one admitted request at a time on its own
//   session and CUDA stream (GpuSession owns a non-blocking stream; allocations are
//   stream-ordered), so independent solves overlap on the GPU; a finished request frees its
//   budget and its worker at once and the next request is admitted.
// * Stream priorities by size: a request's stream takes a priority level by its rows x columns
//   (the highest below 1e5, one level lower per decade above), so that small requests, whose
//   solves are chains of short kernels and host round trips, are not queued behind the large
//   requests' passes.
// * Results do not depend on the mix: every kernel reduces in a fixed order and each request's
//   work stays on its own stream, so a request gives the same bits alone and in the stream.
// * dry_run: the scheduler without the GPU (each request sleeps dry_run_us), for host-side tests.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace fereg {

struct ServeRequest {
    int model = 0;  // 0 OLS, 1 IV, 2 logit, 3 Poisson
    std::vector<const u32*> codes, cl_codes;
    std::vector<u32> g, cl_g;
    const double* w = nullptr;  // kept-order weights (OLS / IV) or null
    int weight_kind = 0;
    size_t n = 0;
    std::vector<const double*> cols;  // [y, exog (nx), endog (ne), inst (ni)], kept order
    size_t nx = 0, ne = 0, ni = 0;
    int vce = 0;
    double tol = 1e-8;
    size_t maxiter = 16000;
    int precision = 0;
    double* b = nullptr;  // caller buffers: k_all and k_all^2 values
    double* V = nullptr;
    u64 dry_run_us = 0;
};

struct ServeResult {
    int rc = 0;
    std::string msg;
    double submit_s = 0, admit_s = 0, done_s = 0;  // seconds since the server started
    double prep_s = 0;  // session preparation (cell structure, uploads) and the row gather
    u64 bytes = 0;
    double N = 0;
    u64 iterations = 0;
    u64 launches = 0;  // kernels the request's session launched
    bool converged = true;
};

// Estimated device bytes of a request's session (see server.cu).
u64 request_bytes(const ServeRequest& r);

class Server {
   public:
    Server(int workers, u64 budget, bool dry_run);
    ~Server();
    u64 submit(const ServeRequest& r);  // ticket; throws Error(909) when larger than the budget
    ServeResult wait(u64 ticket);       // blocks until the request is done
    // submitted, completed, rejected, peak admitted bytes, peak running, budget, running, kernel
    // launches of the completed requests
    void stats(u64* out) const;

   private:
    struct Entry {
        ServeRequest req;
        ServeResult res;
        bool done = false;
    };
    void worker();
    void run(Entry& e);
    double now() const;

    int device_ = 0;
    bool dry_ = false;
    u64 budget_ = 0, in_use_ = 0, peak_ = 0;
    u64 next_ = 1, submitted_ = 0, completed_ = 0, rejected_ = 0, launches_ = 0;
    int running_ = 0, peak_running_ = 0;
    bool stop_ = false;
    std::chrono::steady_clock::time_point t0_;
    mutable std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<u64> pending_;
    std::unordered_map<u64, Entry> entries_;
    std::vector<std::thread> threads_;
};

}  // namespace fereg
