// Serving engine (see server.h).
#include "server.h"

#include <cuda_runtime.h>

#include <algorithm>

#include "absorber.h"
#include "session.h"

namespace fereg {

// Device bytes a request's session holds, from its sizes (an upper estimate): the kept-order
// columns and the row-order block (a third block for GLM's raw copy), per-row state (term and
// cluster codes, row order, cluster permutations, structure tables, residuals, weights, GLM
// working vectors), the PCG vectors of the reduced system (m <= sum of levels, ~10 m x R
// doubles) and a fixed 32 MiB for tiles, partials and the small block.
u64 request_bytes(const ServeRequest& r) {
    const u64 n = r.n, R = 1 + r.nx + r.ne + r.ni;
    const u64 blocks = r.model >= 2 ? 3 : 2;
    const u64 nt = r.codes.size(), nc = r.cl_codes.size();
    const u64 per_row = R * 8 * blocks + 4 * (3 * nt + 3 * nc + 6) + 8 * (r.model >= 2 ? 12 : 6);
    u64 levels = 0;
    for (u32 x : r.g) levels += x;
    // the dense small super-block (the smallest terms besides FE1 up to SMALL_LIMIT levels, when
    // at most 1024 coordinates): factor, its work arrays and inverse (4 ms^2 doubles) and the
    // partial rows of its assembly (at most 4096 + ms rows of ms doubles)
    std::vector<u32> others(r.g.begin(), r.g.end());
    const int f1 = fe1_index(r.g);
    if (f1 >= 0) others.erase(others.begin() + f1);
    std::sort(others.begin(), others.end());
    u64 ms = 0;
    for (u32 x : others) {
        if (ms + x > SMALL_LIMIT) break;
        ms += x;
    }
    const u64 dense = ms > 0 && ms <= 1024 ? (4 * ms * ms + (4096 + ms) * ms) * 8 : 0;
    return n * per_row + levels * R * 8 * 10 + dense + (32ull << 20);
}

Server::Server(int workers, u64 budget, bool dry_run) : dry_(dry_run), t0_(std::chrono::steady_clock::now()) {
    if (workers <= 0) workers = 4;
    if (!dry_) {
        CK(cudaGetDevice(&device_));
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        if (budget == 0) budget = u64(0.8 * double(fr));
        // keep released pool memory mapped up to the budget: requests reuse it instead of
        // mapping fresh pages per allocation
        cudaMemPool_t pool;
        CK(cudaDeviceGetDefaultMemPool(&pool, device_));
        u64 thr = budget;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    }
    if (budget == 0) throw Error(RC_INVALID_INPUT, "fereg_server_create: a dry-run server needs a budget");
    budget_ = budget;
    for (int i = 0; i < workers; i++) threads_.emplace_back([this] { worker(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : threads_) t.join();
}

double Server::now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

u64 Server::submit(const ServeRequest& r) {
    if (r.model < 0 || r.model > 3) throw Error(RC_INVALID_INPUT, "fereg_server_submit: unknown model");
    if (r.cols.size() != 1 + r.nx + r.ne + r.ni) throw Error(RC_INVALID_INPUT, "fereg_server_submit: column count");
    if (r.model == 1 && r.ne == 0) throw Error(RC_INVALID_INPUT, "fereg_server_submit: IV without endogenous regressors");
    if (r.model != 1 && (r.ne || r.ni)) throw Error(RC_INVALID_INPUT, "fereg_server_submit: instruments outside IV");
    if (r.model >= 2 && r.w) throw Error(RC_INVALID_INPUT, "fereg_server_submit: weighted GLM requests");
    const u64 bytes = request_bytes(r);
    std::lock_guard<std::mutex> lk(mu_);
    if (bytes > budget_) {
        rejected_++;
        throw Error(RC_OUT_OF_MEMORY, "fereg_server_submit: the request needs more device memory than the budget");
    }
    const u64 t = next_++;
    Entry& e = entries_[t];
    e.req = r;
    e.res.bytes = bytes;
    e.res.submit_s = now();
    pending_.push_back(t);
    submitted_++;
    cv_work_.notify_all();
    return t;
}

ServeResult Server::wait(u64 ticket) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = entries_.find(ticket);
    if (it == entries_.end()) throw Error(RC_INVALID_INPUT, "fereg_server_wait: unknown ticket");
    Entry* e = &it->second;  // element addresses survive rehashing, iterators do not
    cv_done_.wait(lk, [&] { return e->done; });
    ServeResult res = e->res;
    entries_.erase(ticket);
    return res;
}

void Server::stats(u64* out) const {
    std::lock_guard<std::mutex> lk(mu_);
    out[0] = submitted_;
    out[1] = completed_;
    out[2] = rejected_;
    out[3] = peak_;
    out[4] = u64(peak_running_);
    out[5] = budget_;
    out[6] = u64(running_);
    out[7] = launches_;
}

void Server::worker() {
    if (!dry_) cudaSetDevice(device_);
    for (;;) {
        u64 t = 0;
        Entry* e = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu_);
            // admit the head of the queue when its estimate fits next to the running requests
            cv_work_.wait(lk, [&] {
                return stop_ || (!pending_.empty() && in_use_ + entries_[pending_.front()].res.bytes <= budget_);
            });
            if (stop_) return;
            t = pending_.front();
            pending_.pop_front();
            e = &entries_[t];
            in_use_ += e->res.bytes;
            peak_ = std::max(peak_, in_use_);
            running_++;
            peak_running_ = std::max(peak_running_, running_);
            e->res.admit_s = now();
        }
        run(*e);
        {
            std::lock_guard<std::mutex> lk(mu_);
            in_use_ -= e->res.bytes;
            running_--;
            completed_++;
            launches_ += e->res.launches;
            e->res.done_s = now();
            e->done = true;
        }
        cv_done_.notify_all();
        cv_work_.notify_all();
    }
}

// Stream priority level of a request: 0 (highest) below 1e5 row-columns, one level lower per
// decade above. A small request's solve is a long chain of short kernels and host round trips;
// at equal priority each of its kernels queues behind the large requests' passes.
static int priority_level(const ServeRequest& q) {
    const double work = double(q.n) * double(std::max<size_t>(1, q.cols.size()));
    int level = 0;
    for (double b = 1e5; work >= b && level < 3; b *= 10.0) level++;
    return level;
}

void Server::run(Entry& e) {
    const ServeRequest& q = e.req;
    ServeResult& res = e.res;
    if (dry_) {
        std::this_thread::sleep_for(std::chrono::microseconds(q.dry_run_us));
        res.N = double(q.n);
        return;
    }
    try {
        Ctx ctx;
        ctx.priority_level = priority_level(q);
        ctx.autotune = false;
        const double t0 = now();
        GpuSession s(q.codes, q.g, q.cl_codes, q.cl_g, q.w, q.w ? q.weight_kind : 0, q.n, 0, ctx);
        double* rows = s.gather_columns(q.cols.data(), q.cols.size());
        res.prep_s = now() - t0;
        const Precision prec = q.precision == 1 ? Precision::F32_REFINED : Precision::F64;
        if (q.model == 0) {
            OlsSpec sp;
            sp.vce = q.vce;
            sp.tol = q.tol;
            sp.maxiter = q.maxiter;
            sp.prec = prec;
            OlsOut o;
            o.b = q.b;
            o.V = q.V;
            s.ols(rows, true, q.nx, sp, o);
            res.N = o.N;
            res.iterations = u64(o.ic);
        } else if (q.model == 1) {
            GpuSession::IvSpec sp;
            sp.vce = q.vce;
            sp.tol = q.tol;
            sp.maxiter = q.maxiter;
            sp.prec = prec;
            GpuSession::IvOut o;
            o.b = q.b;
            o.V = q.V;
            s.iv(rows, true, q.nx, q.ne, q.ni, sp, o);
            res.N = o.N;
            res.iterations = u64(o.ic);
        } else {
            GpuSession::GlmSpec sp;
            sp.family = q.model == 2 ? 1 : 0;
            sp.vce = q.vce;
            sp.tol = q.tol;
            sp.inner_maxiter = q.maxiter;
            sp.prec = prec;
            GpuSession::GlmOut o;
            o.b = q.b;
            o.V = q.V;
            s.glm(rows, true, q.nx, sp, o);
            res.N = o.N;
            res.iterations = o.pcg_iterations;
            res.converged = o.converged;
        }
        res.launches = s.launches();
    } catch (const Error& ex) {
        res.rc = ex.rc;
        res.msg = ex.what();
    } catch (const std::exception& ex) {
        res.rc = RC_INTERNAL;
        res.msg = ex.what();
    }
}

}  // namespace fereg
