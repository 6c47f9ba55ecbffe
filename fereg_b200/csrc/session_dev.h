// Device state of a GpuSession (shared by the OLS call and the wild bootstrap).
#pragma once

#include <vector>

#include "device.cuh"
#include "session.h"

namespace fereg {

// A CUDA stream owned by its holder.
struct OwnedStream {
    cudaStream_t s = nullptr;
    OwnedStream() = default;
    OwnedStream(const OwnedStream&) = delete;
    OwnedStream& operator=(const OwnedStream&) = delete;
    ~OwnedStream() {
        if (s) cudaStreamDestroy(s);
    }
};

// The degrees-of-freedom pass (nested checks and the union-finds of the FE pairs) runs on its own
// stream (one priority step below the session's) from a host thread of its own; these are its
// buffers. gv (the mobility groups of the first pair, row labels) is read on the session's
// stream once the pass has been joined.
struct DofScratch {
    OwnedStream st;              // declared first: destroyed after the buffers allocated on it
    cudaEvent_t ready = nullptr; // recorded on the session's stream before the pass starts
    cudaEvent_t ta = nullptr, tb = nullptr;  // phase timing of the pass (when profiling)
    DBuf<u32> uf, flags, scan, bsum, total, gv, map;
    DBuf<int> err;
    u64 launches = 0;
    ~DofScratch() {
        if (ready) cudaEventDestroy(ready);
    }
};

// The column statistics of an OLS call run on a side stream (one priority step below the
// session's) beside the FE solve; their sums, first row and error flag come back into pinned host
// memory (room for CS_MAXR columns, the most an OLS block has).
constexpr int CS_MAXR = 64;
struct ColStatsSide {
    OwnedStream st;
    cudaEvent_t ready = nullptr, done = nullptr;
    double* sums = nullptr;  // 6 x CS_MAXR
    double* c0 = nullptr;    // CS_MAXR
    int* late = nullptr;
    ~ColStatsSide() {
        if (ready) cudaEventDestroy(ready);
        if (done) cudaEventDestroy(done);
        if (sums) cudaFreeHost(sums);
        if (c0) cudaFreeHost(c0);
        if (late) cudaFreeHost(late);
    }
};

// Device state of a session.
struct SessionDev {
    DofScratch dof;
    ColStatsSide cside;
    std::vector<DBuf<u32>> tcodes, ccodes;  // kept order
    struct Subset {
        DBuf<int> perm;  // rows (row order) grouped by cluster, stable
        DBuf<u32> coff;  // G + 1
        u32 G = 0;
        double sign = 1.0;
        std::vector<u32> kc;  // host: the combined cluster code of every kept observation
    };
    std::vector<Subset> subsets;
    DBuf<double> w_raw, wv;  // row order
    DBuf<double> rows, part, sums, e, om, S, shift, beta;
    DBuf<int> col, err;
    DBuf<u32> map;
    DBuf<double> pstat;
    DBuf<double> cgram, jk;  // CRV3: per-cluster Grams, a leave-out block
    DBuf<double> h;          // HC2 / HC3: the FE leverage per row
    DBuf<double> colbuf;  // kept-order columns of a gather
    DBuf<u32> pi;         // row order -> kept position
    cudaStream_t st = nullptr;
    u64 launches = 0;
    // phase timing (CUDA events on the session's stream)
    bool prof = false;
    double ms[GpuSession::S_NSLOTS] = {};
    u64 cnt[GpuSession::S_NSLOTS] = {};
    std::vector<cudaEvent_t> pool;
    struct Open {
        int slot;
        cudaEvent_t a, b;
    };
    std::vector<Open> open;
    // The side stream of the column statistics, created at first use.
    ColStatsSide& colstats_side() {
        ColStatsSide& c = cside;
        if (!c.st.s) {
            int least = 0, greatest = 0, own = 0;
            CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            CK(cudaStreamGetPriority(st, &own));
            CK(cudaStreamCreateWithPriority(&c.st.s, cudaStreamNonBlocking, std::min(least, own + 1)));
            CK(cudaEventCreateWithFlags(&c.ready, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
            CK(cudaMallocHost(&c.sums, 6 * CS_MAXR * sizeof(double)));
            CK(cudaMallocHost(&c.c0, CS_MAXR * sizeof(double)));
            CK(cudaMallocHost(&c.late, sizeof(int)));
        }
        return c;
    }
    cudaEvent_t event() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        return e;
    }
    int begin(int slot) {
        if (!prof) return -1;
        open.push_back(Open{slot, event(), nullptr});
        CK(cudaEventRecord(open.back().a, st));
        return int(open.size()) - 1;
    }
    void end(int h) {
        if (h < 0) return;
        open[size_t(h)].b = event();
        CK(cudaEventRecord(open[size_t(h)].b, st));
    }
    void collect() {
        for (auto& o : open) {
            if (o.b) {
                CK(cudaEventSynchronize(o.b));
                float t = 0;
                CK(cudaEventElapsedTime(&t, o.a, o.b));
                ms[o.slot] += t;
                cnt[o.slot]++;
                pool.push_back(o.b);
            }
            pool.push_back(o.a);
        }
        open.clear();
    }
    ~SessionDev() {
        for (auto& o : open) {
            cudaEventDestroy(o.a);
            if (o.b) cudaEventDestroy(o.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

}  // namespace fereg
