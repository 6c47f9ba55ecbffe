// Device helpers: error checks, buffers, warp lane layouts.
#pragma once

#include <algorithm>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <utility>

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "common.h"

namespace fereg {

inline void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) throw Error(RC_OUT_OF_MEMORY, std::string("fereg: insufficient memory (") + what + ")");
    throw Error(RC_INTERNAL, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
#define CK(x) ::fereg::cuda_check((x), #x)

// Stream-ordered allocation. While an AllocScope is active on a thread, DBuf allocations made on
// that thread come from the device's memory pool in the order of the scope's stream
// (cudaMallocAsync / cudaFreeAsync on the stream the owner runs all its work on), so that
// releasing a buffer does not wait for the whole device, as cudaFree does; concurrent sessions
// on their own streams then never stall one another. Without a scope DBuf uses cudaMalloc /
// cudaFree.
inline cudaStream_t& alloc_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}
struct AllocScope {
    cudaStream_t prev;
    explicit AllocScope(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocScope() { alloc_stream() = prev; }
    AllocScope(const AllocScope&) = delete;
    AllocScope& operator=(const AllocScope&) = delete;
};

// CTAs of `kernel` resident on one SM at `threads` threads and `smem` dynamic shared memory, the
// occupancy query cached per (kernel, threads, shared memory, device) for the process.
template <class K>
inline int resident_ctas(K kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t, int>, int> memo;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    const auto key = std::make_tuple(reinterpret_cast<const void*>(kernel), threads, smem, dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    memo[key] = per_sm;
    return per_sm;
}

// Keeps memory released to the device's default pool mapped, up to 40% of the device memory (or
// more, when the caller set more), once per device and process: the sessions' stream-ordered
// allocations then reuse pool pages instead of mapping fresh ones at every call (the default
// threshold of 0 returns the pool's memory at each synchronization). A per-process attribute of
// the pool, not a device setting.
inline void keep_pool_mapped() {
    static std::mutex mu;
    static std::set<int> done;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (!done.insert(dev).second) return;
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    u64 cur = 0;
    CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur));
    u64 thr = std::max<u64>(cur, u64(0.4 * double(tot)));
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
}

// Owned device allocation.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;  // the stream of a pooled allocation
    bool pooled = false;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s), pooled(o.pooled) {
        o.p = nullptr;
        o.n = 0;
    }
    DBuf& operator=(DBuf&& o) noexcept {
        release();
        p = o.p;
        n = o.n;
        s = o.s;
        pooled = o.pooled;
        o.p = nullptr;
        o.n = 0;
        return *this;
    }
    ~DBuf() { release(); }
    void release() {
        if (p) {
            if (pooled) cudaFreeAsync(p, s);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        const cudaStream_t st = alloc_stream();
        if (st) {
            CK(cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), st));
            s = st;
            pooled = true;
        } else {
            CK(cudaMalloc(&p, count * sizeof(T)));
            pooled = false;
        }
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t st) {
        alloc(count);
        if (count) CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    void upload(const std::vector<T>& h, cudaStream_t st) { upload(h.data(), h.size(), st); }
};

// Raises a kernel's dynamic-shared-memory limit to the most a block can take (the per-block
// opt-in maximum less the kernel's static shared memory), once per kernel and device, and
// returns that limit. The limit is a process-wide attribute: it is always set to the same value,
// so concurrent sessions never lower it under one another, and later calls cost no driver call.
template <class K>
inline int smem_limit(K kernel) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> lim;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = lim.find(key);
    if (it != lim.end()) return it->second;
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    const int v = optin - int(fa.sharedSizeBytes);
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, v));
    lim.emplace(key, v);
    return v;
}

constexpr unsigned FULL = 0xffffffffu;

// Padded width (a power of two up to 32) of a chunk of Rc columns: lanes of a warp form
// 32 / width groups of `width` consecutive columns.
__host__ __device__ constexpr int rcp_of(int Rc) {
    return Rc <= 1 ? 1 : Rc <= 2 ? 2 : Rc <= 4 ? 4 : Rc <= 8 ? 8 : Rc <= 16 ? 16 : 32;
}

// Lane layout of a warp over (entry slot, column) pairs for a block of R columns: with R <= 32
// the warp holds G = 32/R slots of R consecutive columns (lane = slot*R + col), so consecutive
// lanes touch consecutive doubles of a row-major row block; with R > 32 the columns are walked
// in chunks of 32 with one slot.
struct LaneMap {
    int G, slot, col;
    bool on;
};

__device__ __forceinline__ int col_chunks(int R) { return R <= 32 ? 1 : (R + 31) / 32; }

__device__ __forceinline__ LaneMap lane_map(int R, int lane, int chunk) {
    if (R <= 32) {
        int G = 32 / R;
        return {G, lane / R, lane % R, lane < G * R};
    }
    int col = chunk * 32 + lane;
    return {1, 0, col, col < R};
}

// Sum of `v` over the slots holding the same column, in slot order (every lane gets the sum;
// inactive lanes must hold 0).
template <class T>
__device__ __forceinline__ T slot_sum(T v, const LaneMap& L, int R) {
    if (L.G == 1) return v;
    T s = T(0);
    const int col = R <= 32 ? (threadIdx.x & 31) % R : 0;
    for (int g = 0; g < L.G; g++) s += __shfl_sync(FULL, v, g * R + col);
    return s;
}

}  // namespace fereg
