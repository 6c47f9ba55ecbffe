// Sample preparation on the device (factor.rs, sample.rs): FE-id compression (factorize,
// combine, restrict) and the cyclic singleton / `fe` separation drops. Integer and byte work;
// every result is bit-exact against the reference's definitions (codes in ascending value order,
// drop counts per pass).
#pragma once

#include "device.cuh"

namespace fereg {

// factor.rs:26-31 f64_key: an order-preserving map of doubles (with -0 = +0) to u64.
__device__ __forceinline__ u64 f64_key_dev(double x) {
    if (x == 0.0) x = 0.0;
    const u64 bits = u64(__double_as_longlong(x));
    return (bits >> 63) ? ~bits : (bits | (1ull << 63));
}

constexpr int PREP_TB = 256;

// Keys and identity values; per-CTA min / max of the values; flags[0] = a NaN, flags[1] = a value
// that is not an integer below 2^53 in magnitude (no direct table).
__global__ void __launch_bounds__(PREP_TB) k_prep_keys(const double* __restrict__ x, size_t n, u64* __restrict__ keys,
                                                       u32* __restrict__ idx, double* __restrict__ pmin,
                                                       double* __restrict__ pmax, int* flags) {
    __shared__ double smin[PREP_TB], smax[PREP_TB];
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    double lo = inf, hi = -inf;
    for (size_t i = size_t(blockIdx.x) * PREP_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * PREP_TB) {
        const double v = x[i];
        if (v != v) atomicExch(flags, 1);
        else if (!(fabs(v) < 9007199254740992.0) || v != floor(v)) atomicExch(flags + 1, 1);
        keys[i] = f64_key_dev(v);
        idx[i] = u32(i);
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    __syncthreads();
    for (int h = PREP_TB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + h]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pmin[blockIdx.x] = smin[0];
        pmax[blockIdx.x] = smax[0];
    }
}

// Direct table: present[x - vmin] = 1 (idempotent stores).
__global__ void k_prep_mark(const double* __restrict__ x, size_t n, double vmin, u32* __restrict__ present) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        present[u64(x[i] - vmin)] = 1u;
}

// codes[i] = the rank of x[i] among the present values (exclusive scan of `present`).
__global__ void k_prep_table_codes(const double* __restrict__ x, size_t n, double vmin, const u32* __restrict__ rank,
                                   u32* __restrict__ codes) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        codes[i] = rank[u64(x[i] - vmin)];
}

// Mixed-radix keys of a combination of code columns (factor.rs:255 combine):
// key = (...(c_0 nl_1 + c_1) nl_2 + ...) in part order.
__global__ void k_prep_combine_keys(const u32* const* __restrict__ parts, const u32* __restrict__ nl, int np, size_t n,
                                    u64* __restrict__ keys, u32* __restrict__ idx) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        u64 k = 0;
        for (int p = 0; p < np; p++) k = k * u64(nl[p]) + parts[p][i];
        keys[i] = k;
        idx[i] = u32(i);
    }
}

// Direct table over integer keys: present[key - kmin] = 1; codes from its scan.
__global__ void k_prep_mark_keys(const u64* __restrict__ keys, size_t n, u64 kmin, u32* __restrict__ present) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        present[keys[i] - kmin] = 1u;
}
__global__ void k_prep_key_codes(const u64* __restrict__ keys, size_t n, u64 kmin, const u32* __restrict__ rank,
                                 u32* __restrict__ codes) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        codes[i] = rank[keys[i] - kmin];
}

// Per-CTA min / max of u64 keys.
__global__ void __launch_bounds__(PREP_TB) k_prep_key_range(const u64* __restrict__ keys, size_t n,
                                                            u64* __restrict__ pmin, u64* __restrict__ pmax) {
    __shared__ u64 smin[PREP_TB], smax[PREP_TB];
    u64 lo = ~0ull, hi = 0;
    for (size_t i = size_t(blockIdx.x) * PREP_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * PREP_TB) {
        lo = min(lo, keys[i]);
        hi = max(hi, keys[i]);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    __syncthreads();
    for (int h = PREP_TB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            smin[threadIdx.x] = min(smin[threadIdx.x], smin[threadIdx.x + h]);
            smax[threadIdx.x] = max(smax[threadIdx.x], smax[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pmin[blockIdx.x] = smin[0];
        pmax[blockIdx.x] = smax[0];
    }
}

// ---------------------------------------------------------------------------------------------
// Stable LSD radix sort of (u64 key, u32 value) pairs, 8-bit digits. A pass over digit `shift`:
// per-tile digit histograms (digit-major: hist[d * ntiles + t]), their exclusive scan, then a
// stable scatter: each tile walks its elements in chunks of RS_TB in order; within a chunk a warp
// ranks equal digits with __match_any_sync and the warps' counts are prefixed in warp order.
constexpr int RS_TB = 256, RS_ITEMS = 16, RS_TILE = RS_TB * RS_ITEMS, RS_W = RS_TB / 32;

__global__ void __launch_bounds__(RS_TB) k_rs_hist(const u64* __restrict__ keys, size_t n, int shift, u32 ntiles,
                                                   u32* __restrict__ hist) {
    __shared__ u32 h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = size_t(blockIdx.x) * RS_TILE;
    for (int t = 0; t < RS_ITEMS; t++) {
        const size_t i = base + size_t(t) * RS_TB + threadIdx.x;
        if (i < n) atomicAdd(&h[u32(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[size_t(threadIdx.x) * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_TB) k_rs_scatter(const u64* __restrict__ kin, const u32* __restrict__ vin,
                                                      size_t n, int shift, u32 ntiles, const u32* __restrict__ offs,
                                                      u64* __restrict__ kout, u32* __restrict__ vout) {
    __shared__ u32 run[256], wcnt[RS_W][257], wpre[RS_W][256], tot[256];
    const u32 lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    run[threadIdx.x] = offs[size_t(threadIdx.x) * ntiles + blockIdx.x];
    const size_t base = size_t(blockIdx.x) * RS_TILE;
    for (int t = 0; t < RS_ITEMS; t++) {
        for (u32 q = 0; q < RS_W; q++) wcnt[q][threadIdx.x] = 0;
        __syncthreads();
        const size_t i = base + size_t(t) * RS_TB + threadIdx.x;
        const bool valid = i < n;
        const u64 k = valid ? kin[i] : 0;
        const u32 d = valid ? (u32(k >> shift) & 255u) : 256u;
        const u32 peers = __match_any_sync(FULL, d);
        const u32 rank = __popc(peers & ((1u << lane) - 1u));
        if (rank == 0) wcnt[w][d] = __popc(peers);
        __syncthreads();
        {
            u32 s = 0;
            for (u32 q = 0; q < RS_W; q++) {
                wpre[q][threadIdx.x] = s;
                s += wcnt[q][threadIdx.x];
            }
            tot[threadIdx.x] = s;
        }
        __syncthreads();
        if (valid) {
            const u32 pos = run[d] + wpre[w][d] + rank;
            kout[pos] = k;
            vout[pos] = vin[i];
        }
        __syncthreads();
        run[threadIdx.x] += tot[threadIdx.x];
    }
}

// flags[i] = 1 where the sorted key differs from its predecessor (a new level).
__global__ void k_prep_new_level(const u64* __restrict__ keys, size_t n, u32* __restrict__ flags) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// codes[idx[i]] = the level of sorted position i (inclusive count of new levels - 1).
__global__ void k_prep_sorted_codes(const u32* __restrict__ idx, const u32* __restrict__ flags,
                                    const u32* __restrict__ excl, size_t n, u32* __restrict__ codes) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        codes[idx[i]] = excl[i] + flags[i] - 1u;
}

// ---------------------------------------------------------------------------------------------
// One pass of drop_singletons over one term (sample.rs:154-238): per-level weighted counts of the
// alive rows and of those with a nonzero outcome (the `fe` rule), then the verdict per row:
// singleton (count 1), else separated (Poisson: no nonzero outcome; logit: none or all).
// Counts are sums of integer weights (1 or frequency weights), exact in any order.
__global__ void k_sing_count(const u32* __restrict__ codes, size_t n, const uint8_t* __restrict__ alive,
                             const double* __restrict__ fw, const double* __restrict__ y, double* __restrict__ cnt,
                             double* __restrict__ pos) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        if (!alive[i]) continue;
        const double w = fw ? fw[i] : 1.0;
        atomicAdd(&cnt[codes[i]], w);
        if (y && y[i] != 0.0) atomicAdd(&pos[codes[i]], w);
    }
}

// family: 0 none, 1 Poisson, 2 logit. out[0] += singletons, out[1] += separated.
__global__ void k_sing_drop(const u32* __restrict__ codes, size_t n, uint8_t* __restrict__ alive,
                            const double* __restrict__ cnt, const double* __restrict__ pos, int singletons, int family,
                            unsigned long long* out) {
    unsigned long long s = 0, f = 0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        if (!alive[i]) continue;
        const double k = cnt[codes[i]];
        if (singletons && k == 1.0) {
            alive[i] = 0;
            s++;
        } else if (family) {
            const double p = pos[codes[i]];
            if (p == 0.0 || (family == 2 && p == k)) {
                alive[i] = 0;
                f++;
            }
        }
    }
    if (s) atomicAdd(out, s);
    if (f) atomicAdd(out + 1, f);
}

// present[codes[i]] = 1 over the kept rows.
__global__ void k_prep_present(const u32* __restrict__ codes, size_t n, const uint8_t* __restrict__ alive,
                               u32* __restrict__ present) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        if (alive[i]) present[codes[i]] = 1u;
}

// Compaction (factor.rs:281 restrict): out[rank of kept row i] = the new code of its level.
__global__ void k_prep_restrict(const u32* __restrict__ codes, size_t n, const uint8_t* __restrict__ alive,
                                const u32* __restrict__ kept_rank, const u32* __restrict__ level_rank,
                                u32* __restrict__ out) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        if (alive[i]) out[kept_rank[i]] = level_rank[codes[i]];
}

__global__ void k_prep_alive_u32(const uint8_t* __restrict__ alive, size_t n, u32* __restrict__ out) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = alive[i] ? 1u : 0u;
}

}  // namespace fereg
