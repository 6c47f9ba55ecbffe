// Exclusive scan of u32 arrays in three launches: per-tile sums, a one-block scan of the tile
// sums (with the total), and the per-tile scan. Internal linkage: every translation unit that
// launches it holds its own copy.
#pragma once

#include "device.cuh"

namespace fereg {

constexpr int SCAN_TB = 256, SCAN_ITEMS = 8, SCAN_TILE = SCAN_TB * SCAN_ITEMS;

static __device__ __forceinline__ u32 block_excl_scan(u32 v, u32* sh, u32* total) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < SCAN_TB; off <<= 1) {
        const u32 t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0u;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    const u32 incl = sh[threadIdx.x];
    if (total) *total = sh[SCAN_TB - 1];
    __syncthreads();
    return incl - v;
}

static __global__ void __launch_bounds__(SCAN_TB) k_scan_sums(const u32* __restrict__ in, size_t n, u32* __restrict__ bsum) {
    __shared__ u32 sh[SCAN_TB];
    const size_t base = size_t(blockIdx.x) * SCAN_TILE + size_t(threadIdx.x) * SCAN_ITEMS;
    u32 s = 0;
    for (int t = 0; t < SCAN_ITEMS; t++)
        if (base + t < n) s += in[base + t];
    u32 tot;
    block_excl_scan(s, sh, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

static __global__ void __launch_bounds__(SCAN_TB) k_scan_top(u32* bsum, u32 nb, u32* total) {
    __shared__ u32 sh[SCAN_TB];
    u32 carry = 0;
    for (u32 b0 = 0; b0 < nb; b0 += SCAN_TB) {
        const u32 b = b0 + threadIdx.x;
        const u32 v = b < nb ? bsum[b] : 0u;
        u32 tot;
        const u32 ex = block_excl_scan(v, sh, &tot);
        if (b < nb) bsum[b] = carry + ex;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

static __global__ void __launch_bounds__(SCAN_TB) k_scan_apply(const u32* __restrict__ in, size_t n,
                                                        const u32* __restrict__ bsum, u32* __restrict__ out) {
    __shared__ u32 sh[SCAN_TB];
    const size_t base = size_t(blockIdx.x) * SCAN_TILE + size_t(threadIdx.x) * SCAN_ITEMS;
    u32 v[SCAN_ITEMS], s = 0;
    for (int t = 0; t < SCAN_ITEMS; t++) {
        v[t] = base + t < n ? in[base + t] : 0u;
        s += v[t];
    }
    u32 run = block_excl_scan(s, sh, nullptr) + bsum[blockIdx.x];
    for (int t = 0; t < SCAN_ITEMS; t++) {
        if (base + t < n) out[base + t] = run;
        run += v[t];
    }
}

}  // namespace fereg
