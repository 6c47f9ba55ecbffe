// Sample preparation on the device: factorize / combine / restrict (factor.rs:38,255,281) and
// drop_singletons with the GLM `fe` rule (sample.rs:44-72,154-238). Host arrays in and out; the
// work runs on the device on a stream of its own (kernels in prep.cuh).
#include "prep.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "prep.cuh"
#include "scan.cuh"

namespace fereg {

namespace {

int grid_of(size_t n, int tb) { return int(std::max<size_t>(1, std::min<size_t>((n + tb - 1) / tb, 148 * 16))); }

struct Stream {
    cudaStream_t st = nullptr;
    Stream() { CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)); }
    ~Stream() {
        if (st) cudaStreamDestroy(st);
    }
};

// Exclusive scan of n u32 values into out; returns the total.
u32 excl_scan(const u32* in, size_t n, u32* out, cudaStream_t st) {
    DBuf<u32> bsum, total;
    const u32 nblk = u32((n + SCAN_TILE - 1) / SCAN_TILE);
    bsum.alloc(size_t(nblk) + 1);
    total.alloc(1);
    k_scan_sums<<<std::max<u32>(1, nblk), SCAN_TB, 0, st>>>(in, n, bsum.p);
    k_scan_top<<<1, SCAN_TB, 0, st>>>(bsum.p, nblk, total.p);
    k_scan_apply<<<std::max<u32>(1, nblk), SCAN_TB, 0, st>>>(in, n, bsum.p, out);
    u32 t = 0;
    CK(cudaMemcpyAsync(&t, total.p, sizeof(u32), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return t;
}

// min / max of device u64 keys.
void key_range(const u64* keys, size_t n, u64& lo, u64& hi, cudaStream_t st) {
    const int G = grid_of(n, PREP_TB);
    DBuf<u64> pmin, pmax;
    pmin.alloc(G);
    pmax.alloc(G);
    k_prep_key_range<<<G, PREP_TB, 0, st>>>(keys, n, pmin.p, pmax.p);
    std::vector<u64> a(G), b(G);
    CK(cudaMemcpyAsync(a.data(), pmin.p, G * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(b.data(), pmax.p, G * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    lo = *std::min_element(a.begin(), a.end());
    hi = *std::max_element(b.begin(), b.end());
}

// The direct table is used when the key range is at most max(2n, 2^20) (factor.rs:38).
bool direct_ok(u64 range, size_t n) { return range <= std::max<u64>(2 * u64(n), u64(1) << 20); }

// Codes of u64 keys by a direct table over [lo, hi].
u32 codes_by_table(const u64* keys, size_t n, u64 lo, u64 hi, u32* codes, cudaStream_t st) {
    const size_t range = size_t(hi - lo) + 1;
    DBuf<u32> present, rank;
    present.alloc(range);
    rank.alloc(range);
    CK(cudaMemsetAsync(present.p, 0, range * sizeof(u32), st));
    k_prep_mark_keys<<<grid_of(n, 256), 256, 0, st>>>(keys, n, lo, present.p);
    const u32 nlev = excl_scan(present.p, range, rank.p, st);
    k_prep_key_codes<<<grid_of(n, 256), 256, 0, st>>>(keys, n, lo, rank.p, codes);
    CK(cudaGetLastError());
    return nlev;
}

// Codes of u64 keys by a stable LSD radix sort of (key, row) over the digits that differ.
u32 codes_by_sort(u64* keys, u32* idx, size_t n, u64 lo, u64 hi, u32* codes, cudaStream_t st) {
    int top = 0;  // bits above the highest differing bit are the same in every key
    for (u64 d = lo ^ hi; d; d >>= 1) top++;
    DBuf<u64> k2;
    DBuf<u32> v2, hist, offs, flags, excl;
    k2.alloc(n);
    v2.alloc(n);
    const u32 ntiles = u32((n + RS_TILE - 1) / RS_TILE);
    hist.alloc(size_t(ntiles) * 256);
    offs.alloc(size_t(ntiles) * 256);
    u64* ka = keys;
    u64* kb = k2.p;
    u32* va = idx;
    u32* vb = v2.p;
    for (int shift = 0; shift < top; shift += 8) {
        k_rs_hist<<<ntiles, RS_TB, 0, st>>>(ka, n, shift, ntiles, hist.p);
        excl_scan(hist.p, size_t(ntiles) * 256, offs.p, st);
        k_rs_scatter<<<ntiles, RS_TB, 0, st>>>(ka, va, n, shift, ntiles, offs.p, kb, vb);
        CK(cudaGetLastError());
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    flags.alloc(n);
    excl.alloc(n);
    k_prep_new_level<<<grid_of(n, 256), 256, 0, st>>>(ka, n, flags.p);
    const u32 nlev = excl_scan(flags.p, n, excl.p, st);
    k_prep_sorted_codes<<<grid_of(n, 256), 256, 0, st>>>(va, flags.p, excl.p, n, codes);
    CK(cudaGetLastError());
    return nlev;
}

u32 codes_of_keys(u64* keys, u32* idx, size_t n, u32* codes, cudaStream_t st) {
    u64 lo = 0, hi = 0;
    key_range(keys, n, lo, hi, st);
    if (direct_ok(hi - lo, n)) return codes_by_table(keys, n, lo, hi, codes, st);
    return codes_by_sort(keys, idx, n, lo, hi, codes, st);
}

// Every code of a column must be below its level count (the kernels index by it).
void check_codes(const u32* c, size_t n, u32 g, const char* what) {
    for (size_t i = 0; i < n; i++)
        if (c[i] >= g) throw Error(RC_INVALID_INPUT, std::string(what) + ": a code is not below its level count");
}

}  // namespace

u32 device_excl_scan(const u32* in, size_t n, u32* out, cudaStream_t st) { return excl_scan(in, n, out, st); }

void device_sort_pairs(u64*& keys, u32*& vals, u64* keys_alt, u32* vals_alt, size_t n, int bits, cudaStream_t st) {
    if (n == 0 || bits <= 0) return;
    DBuf<u32> hist, offs;
    const u32 ntiles = u32((n + RS_TILE - 1) / RS_TILE);
    hist.alloc(size_t(ntiles) * 256);
    offs.alloc(size_t(ntiles) * 256);
    u64* ka = keys;
    u64* kb = keys_alt;
    u32* va = vals;
    u32* vb = vals_alt;
    for (int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<ntiles, RS_TB, 0, st>>>(ka, n, shift, ntiles, hist.p);
        excl_scan(hist.p, size_t(ntiles) * 256, offs.p, st);
        k_rs_scatter<<<ntiles, RS_TB, 0, st>>>(ka, va, n, shift, ntiles, offs.p, kb, vb);
        CK(cudaGetLastError());
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    keys = ka;
    vals = va;
}

u32 prep_factorize(const double* x, size_t n, u32* codes_out) {
    if (n == 0) return 0;
    Stream S;
    cudaStream_t st = S.st;
    AllocScope alloc_scope(st);
    DBuf<double> dx, pmin, pmax;
    DBuf<u64> keys;
    DBuf<u32> idx, codes;
    DBuf<int> flags;
    dx.upload(x, n, st);
    keys.alloc(n);
    idx.alloc(n);
    codes.alloc(n);
    const int G = grid_of(n, PREP_TB);
    pmin.alloc(G);
    pmax.alloc(G);
    flags.alloc(2);
    CK(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), st));
    k_prep_keys<<<G, PREP_TB, 0, st>>>(dx.p, n, keys.p, idx.p, pmin.p, pmax.p, flags.p);
    int fl[2];
    std::vector<double> a(G), b(G);
    CK(cudaMemcpyAsync(fl, flags.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(a.data(), pmin.p, G * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(b.data(), pmax.p, G * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (fl[0]) throw Error(RC_INVALID_INPUT, "missing values in factor");
    const double vmin = *std::min_element(a.begin(), a.end()), vmax = *std::max_element(b.begin(), b.end());
    const double span = vmax - vmin;
    u32 nlev;
    if (!fl[1] && span <= double(std::max<u64>(2 * u64(n), u64(1) << 20))) {  // integers in a small range: table
        const size_t range = size_t(vmax - vmin) + 1;
        DBuf<u32> present, rank;
        present.alloc(range);
        rank.alloc(range);
        CK(cudaMemsetAsync(present.p, 0, range * sizeof(u32), st));
        k_prep_mark<<<grid_of(n, 256), 256, 0, st>>>(dx.p, n, vmin, present.p);
        nlev = excl_scan(present.p, range, rank.p, st);
        k_prep_table_codes<<<grid_of(n, 256), 256, 0, st>>>(dx.p, n, vmin, rank.p, codes.p);
    } else {
        u64 lo = 0, hi = 0;
        key_range(keys.p, n, lo, hi, st);
        nlev = codes_by_sort(keys.p, idx.p, n, lo, hi, codes.p, st);
    }
    CK(cudaMemcpyAsync(codes_out, codes.p, n * sizeof(u32), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return nlev;
}

u32 prep_combine(const std::vector<const u32*>& parts, const std::vector<u32>& nl, size_t n, u32* codes_out) {
    if (n == 0) return 0;
    if (parts.size() == 1) {  // factor.rs:255: one part is its own codes
        std::copy(parts[0], parts[0] + n, codes_out);
        return nl[0];
    }
    Stream S;
    cudaStream_t st = S.st;
    AllocScope alloc_scope(st);
    std::vector<DBuf<u32>> dp(parts.size());
    std::vector<const u32*> ptrs;
    for (size_t p = 0; p < parts.size(); p++) check_codes(parts[p], n, nl[p], "fereg_combine");
    for (size_t p = 0; p < parts.size(); p++) {
        dp[p].upload(parts[p], n, st);
        ptrs.push_back(dp[p].p);
    }
    DBuf<const u32*> dptrs;
    dptrs.upload(ptrs, st);
    DBuf<u32> dnl, idx, codes;
    DBuf<u64> keys;
    dnl.upload(nl, st);
    keys.alloc(n);
    idx.alloc(n);
    codes.alloc(n);
    k_prep_combine_keys<<<grid_of(n, 256), 256, 0, st>>>(dptrs.p, dnl.p, int(parts.size()), n, keys.p, idx.p);
    const u32 nlev = codes_of_keys(keys.p, idx.p, n, codes.p, st);
    CK(cudaMemcpyAsync(codes_out, codes.p, n * sizeof(u32), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return nlev;
}

DropCounts prep_drop(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n, const double* fw,
                     const double* y, int family, bool singletons, uint8_t* alive) {
    DropCounts out;
    const size_t nterms = codes.size();
    if (nterms == 0 || n == 0 || (!singletons && family == 0)) return out;
    Stream S;
    cudaStream_t st = S.st;
    AllocScope alloc_scope(st);
    std::vector<DBuf<u32>> dc(nterms);
    for (size_t t = 0; t < nterms; t++) check_codes(codes[t], n, g[t], "fereg_drop_singletons");
    for (size_t t = 0; t < nterms; t++) dc[t].upload(codes[t], n, st);
    DBuf<uint8_t> dalive;
    DBuf<double> dfw, dy, cnt, pos;
    DBuf<unsigned long long> sf;
    dalive.upload(alive, n, st);
    if (fw) dfw.upload(fw, n, st);
    if (family && y) dy.upload(y, n, st);
    const u32 gmax = *std::max_element(g.begin(), g.end());
    cnt.alloc(gmax);
    pos.alloc(gmax);
    sf.alloc(2);
    // cycle over the terms in absorb order until nterms consecutive passes drop nothing
    size_t remaining = nterms, i = 0;
    while (remaining > 0) {
        const size_t t = i % nterms;
        i++;
        CK(cudaMemsetAsync(cnt.p, 0, g[t] * sizeof(double), st));
        CK(cudaMemsetAsync(pos.p, 0, g[t] * sizeof(double), st));
        CK(cudaMemsetAsync(sf.p, 0, 2 * sizeof(unsigned long long), st));
        k_sing_count<<<grid_of(n, 256), 256, 0, st>>>(dc[t].p, n, dalive.p, fw ? dfw.p : nullptr,
                                                      family && y ? dy.p : nullptr, cnt.p, pos.p);
        k_sing_drop<<<grid_of(n, 256), 256, 0, st>>>(dc[t].p, n, dalive.p, cnt.p, pos.p, singletons ? 1 : 0,
                                                     family && y ? family : 0, sf.p);
        unsigned long long h[2];
        CK(cudaMemcpyAsync(h, sf.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out.singletons += h[0];
        out.separated += h[1];
        remaining = h[0] + h[1] > 0 ? nterms - 1 : remaining - 1;
    }
    CK(cudaMemcpyAsync(alive, dalive.p, n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return out;
}

u32 prep_restrict(const u32* codes, u32 g, const uint8_t* alive, size_t n, u32* out, size_t* kept) {
    Stream S;
    cudaStream_t st = S.st;
    AllocScope alloc_scope(st);
    DBuf<u32> dc, present, level_rank, a32, kept_rank, dout;
    DBuf<uint8_t> dalive;
    check_codes(codes, n, g, "fereg_restrict");
    dc.upload(codes, n, st);
    dalive.upload(alive, n, st);
    present.alloc(std::max<u32>(1, g));
    level_rank.alloc(std::max<u32>(1, g));
    CK(cudaMemsetAsync(present.p, 0, std::max<u32>(1, g) * sizeof(u32), st));
    k_prep_present<<<grid_of(n, 256), 256, 0, st>>>(dc.p, n, dalive.p, present.p);
    const u32 nlev = excl_scan(present.p, g, level_rank.p, st);
    a32.alloc(n);
    kept_rank.alloc(n);
    k_prep_alive_u32<<<grid_of(n, 256), 256, 0, st>>>(dalive.p, n, a32.p);
    const u32 nk = excl_scan(a32.p, n, kept_rank.p, st);
    dout.alloc(std::max<u32>(1, nk));
    k_prep_restrict<<<grid_of(n, 256), 256, 0, st>>>(dc.p, n, dalive.p, kept_rank.p, level_rank.p, dout.p);
    if (nk) CK(cudaMemcpyAsync(out, dout.p, size_t(nk) * sizeof(u32), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    if (kept) *kept = nk;
    return nlev;
}

}  // namespace fereg
