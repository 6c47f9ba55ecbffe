// Kernels for the short lists: segments of at most WT cells (and WT rows) and coordinate lists
// of at most PULL_WARP_MAX entries. Longer lists go to the CTA tiles (tiles.cuh).
//
// The operator's passes (k_vseg_apply, k_vpull_apply) run on the PCG's padded vectors (a row
// stride that is a multiple of 4): lane j of a group of L lanes holds 4 consecutive columns,
// gathered with 16-byte loads. The segment pass gives each group one segment at a time and the
// group walks its cells in order; the list pass deals a list's entries to the groups and adds
// their sums in group order.
//
// The right-hand side's segment pass (k_grhs) uses lane groups over the caller's rows: lane j of
// a group holds columns j and j + L of the launch's column chunk; the group loads the indices of
// L cells at once, one per lane and coalesced, and takes the cells in turn with the indices
// broadcast by shuffles. The small coordinates accumulate in lane-private shared slots that the
// CTA adds in a fixed order.
//
// The right-hand side's list pass and the residualization use warp tiles: a warp takes whole
// consecutive segments (at most WSEG segments, WT cells and WT rows in all) or whole consecutive
// coordinate lists (at most PULL_WARP_MAX entries). The tile's indices are staged first, one lane
// per cell, segment or entry, into the warp's shared memory. Then every loop runs on all lanes as
// (group g, column j) pairs: a column chunk of Rc columns is padded to RCP (a power of two), the
// warp holds G = 32 / RCP groups, and cells and rows are dealt to the groups in turn (cell i to
// group i mod G). Segment sums: while a lane walks its cells (in order) it keeps a running sum of
// the current segment and parks it in a lane-private slot when the segment ends; the segment's
// value is then the sum of its G slots in group order.
//
// Every lane's sums run in a fixed order: results do not depend on timing. The number of blocks
// is a template parameter NBK (the exact count up to WNB - 1; WNB means WNB or more, the ones past
// WNB read from global memory).
#pragma once

#include "bulk.cuh"
#include "tiles.cuh"

namespace fereg {

constexpr int WT = 32;                // cells (rows) per segment tile
constexpr int WSEG = 8;               // segments per segment tile
constexpr int WCOLS = 32;             // columns per launch of the warp kernels
constexpr int WPB = 8;                // warps per CTA
constexpr u32 PULL_WARP_MAX = 256;    // entries of the coordinate lists of one list tile
constexpr int WLIST = 32;             // lists per list tile
constexpr int WNB = 4;                // blocks whose coordinates a segment tile stages
constexpr int WNO = WNB - 1;          // other blocks whose coordinates a list tile stages

// Warp tiles over short lists: (k0, k1, e0, e1) = lists [k0, k1) covering entries [e0, e1).
struct WarpTiles {
    u32 n;
    const uint4* t;
};

__device__ __forceinline__ u32 wlane() { return threadIdx.x & 31u; }
__device__ __forceinline__ u32 wid_in_cta() { return threadIdx.x >> 5; }

// The block-count key.
__host__ __device__ constexpr int nbk_of(u32 nb) { return nb < u32(WNB) ? int(nb) : WNB; }

// Lane = (group g, column j) for a chunk padded to RCP columns.
template <int RCP>
struct Lanes {
    static constexpr int G = 32 / RCP;
    static constexpr int KN = WT / G;           // tile cells (rows) per group
    static constexpr int CH = KN < 8 ? KN : 8;  // loads held in registers at once
    u32 lane, g, j;
    bool on;
    __device__ __forceinline__ explicit Lanes(int Rc)
        : lane(wlane()), g(wlane() / RCP), j(wlane() % RCP), on(int(wlane() % RCP) < Rc) {}
};

// Sum of v over the groups (same column), groups in order; every lane gets its column's sum.
template <int RCP, class T>
__device__ __forceinline__ T group_total(T v, const Lanes<RCP>& L) {
    if constexpr (RCP == 32) {
        return v;
    } else {
        T s = T(0);
#pragma unroll
        for (int g = 0; g < 32 / RCP; g++) s += __shfl_sync(FULL, v, g * RCP + int(L.j));
        return s;
    }
}

__host__ __device__ constexpr size_t al16(size_t b) { return (b + 15) / 16 * 16; }

// Per-warp staging of a segment tile.
struct SegStage {
    u32* send;    // local end (cell) of each segment of the tile (WSEG)
    double* n1i;  // 1/n1 of each segment (WSEG)
    double* cw;   // cell weights
    u32* code;    // block coordinates of the cells (WNB x WT)
    u32* row0;    // first row of each cell (WT + 1), rows passes
    u32* rcell;   // local cell of each local row, rows passes
    u32* segl;    // local segment of each cell
};
__host__ __device__ constexpr size_t segstage_bytes() {
    return al16(WSEG * 4) + al16(WSEG * 8) + al16(WT * 8) + al16(WNB * WT * 4) + al16((WT + 1) * 4) + 2 * al16(WT * 4);
}
__device__ __forceinline__ SegStage seg_stage_at(unsigned char* p) {
    SegStage s;
    s.send = reinterpret_cast<u32*>(p);
    p += al16(WSEG * 4);
    s.n1i = reinterpret_cast<double*>(p);
    p += al16(WSEG * 8);
    s.cw = reinterpret_cast<double*>(p);
    p += al16(WT * 8);
    s.code = reinterpret_cast<u32*>(p);
    p += al16(WNB * WT * 4);
    s.row0 = reinterpret_cast<u32*>(p);
    p += al16((WT + 1) * 4);
    s.rcell = reinterpret_cast<u32*>(p);
    p += al16(WT * 4);
    s.segl = reinterpret_cast<u32*>(p);
    return s;
}

// Bytes per warp (Rc columns): per-cell values u (WT x Rc), lane-private segment slots ps
// (WSEG x 32), the staging; the residualization adds the tile's b1 (WSEG x Rc).
__host__ __device__ constexpr size_t wseg_bytes(int Rc, size_t tsz) {
    return al16(WT * Rc * tsz) + al16(WSEG * 32 * tsz) + segstage_bytes();
}
__host__ __device__ constexpr size_t wresid_bytes(int Rc) { return wseg_bytes(Rc, 8) + al16(WSEG * Rc * 8); }

// Stages the tile's per-segment scalars and the cells' weights, first `ncode` block coordinates
// and (with `rows`, non-trivial cells) first rows. The caller syncs the warp afterwards.
__device__ __forceinline__ void stage_cells(const DevStruct& S, const DevWeights& W, u32 s0, u32 s1, u32 c0, u32 c1,
                                            const SegStage& st, u32 ncode, bool rows) {
    const u32 lane = wlane();
    if (lane < s1 - s0) {
        st.send[lane] = S.seg_off[s0 + lane + 1] - c0;
        st.n1i[lane] = W.n1inv[s0 + lane];
    }
    const u32 c = c0 + lane;
    if (c < c1) {
        st.cw[lane] = cellw(W, c);
#pragma unroll
        for (u32 b = 0; b < u32(WNB); b++)
            if (b < ncode) st.code[b * WT + lane] = __ldcs(S.coord + size_t(b) * S.M + c);
        if (rows && S.cell_row) {
            st.row0[lane] = S.cell_row[c];
            if (c == c1 - 1) st.row0[lane + 1] = S.cell_row[c + 1];
        }
    }
}

// After the staging (and a __syncwarp): local segment of each cell and, for non-trivial cells
// in the rows passes, local cell of each tile row.
__device__ __forceinline__ void stage_maps(u32 nc, const SegStage& st, bool rcell) {
    const u32 lane = wlane();
    if (lane < nc) {
        u32 s = 0;
        while (st.send[s] <= lane) s++;
        st.segl[lane] = s;
        if (rcell) {
            const u32 base = st.row0[0];
            for (u32 r = st.row0[lane] - base; r < st.row0[lane + 1] - base; r++) st.rcell[r] = lane;
        }
    }
}

// Sum over the blocks of src[coord_b(cell)]: code points at the cell's staged coordinates
// (stride WT per block), src at this lane's column, ci = the cell's global index.
template <int NBK, class T>
__device__ __forceinline__ T gather_cell(const DevStruct& S, const u32* code, const T* __restrict__ src, u32 Ru,
                                         u32 ci) {
    T v = T(0);
#pragma unroll
    for (int b = 0; b < NBK; b++) v += src[size_t(code[b * WT]) * Ru];
    if constexpr (NBK == WNB)
        for (u32 b = WNB; b < S.nb; b++) v += src[size_t(S.coord[size_t(b) * S.M + ci]) * Ru];
    return v;
}

// Running sum of a lane over the tile's segments (its cells come in segment order): the sum of
// each segment is parked in the lane-private slot ps[segment * 32 + lane] (0 when the lane has
// no cell of the segment).
template <class T>
struct SegRun {
    u32 cur = 0;
    T run = T(0);
    __device__ __forceinline__ void add(u32 s, T w, T* ps, u32 lane) {
        while (cur < s) {
            ps[cur * 32 + lane] = run;
            run = T(0);
            cur++;
        }
        run += w;
    }
    __device__ __forceinline__ void finish(u32 ns, T* ps, u32 lane) {
        while (cur < ns) {
            ps[cur * 32 + lane] = run;
            run = T(0);
            cur++;
        }
    }
};

// Segment value of column j: the groups' slots added in group order.
template <int RCP, class T>
__device__ __forceinline__ T seg_total(const T* ps, u32 sl, u32 j) {
    T s = T(0);
#pragma unroll
    for (int g = 0; g < 32 / RCP; g++) s += ps[sl * 32 + g * RCP + j];
    return s;
}

// ---------------------------------------------------------------------------------------------
// Lane groups over the short segments: a group of L lanes takes one segment at a time, lane j of
// the group holding columns j and j + L of the launch's column chunk (L = lanes_of(Rc): two
// columns per lane, so 32 / L cells share every warp instruction). The small coordinates' sums
// sit in lane-private shared slots, two per small code: slot(k, c) = (2k + c) * 32 + lane.
__host__ __device__ constexpr int lanes_of(int Rc) { return rcp_of((Rc + 1) / 2); }

// CTA end of the lane-group kernels: adds the lane-private small-coordinate slots of the warps and
// groups, in that order, into the CTA's partial row (cta_small[blockIdx][k * R + j0 + col]).
template <int L, class T>
__device__ __forceinline__ void flush_pairs(const T* wacc_all, u32 ms_acc, int Rc, int j0, int R, T* cta_small) {
    __syncthreads();
    T* mine = cta_small + size_t(blockIdx.x) * ms_acc * R;
    for (u32 i = threadIdx.x; i < ms_acc * u32(Rc); i += blockDim.x) {
        const u32 k = i / u32(Rc), col = i % u32(Rc), c = col / u32(L), j = col % u32(L);
        T s = T(0);
        for (int w = 0; w < WPB; w++)
#pragma unroll
            for (int g = 0; g < 32 / L; g++) s += wacc_all[((size_t(w) * ms_acc + k) * 2 + c) * 32 + g * L + j];
        mine[size_t(k) * R + j0 + col] = s;
    }
}

// ---------------------------------------------------------------------------------------------
// The operator's passes on the PCG's padded vectors (row stride Rv, a multiple of 4, 16-byte
// aligned rows): lane j of a group of L lanes holds the 4 consecutive columns j0 + 4j .. j0 + 4j + 3
// of the launch's chunk, gathered with 16-byte loads (two per row in FP64, one in FP32).
constexpr int VCOLS = 128;  // columns per launch of the padded-vector passes (32 lanes x 4)

template <class T>
struct V4 {
    T a, b, c, d;
};
__device__ __forceinline__ V4<double> ld4(const double* p) {
    const double2 x = __ldg(reinterpret_cast<const double2*>(p));
    const double2 y = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return V4<double>{x.x, x.y, y.x, y.y};
}
__device__ __forceinline__ V4<float> ld4(const float* p) {
    const float4 x = __ldg(reinterpret_cast<const float4*>(p));
    return V4<float>{x.x, x.y, x.z, x.w};
}
// L2-coherent load of values written earlier in the same pass sequence (t)
__device__ __forceinline__ V4<double> ld4cg(const double* p) {
    const double2 x = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 y = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return V4<double>{x.x, x.y, y.x, y.y};
}
__device__ __forceinline__ V4<float> ld4cg(const float* p) {
    const float4 x = __ldcg(reinterpret_cast<const float4*>(p));
    return V4<float>{x.x, x.y, x.z, x.w};
}
__device__ __forceinline__ void st4(double* p, const V4<double>& v) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v.a, v.b);
    reinterpret_cast<double2*>(p)[1] = make_double2(v.c, v.d);
}
__device__ __forceinline__ void st4(float* p, const V4<float>& v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.a, v.b, v.c, v.d);
}
template <class T>
__device__ __forceinline__ void add4(V4<T>& s, const V4<T>& v) {
    s.a += v.a;
    s.b += v.b;
    s.c += v.c;
    s.d += v.d;
}
template <class T>
__device__ __forceinline__ void sub4(V4<T>& s, const V4<T>& v) {
    s.a -= v.a;
    s.b -= v.b;
    s.c -= v.c;
    s.d -= v.d;
}
template <class T>
__device__ __forceinline__ void fma4(V4<T>& s, T w, const V4<T>& v) {
    s.a += w * v.a;
    s.b += w * v.b;
    s.c += w * v.c;
    s.d += w * v.d;
}
// The rows of the small coordinates (0 .. ms_acc - 1, the first blocks) of the launch's column
// chunk, staged in shared memory once per CTA: every cell holds one of them per small block, and a
// gather from shared memory spares the L1 the tag and line work of a global gather.
template <class T>
__device__ __forceinline__ void stage_small(T* sp, const T* __restrict__ P, size_t Ru, int j0, int Rc, u32 ms) {
    for (u32 i = threadIdx.x; i < ms * u32(Rc); i += blockDim.x)
        sp[i] = P[size_t(i / u32(Rc)) * Ru + j0 + i % u32(Rc)];
    __syncthreads();
}
__device__ __forceinline__ V4<double> ld4s(const double* p) {
    const double2 x = reinterpret_cast<const double2*>(p)[0];
    const double2 y = reinterpret_cast<const double2*>(p)[1];
    return V4<double>{x.x, x.y, y.x, y.y};
}
__device__ __forceinline__ V4<float> ld4s(const float* p) {
    const float4 x = *reinterpret_cast<const float4*>(p);
    return V4<float>{x.x, x.y, x.z, x.w};
}
// Shared memory of the staged small rows for an Rc-column chunk (0: none staged).
template <class T>
__host__ __device__ constexpr size_t small_stage_bytes(u32 ms, int Rc) {
    return al16(size_t(ms) * size_t(Rc) * sizeof(T));
}

// Lanes per group for an Rc-column chunk (Rc a multiple of 4).
__host__ __device__ constexpr int vlanes_of(int Rc) { return rcp_of((Rc + 3) / 4); }

// Sum over the blocks of the rows P[coord_b(c)] (this lane's 4 columns): the first NL blocks'
// coordinates in `code`, the ones past WNB (NBK == WNB) read from the structure.
template <int NBK, class T>
__device__ __forceinline__ V4<T> gather4(const DevStruct& S, const u32* code, const T* __restrict__ Pj, size_t Ru,
                                         u32 c, const T* spj, int nsm, int Rc) {
    constexpr int NL = NBK < WNB ? NBK : WNB;
    // the first nsm blocks are small, their rows staged at spj (stride Rc)
    V4<T> u = nsm > 0 ? ld4s(spj + size_t(code[0]) * Rc) : ld4(Pj + size_t(code[0]) * Ru);
#pragma unroll
    for (int b = 1; b < NL; b++) add4(u, b < nsm ? ld4s(spj + size_t(code[b]) * Rc) : ld4(Pj + size_t(code[b]) * Ru));
    if constexpr (NBK == WNB)
        for (u32 b = WNB; b < S.nb; b++) add4(u, ld4(Pj + size_t(__ldg(S.coord + size_t(b) * S.M + c)) * Ru));
    return u;
}

// Operator pass 1 (operator.rs:894-948) on the short segments, one segment per lane group:
// t_s = n1inv_s sum_c W_c u_c with u_c = sum_b P[coord_b(c)]. segs lists the short segments in
// order; group q of the grid takes segs[q], segs[q + groups], ... Each group walks its segment's
// cells in order, two cells' gathers in flight together, the lanes' sums in cell order.
template <class T, int L, int NBK, bool WEIGHTED>
__global__ void __launch_bounds__(WPB * 32, 4) k_vseg_apply(DevStruct S, DevWeights W, const u32* __restrict__ segs,
                                                            u32 nsegs, const T* __restrict__ P, int Rv, int j0, int Rc,
                                                            T* __restrict__ t, int stage) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int G = 32 / L;
    constexpr int NL = NBK < WNB ? NBK : WNB;
    const u32 lane = wlane(), g = lane / L, j = lane % L;
    const bool on = int(4 * j) < Rc;
    const size_t Ru = size_t(Rv);
    const T* Pj = P + j0 + 4 * j;
    T* sp = reinterpret_cast<T*>(smem_raw);
    const int nsm = stage ? int(S.ns_acc) : 0;
    if (nsm) stage_small(sp, P, Ru, j0, Rc, S.ms_acc);
    const T* spj = sp + 4 * j;
    const u32 groups = gridDim.x * WPB * G;
    for (u32 q = (blockIdx.x * WPB + wid_in_cta()) * G + g; q < nsegs; q += groups) {
        const u32 s = segs[q];
        const u32 c0 = S.seg_off[s], c1 = S.seg_off[s + 1];
        V4<T> acc{T(0), T(0), T(0), T(0)};
        if (on) {
            u32 c = c0;
            for (; c + 2 <= c1; c += 2) {
                u32 k0[NL], k1[NL];
#pragma unroll
                for (int b = 0; b < NL; b++) {
                    k0[b] = __ldg(S.coord + size_t(b) * S.M + c);
                    k1[b] = __ldg(S.coord + size_t(b) * S.M + c + 1);
                }
                const V4<T> u0 = gather4<NBK>(S, k0, Pj, Ru, c, spj, nsm, Rc);
                const V4<T> u1 = gather4<NBK>(S, k1, Pj, Ru, c + 1, spj, nsm, Rc);
                if constexpr (WEIGHTED) {
                    fma4(acc, T(W.cell_w[c]), u0);
                    fma4(acc, T(W.cell_w[c + 1]), u1);
                } else {
                    add4(acc, u0);
                    add4(acc, u1);
                }
            }
            if (c < c1) {
                u32 k0[NL];
#pragma unroll
                for (int b = 0; b < NL; b++) k0[b] = __ldg(S.coord + size_t(b) * S.M + c);
                const V4<T> u0 = gather4<NBK>(S, k0, Pj, Ru, c, spj, nsm, Rc);
                if constexpr (WEIGHTED) fma4(acc, T(W.cell_w[c]), u0);
                else add4(acc, u0);
            }
            const T n1i = T(W.n1inv[s]);
            st4(t + size_t(s) * Ru + j0 + 4 * j, V4<T>{acc.a * n1i, acc.b * n1i, acc.c * n1i, acc.d * n1i});
        }
    }
}

// Staging of a coordinate-list tile: list ends and the entries' indices.
struct PullStage {
    u32* kend;  // local end (entry) of each list (WLIST lists at most)
    u32* seg;   // PULL_WARP_MAX entries
    u32* cell;
    u32* oth;   // WNO x PULL_WARP_MAX
};
__host__ __device__ constexpr size_t pull_bytes() {
    return al16(WLIST * 4) + al16(PULL_WARP_MAX * 4) * 2 + al16(WNO * PULL_WARP_MAX * 4);
}
__device__ __forceinline__ PullStage pull_stage_at(unsigned char* p) {
    PullStage s;
    s.kend = reinterpret_cast<u32*>(p);
    p += al16(WLIST * 4);
    s.seg = reinterpret_cast<u32*>(p);
    p += al16(PULL_WARP_MAX * 4);
    s.cell = reinterpret_cast<u32*>(p);
    p += al16(PULL_WARP_MAX * 4);
    s.oth = reinterpret_cast<u32*>(p);
    return s;
}

__device__ __forceinline__ void stage_pull(const DevStruct& S, u32 k0, u32 k1, u32 e0, u32 e1, const PullStage& st,
                                           bool cells, u32 nstage) {
    const u32 lane = wlane();
    if (lane < k1 - k0) st.kend[lane] = S.pl_off[k0 + lane + 1] - e0;
    const u32 no = S.nb - 1;
    for (u32 i = lane; i < e1 - e0; i += 32) {
        const u32 e = e0 + i;
        st.seg[i] = __ldcs(S.pl_seg + e);
        if (cells) st.cell[i] = __ldcs(S.pl_cell + e);
#pragma unroll
        for (u32 o = 0; o < u32(WNO); o++)
            if (o < nstage) st.oth[o * PULL_WARP_MAX + i] = __ldcs(S.pl_other + size_t(e) * no + o);
    }
}

// Per-warp buffer of the list pass's software pipeline: the tile's list ends (pl_off, global
// entry indices), and per entry its segment, cell (weighted cells only) and NO other coordinates.
template <int NO, bool WEIGHTED>
__host__ __device__ constexpr size_t vpull_buf_bytes() {
    return al16(WLIST * 4) + al16(PULL_WARP_MAX * 4) * (1 + (WEIGHTED ? 1 : 0) + NO);
}
// Per-warp shared memory of the list pass: two pipeline buffers, or (weighted cells) one stage.
template <int NO, bool WEIGHTED>
__host__ __device__ constexpr size_t vpull_warp_bytes() {
    return WEIGHTED ? pull_bytes() : 2 * vpull_buf_bytes<NO, WEIGHTED>();
}
struct VPullBuf {
    u32* kend;
    u32* seg;
    u32* cell;
    u32* oth;  // NO x PULL_WARP_MAX
};
template <int NO, bool WEIGHTED>
__device__ __forceinline__ VPullBuf vpull_buf_at(unsigned char* p) {
    VPullBuf b;
    b.kend = reinterpret_cast<u32*>(p);
    p += al16(WLIST * 4);
    b.seg = reinterpret_cast<u32*>(p);
    p += al16(PULL_WARP_MAX * 4);
    b.cell = reinterpret_cast<u32*>(p);
    if (WEIGHTED) p += al16(PULL_WARP_MAX * 4);
    b.oth = reinterpret_cast<u32*>(p);
    return b;
}
// Issues the copies of list tile tb into buffer b (the caller commits the group).
template <int NO, bool WEIGHTED>
__device__ __forceinline__ void vpull_prefetch(const DevStruct& S, const uint4& tb, const VPullBuf& b) {
    const u32 lane = wlane(), k0 = tb.x, k1 = tb.y, e0 = tb.z, ne = tb.w - tb.z;
    const u32 no = S.nb - 1;
    if (lane < k1 - k0) cp_async4(b.kend + lane, S.pl_off + k0 + lane + 1);
    for (u32 i = lane; i < ne; i += 32) {
        cp_async4(b.seg + i, S.pl_seg + e0 + i);
        if (WEIGHTED) cp_async4(b.cell + i, S.pl_cell + e0 + i);
#pragma unroll
        for (int o = 0; o < NO; o++) cp_async4(b.oth + o * PULL_WARP_MAX + i, S.pl_other + size_t(e0 + i) * no + o);
    }
}

// Operator pass 2 on short coordinate lists (k >= ms_acc) with the padded vectors:
// Y[k] = nr_k P[k] + sum over the cells c of k of W_c (sum_{other b} P[coord_b(c)] - t_{s(c)}).
// Warp tiles of whole lists; the entries are dealt to groups of L lanes (lane j holding 4
// columns), and the groups' sums are added by a fixed xor butterfly. Unweighted cells: software
// pipelined, cp.async copies bring the next tile's list ends and entries' segments and other
// coordinates into the second of two shared buffers while a warp works on one tile (measured:
// the 1e6-row bootstrap panel's list pass 8% faster). Weighted cells stage each tile before
// working on it, in the shared memory they always took (the pipelined form, with its larger
// buffers, measured 1.7x slower on the gravity panel's weighted lists).
template <class T, int L, int NBK, bool WEIGHTED>
__global__ void __launch_bounds__(WPB * 32, 4) k_vpull_apply(DevStruct S, DevWeights W, WarpTiles wt,
                                                             const T* __restrict__ P, const T* __restrict__ t, int Rv,
                                                             int j0, int Rc, T* __restrict__ Y, int stage) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int G = 32 / L;
    constexpr int NO = NBK - 1;  // staged other blocks (all of them below WNB blocks)
    constexpr u32 BB = u32(vpull_buf_bytes<NO, WEIGHTED>());
    constexpr u32 WS = u32(vpull_warp_bytes<NO, WEIGHTED>());
    unsigned char* mine = smem_raw + size_t(wid_in_cta()) * WS;
    const u32 lane = wlane(), g = lane / L, j = lane % L;
    const bool on = int(4 * j) < Rc;
    const size_t Ru = size_t(Rv);
    const u32 no = S.nb - 1;
    const T* Pj = P + j0 + 4 * j;
    const T* tj = t + j0 + 4 * j;
    // the lists are of large coordinates: the small blocks come first among a cell's other blocks
    T* sp = reinterpret_cast<T*>(smem_raw + size_t(WPB) * WS);
    const int nsm = stage ? int(S.ns_acc) : 0;
    if (nsm) stage_small(sp, P, Ru, j0, Rc, S.ms_acc);
    const T* spj = sp + 4 * j;
    auto total = [&](T v) {  // sum over the groups of the same lane slot, a fixed butterfly
#pragma unroll
        for (int o = L; o < 32; o <<= 1) v += __shfl_xor_sync(FULL, v, o);
        return v;
    };
    // the lists of one staged tile; kend[kl] - kbase: local end of list kl
    auto work = [&](const u32* kend, u32 kbase, const u32* seg, const u32* cell, const u32* oth, u32 k0, u32 k1,
                    u32 e0) {
        u32 i0 = 0;
        for (u32 kl = 0; kl < k1 - k0; kl++) {
            const u32 ie = kend[kl] - kbase;
            V4<T> acc{T(0), T(0), T(0), T(0)};
            if (on) {
#pragma unroll 4
                for (u32 i = i0 + g; i < ie; i += G) {
                    V4<T> v = ld4cg(tj + size_t(seg[i]) * Ru);
                    v.a = -v.a;
                    v.b = -v.b;
                    v.c = -v.c;
                    v.d = -v.d;
#pragma unroll
                    for (int o = 0; o < NO; o++) {
                        const u32 x = oth[o * PULL_WARP_MAX + i];
                        add4(v, o < nsm ? ld4s(spj + size_t(x) * Rc) : ld4(Pj + size_t(x) * Ru));
                    }
                    if constexpr (NBK == WNB)
                        for (u32 o = WNO; o < no; o++)
                            add4(v, ld4(Pj + size_t(S.pl_other[size_t(e0 + i) * no + o]) * Ru));
                    if constexpr (WEIGHTED) fma4(acc, T(W.cell_w[cell[i]]), v);
                    else add4(acc, v);
                }
            }
            acc.a = total(acc.a);
            acc.b = total(acc.b);
            acc.c = total(acc.c);
            acc.d = total(acc.d);
            if (g == 0 && on) {
                const size_t o = size_t(k0 + kl) * Ru + j0 + 4 * j;
                const T nrk = T(W.nr[k0 + kl]);
                const V4<T> pk = ld4(P + o);
                st4(Y + o, V4<T>{nrk * pk.a + acc.a, nrk * pk.b + acc.b, nrk * pk.c + acc.c, nrk * pk.d + acc.d});
            }
            i0 = ie;
        }
    };
    const u32 wid = blockIdx.x * WPB + wid_in_cta(), nw = gridDim.x * WPB;
    uint4 tb = wid < wt.n ? wt.t[wid] : make_uint4(0, 0, 0, 0);
    if constexpr (WEIGHTED) {
        const PullStage st = pull_stage_at(mine);
        for (u32 tile = wid; tile < wt.n; tile += nw) {
            const u32 k0 = tb.x, k1 = tb.y, e0 = tb.z;
            stage_pull(S, k0, k1, e0, tb.w, st, true, u32(NO));
            if (tile + nw < wt.n) tb = wt.t[tile + nw];
            __syncwarp();
            work(st.kend, 0u, st.seg, st.cell, st.oth, k0, k1, e0);
            __syncwarp();
        }
    } else {
        uint4 tn = wid + nw < wt.n ? wt.t[wid + nw] : make_uint4(0, 0, 0, 0);  // the next tile
        if (wid < wt.n) vpull_prefetch<NO, WEIGHTED>(S, tb, vpull_buf_at<NO, WEIGHTED>(mine));
        cp_async_commit();
        u32 it = 0;
        for (u32 tile = wid; tile < wt.n; tile += nw, it++) {
            const VPullBuf b = vpull_buf_at<NO, WEIGHTED>(mine + (it & 1) * BB);
            if (tile + nw < wt.n)
                vpull_prefetch<NO, WEIGHTED>(S, tn, vpull_buf_at<NO, WEIGHTED>(mine + ((it + 1) & 1) * BB));
            cp_async_commit();
            const uint4 tc = tb;
            tb = tn;
            if (tile + 2 * nw < wt.n) tn = wt.t[tile + 2 * nw];
            cp_async_wait_prior();  // this tile's copies
            __syncwarp();
            work(b.kend, tc.z, b.seg, b.cell, b.oth, tc.x, tc.y, tc.z);
            __syncwarp();
        }
        cp_async_wait_all();
    }
}

// ---------------------------------------------------------------------------------------------
// Right-hand side pass 1 (operator.rs:969-1066) on the short segments, one segment per lane group
// in the order of k_vseg_apply: b1_s = sum over the segment's rows of w v; per-CTA partials of
// [sum w v^2, sum w v] (cta_part[blockIdx][2R], this chunk's columns); the small coordinates take
// sum_c s_c - (b1_s / n1_s) sum_c W_c per small code (s_c: the sum over the rows of cell c). The
// group streams its segment's rows (contiguous in the block): with one row per cell, in chunks of
// L rows whose small codes and weights lane i loads for row i, four rows' loads in flight;
// otherwise cell by cell over the cell's rows.
// NSA: the small blocks summed (S.ns_acc when the small coordinates are accumulated, else 0).
template <int L, int NSA>
__global__ void __launch_bounds__(WPB * 32, 4) k_grhs(DevStruct S, DevWeights W, const u32* __restrict__ segs,
                                                      u32 nsegs, const double* __restrict__ rows, int R, int j0,
                                                      int Rc, double* __restrict__ b1, double* __restrict__ cta_part,
                                                      double* __restrict__ cta_small) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int G = 32 / L;
    constexpr int U = 4;  // rows whose loads are in flight together (two columns each)
    double* wacc_all = reinterpret_cast<double*>(smem_raw);
    double* colsum = wacc_all + size_t(WPB) * S.ms_acc * 64;  // WPB x 4 x 32: [q c0, q c1, ws c0, ws c1]
    constexpr bool acc = NSA > 0;
    const bool trivial = S.cell_row == nullptr;
    const u32 lane = wlane(), g = lane / L, j = lane % L;
    const bool on0 = int(j) < Rc, on1 = int(j) + L < Rc;
    const unsigned gmask = L == 32 ? FULL : ((1u << L) - 1u) << (g * L);
    const size_t Ru = size_t(R);
    constexpr int ns_acc = NSA;
    double* wacc = wacc_all + size_t(wid_in_cta()) * S.ms_acc * 64 + lane;
    if (acc)
        for (u32 i = 0; i < S.ms_acc * 2; i++) wacc[i * 32] = 0.0;
    double qa = 0.0, qb = 0.0, wa = 0.0, wb = 0.0;  // this lane's [sum w v^2, sum w v], both columns
    const double* vj = rows + j0 + j;
    const u32 groups = gridDim.x * WPB * G;
    u32 q = (blockIdx.x * WPB + wid_in_cta()) * G + g;
    u32 s = q < nsegs ? segs[q] : 0;
    for (; q < nsegs; q += groups) {
        const u32 c0 = S.seg_off[s], c1 = S.seg_off[s + 1];
        const u32 qn = q + groups;
        const u32 sn = qn < nsegs ? segs[qn] : 0;
        double sum0 = 0.0, sum1 = 0.0;
        for (u32 cb = c0; cb < c1; cb += L) {
            const u32 nc = min(c1 - cb, u32(L));
            u32 code[WNB];
#pragma unroll
            for (int b = 0; b < WNB; b++)
                code[b] = (b < ns_acc && j < nc) ? __ldg(S.coord + size_t(b) * S.M + cb + j) : 0u;
            if (trivial) {
                const double wl = (W.w_rows && j < nc) ? W.w_rows[cb + j] : 1.0;
                for (u32 i0 = 0; i0 < nc; i0 += U) {
                    double x0[U], x1[U];
#pragma unroll
                    for (int k = 0; k < U; k++) {
                        const u32 i = i0 + u32(k);
                        const double* row = vj + size_t(cb + i) * Ru;
                        x0[k] = (on0 && i < nc) ? __ldcs(row) : 0.0;
                        x1[k] = (on1 && i < nc) ? __ldcs(row + L) : 0.0;
                    }
#pragma unroll
                    for (int k = 0; k < U; k++) {
                        const u32 i = i0 + u32(k);
                        const double w = W.w_rows ? __shfl_sync(gmask, wl, int(i), L) : 1.0;
                        const double v0 = w * x0[k], v1 = w * x1[k];
                        qa += v0 * x0[k];
                        qb += v1 * x1[k];
                        sum0 += v0;
                        sum1 += v1;
#pragma unroll
                        for (int b = 0; b < WNB; b++)
                            if (b < ns_acc) {
                                double* sl = wacc + __shfl_sync(gmask, code[b], int(i), L) * 64;
                                if (i < nc) {  // slots of columns past Rc are never read
                                    if (on0) sl[0] += v0;
                                    if (on1) sl[32] += v1;
                                }
                            }
                    }
                }
            } else {
                const u32 rb = j < nc ? S.cell_row[cb + j] : 0u;  // lane i: first row of cell i
                const u32 rend = S.cell_row[cb + nc];                // end of the chunk's last cell
                for (u32 i = 0; i < nc; i++) {
                    const u32 r0 = __shfl_sync(gmask, rb, int(i), L);
                    const u32 rn = __shfl_sync(gmask, rb, int(i) + 1, L);
                    const u32 r1 = i + 1 < nc ? rn : rend;
                    double s0 = 0.0, s1 = 0.0;
                    for (u32 r = r0; r < r1; r++) {
                        const double* row = vj + size_t(r) * Ru;
                        const double a0 = on0 ? __ldcs(row) : 0.0, a1 = on1 ? __ldcs(row + L) : 0.0;
                        const double w = W.w_rows ? W.w_rows[r] : 1.0;
                        const double v0 = w * a0, v1 = w * a1;
                        s0 += v0;
                        s1 += v1;
                        qa += v0 * a0;
                        qb += v1 * a1;
                    }
                    sum0 += s0;
                    sum1 += s1;
#pragma unroll
                    for (int b = 0; b < WNB; b++)
                        if (b < ns_acc) {
                            double* sl = wacc + __shfl_sync(gmask, code[b], int(i), L) * 64;
                            if (on0) sl[0] += s0;
                            if (on1) sl[32] += s1;
                        }
                }
            }
        }
        wa += sum0;
        wb += sum1;
        if (on0) b1[size_t(s) * Ru + j0 + j] = sum0;
        if (on1) b1[size_t(s) * Ru + j0 + j + L] = sum1;
        if (acc) {
            const double n1i = W.n1inv[s];
            const double tv0 = sum0 * n1i, tv1 = sum1 * n1i;
            for (u32 cb = c0; cb < c1; cb += L) {
                const u32 nc = min(c1 - cb, u32(L));
                u32 code[WNB];
#pragma unroll
                for (int b = 0; b < WNB; b++)
                    code[b] = (b < ns_acc && j < nc) ? __ldg(S.coord + size_t(b) * S.M + cb + j) : 0u;
                const double wl = j < nc ? cellw(W, cb + j) : 1.0;
                for (u32 i = 0; i < nc; i++) {
                    const double w = __shfl_sync(gmask, wl, int(i), L);
                    const double d0 = w * tv0, d1 = w * tv1;
#pragma unroll
                    for (int b = 0; b < WNB; b++)
                        if (b < ns_acc) {
                            double* sl = wacc + __shfl_sync(gmask, code[b], int(i), L) * 64;
                            if (on0) sl[0] -= d0;
                            if (on1) sl[32] -= d1;
                        }
                }
            }
        }
        s = sn;
    }
    double* cs = colsum + size_t(wid_in_cta()) * 4 * 32 + lane;
    cs[0] = on0 ? qa : 0.0;
    cs[32] = on1 ? qb : 0.0;
    cs[64] = on0 ? wa : 0.0;
    cs[96] = on1 ? wb : 0.0;
    __syncthreads();
    for (u32 i = threadIdx.x; i < 2 * u32(Rc); i += blockDim.x) {
        const u32 half = i / u32(Rc), col = i % u32(Rc), c = col / u32(L), jj = col % u32(L);
        double a = 0.0;
        for (int w = 0; w < WPB; w++)
#pragma unroll
            for (int gg = 0; gg < G; gg++) a += colsum[(size_t(w) * 4 + half * 2 + c) * 32 + gg * L + jj];
        cta_part[size_t(blockIdx.x) * 2 * R + half * R + j0 + col] = a;
    }
    if (acc) flush_pairs<L>(wacc_all, S.ms_acc, Rc, j0, R, cta_small);
}

// Right-hand side pass 2 on short coordinate lists (k >= ms_acc): rhs[k] = sum over the cells c
// of k of (s_c - W_c b1_{s(c)} / n1_{s(c)}). The rows are gathered with the default cache policy:
// a row shares its sectors with the rows of neighbouring coordinates, which nearby warps read.
template <int RCP>
__global__ void __launch_bounds__(WPB * 32, 4) k_wpull_rhs(DevStruct S, DevWeights W, WarpTiles wt,
                                                           const double* __restrict__ rows,
                                                           const double* __restrict__ b1, int R, int j0, int Rc,
                                                           double* __restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using L_t = Lanes<RCP>;
    constexpr int G = L_t::G;
    const PullStage st = pull_stage_at(smem_raw + size_t(wid_in_cta()) * pull_bytes());
    const L_t L(Rc);
    const u32 Ru = u32(R);
    const bool trivial = S.cell_row == nullptr;
    const double* vj = rows + j0 + L.j;
    const double* bj = b1 + j0 + L.j;
    const u32 wid = blockIdx.x * WPB + wid_in_cta(), nw = gridDim.x * WPB;
    uint4 tb = wid < wt.n ? wt.t[wid] : make_uint4(0, 0, 0, 0);
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 k0 = tb.x, k1 = tb.y;
        stage_pull(S, k0, k1, tb.z, tb.w, st, true, 0u);
        if (tile + nw < wt.n) tb = wt.t[tile + nw];
        __syncwarp();
        // this lane's column summed over the entries ib, ib + step, ... < ie of a list
        auto list_sum = [&](u32 ib, u32 ie, u32 step) {
            double acc = 0.0;
            if (trivial) {
#pragma unroll 8
                for (u32 i = ib; i < ie; i += step) {
                    const u32 c = st.cell[i], s = st.seg[i];
                    const double x = __ldg(vj + size_t(c) * Ru);
                    const double sc = W.w_rows ? W.w_rows[c] * x : x;
                    acc += sc - cellw(W, c) * __ldcg(bj + size_t(s) * Ru) * W.n1inv[s];
                }
            } else {
#pragma unroll 4
                for (u32 i = ib; i < ie; i += step) {
                    const u32 c = st.cell[i], s = st.seg[i];
                    double sc = 0.0;
                    const u32 re = S.cell_row[c + 1];
                    for (u32 r = S.cell_row[c]; r < re; r++) {
                        const double x = __ldg(vj + size_t(r) * Ru);
                        sc += W.w_rows ? W.w_rows[r] * x : x;
                    }
                    acc += sc - cellw(W, c) * __ldcg(bj + size_t(s) * Ru) * W.n1inv[s];
                }
            }
            return acc;
        };
        const u32 nk = k1 - k0;
        if (G <= 2 && nk >= u32(G)) {
            // wide rows, two groups: group g takes the lists g, g + 2, ..., each list's entries in
            // order, so that the groups' gathers at one step read the rows of neighbouring
            // coordinates (neighbouring cells, sharing sectors)
            for (u32 kb = 0; kb < nk; kb += G) {
                const u32 kl = kb + L.g;
                if (L.on && kl < nk)
                    Y[size_t(k0 + kl) * Ru + j0 + L.j] = list_sum(kl ? st.kend[kl - 1] : 0u, st.kend[kl], 1u);
            }
        } else {
            // the groups share each list's entries; their sums are added in group order
            u32 i0 = 0;
            for (u32 kl = 0; kl < nk; kl++) {
                const u32 ie = st.kend[kl];
                double acc = L.on ? list_sum(i0 + L.g, ie, u32(G)) : 0.0;
                acc = group_total(acc, L);
                if (L.on && L.g == 0) Y[size_t(k0 + kl) * Ru + j0 + L.j] = acc;
                i0 = ie;
            }
        }
        __syncwarp();
    }
}

// Residualization of short segments (operator.rs:1107-1179): alpha_s = (b1_s - sum W_c u_c) / n1_s,
// u_c = sum_b x[coord_b(c)]; every row of cell c loses alpha_s + u_c.
template <int RCP, int NBK>
__global__ void __launch_bounds__(WPB * 32, 4) k_wresid(DevStruct S, DevWeights W, WarpTiles wt,
                                                        double* __restrict__ rows, int R, int j0, int Rc,
                                                        const double* __restrict__ x, const double* __restrict__ b1,
                                                        double* __restrict__ alpha) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using L_t = Lanes<RCP>;
    constexpr int G = L_t::G;
    constexpr int KS = (WSEG + G - 1) / G;  // tile segments per group
    unsigned char* mine = smem_raw + size_t(wid_in_cta()) * wresid_bytes(Rc);
    double* u = reinterpret_cast<double*>(mine);
    double* ps = reinterpret_cast<double*>(mine + al16(WT * Rc * 8));
    const SegStage st = seg_stage_at(mine + al16(WT * Rc * 8) + al16(WSEG * 32 * 8));
    double* bs = reinterpret_cast<double*>(mine + wseg_bytes(Rc, 8));  // the tile's b1 (WSEG x Rc)
    const bool trivial = S.cell_row == nullptr;
    const L_t L(Rc);
    const u32 Ru = u32(R);
    const double* xj = x + j0 + L.j;
    double* vj = rows + j0 + L.j;
    const u32 ncode = NBK < WNB ? u32(NBK) : u32(WNB);
    const u32 wid = blockIdx.x * WPB + wid_in_cta(), nw = gridDim.x * WPB;
    uint4 tb = wid < wt.n ? wt.t[wid] : make_uint4(0, 0, 0, 0);
    for (u32 tile = wid; tile < wt.n; tile += nw) {
        const u32 s0 = tb.x, ns = tb.y - tb.x, c0 = tb.z, nc = tb.w - tb.z;
        stage_cells(S, W, s0, tb.y, c0, tb.w, st, ncode, !trivial);
        if (L.on) {
            double v[KS];
#pragma unroll
            for (int k = 0; k < KS; k++) {
                const u32 sl = L.g + u32(k * G);
                v[k] = sl < ns ? b1[size_t(s0 + sl) * Ru + j0 + L.j] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < KS; k++) {
                const u32 sl = L.g + u32(k * G);
                if (sl < ns) bs[sl * Rc + L.j] = v[k];
            }
        }
        if (tile + nw < wt.n) tb = wt.t[tile + nw];
        __syncwarp();
        stage_maps(nc, st, !trivial);
        __syncwarp();
        if (L.on) {
            SegRun<double> sr;
            const u32* cg = st.code + L.g;
#pragma unroll
            for (int k0 = 0; k0 < L_t::KN; k0 += L_t::CH) {
                double v[L_t::CH];
#pragma unroll
                for (int k = 0; k < L_t::CH; k++) {
                    const u32 i = L.g + u32((k0 + k) * G);
                    v[k] = i < nc ? gather_cell<NBK>(S, cg + (k0 + k) * G, xj, Ru, c0 + i) : 0.0;
                }
#pragma unroll
                for (int k = 0; k < L_t::CH; k++) {
                    const u32 i = L.g + u32((k0 + k) * G);
                    if (i < nc) {
                        u[i * Rc + L.j] = v[k];
                        sr.add(st.segl[i], st.cw[i] * v[k], ps, L.lane);
                    }
                }
            }
            sr.finish(ns, ps, L.lane);
        }
        __syncwarp();
        if (L.on)
            for (u32 sl = L.g; sl < ns; sl += G) {
                const double al = (bs[sl * Rc + L.j] - seg_total<RCP>(ps, sl, L.j)) * st.n1i[sl];
                if (alpha) alpha[size_t(s0 + sl) * Ru + j0 + L.j] = al;
                ps[sl * 32 + L.j] = al;
            }
        __syncwarp();
        if (L.on) {
            const u32 r0 = trivial ? c0 : st.row0[0];
            const u32 nr = trivial ? nc : st.row0[nc] - r0;
#pragma unroll
            for (int k0 = 0; k0 < L_t::KN; k0 += L_t::CH) {
                double v[L_t::CH];
#pragma unroll
                for (int k = 0; k < L_t::CH; k++) {
                    const u32 r = L.g + u32((k0 + k) * G);
                    v[k] = r < nr ? __ldcs(vj + size_t(r0 + r) * Ru) : 0.0;
                }
#pragma unroll
                for (int k = 0; k < L_t::CH; k++) {
                    const u32 r = L.g + u32((k0 + k) * G);
                    if (r < nr) {
                        const u32 i = trivial ? r : st.rcell[r];
                        __stcs(vj + size_t(r0 + r) * Ru, v[k] - (ps[st.segl[i] * 32 + L.j] + u[i * Rc + L.j]));
                    }
                }
            }
        }
        __syncwarp();
    }
}

// Residualization of the short segments when every cell holds one row and the rows have at most
// FR_MAXR columns (operator.rs:1107-1179), per warp tile of whole segments (at most WT cells, WSEG
// segments). The tile's rows are nc x R contiguous elements, dealt to the lanes in order (element e
// to lane e mod 32), so the row copies and stores and the gathers of x run along the rows on all
// 32 lanes. Software pipelined: while a warp works on one tile, cp.async copies bring the next
// tile's rows, block coordinates, cell weights, segment offsets and 1/n1 into the other of two
// shared buffers. For a tile:
//  1. u(c, j) = sum_b x[coord_b(c), j] (blocks in order), every element's gathers in flight
//     together, into the warp's shared memory U[e];
//  2. alpha(s, j) = (b1(s, j) - sum_c W_c u(c, j)) / n1_s, one (segment, column) pair per lane,
//     the segment's cells in order, into A;
//  3. every element is written back as v - (alpha(s(c), j) + u(c, j)).
constexpr int FR_MAXR = 16;  // widest rows k_fresid takes
constexpr int FR_WPB = 4;    // warps per CTA of k_fresid

// Per-warp shared memory of k_fresid for R columns: two buffers of [rows, coordinates, cell
// weights, segment offsets, 1/n1], then U, A and the cells' local segments.
__host__ __device__ constexpr size_t fr_buf_bytes(int R) {
    return al16(size_t(WT) * R * 8) + al16(size_t(WNB) * WT * 4) + al16(WT * 8) + al16((WSEG + 1) * 4) +
           al16(WSEG * 8);
}
__host__ __device__ constexpr size_t fresid_bytes(int R) {
    return 2 * fr_buf_bytes(R) + al16(size_t(WT) * R * 8) + al16(size_t(WSEG) * R * 8) + al16(WT * 4);
}

struct FrBuf {
    double* v;    // the tile's rows (nc x R)
    u32* code;    // block coordinates (WNB x WT)
    double* cw;   // cell weights (weighted cells only)
    u32* soff;    // seg_off[s0 .. s1]
    double* n1i;  // 1/n1 of the tile's segments
};
__device__ __forceinline__ FrBuf fr_buf_at(unsigned char* p, int R) {
    FrBuf b;
    b.v = reinterpret_cast<double*>(p);
    p += al16(size_t(WT) * R * 8);
    b.code = reinterpret_cast<u32*>(p);
    p += al16(size_t(WNB) * WT * 4);
    b.cw = reinterpret_cast<double*>(p);
    p += al16(WT * 8);
    b.soff = reinterpret_cast<u32*>(p);
    p += al16((WSEG + 1) * 4);
    b.n1i = reinterpret_cast<double*>(p);
    return b;
}

// Issues the copies of tile tb into buffer b (the caller commits the group).
template <int NC>
__device__ __forceinline__ void fr_prefetch(const DevStruct& S, const DevWeights& W, const double* rows, u32 R,
                                            const uint4& tb, const FrBuf& b) {
    const u32 lane = wlane(), s0 = tb.x, ns = tb.y - tb.x, c0 = tb.z, nc = tb.w - tb.z;
    const double* src = rows + size_t(c0) * R;
    for (u32 e = lane; e < nc * R; e += 32) cp_async8(b.v + e, src + e);
    if (lane < nc) {
#pragma unroll
        for (int k = 0; k < NC; k++) cp_async4(b.code + k * WT + lane, S.coord + size_t(k) * S.M + c0 + lane);
        if (W.cell_w) cp_async8(b.cw + lane, W.cell_w + c0 + lane);
    }
    if (lane <= ns) cp_async4(b.soff + lane, S.seg_off + s0 + lane);
    if (lane < ns) cp_async8(b.n1i + lane, W.n1inv + s0 + lane);
}

// The (row, column) of element e = lane + 32 t of an R-column tile, advanced by 32 per step.
struct ElemPos {
    u32 r, c;
    __device__ __forceinline__ void step(u32 q32, u32 r32, u32 R) {
        r += q32;
        c += r32;
        if (c >= R) {
            c -= R;
            r++;
        }
    }
};

// NE: elements per lane of a tile at most (WT R / 32 = R, rounded up to a multiple of 4).
template <int NBK, int NE>
__global__ void __launch_bounds__(FR_WPB * 32, 5) k_fresid(DevStruct S, DevWeights W, WarpTiles wt,
                                                           double* __restrict__ rows, int R,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ b1, double* __restrict__ alpha) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NC = NBK < WNB ? NBK : WNB;  // blocks whose coordinates are staged
    const u32 uR = u32(R);
    unsigned char* mine = smem_raw + size_t(threadIdx.x >> 5) * fresid_bytes(R);
    const u32 bbytes = u32(fr_buf_bytes(R));
    double* U = reinterpret_cast<double*>(mine + 2 * bbytes);
    double* A = U + size_t(WT) * R;
    u32* segl = reinterpret_cast<u32*>(reinterpret_cast<unsigned char*>(A) + al16(size_t(WSEG) * R * 8));
    const u32 lane = wlane();
    const u32 q32 = 32u / uR, r32 = 32u % uR;
    const ElemPos first{lane / uR, lane % uR};
    const size_t Ru = size_t(R);
    const u32 wid = blockIdx.x * FR_WPB + (threadIdx.x >> 5), nw = gridDim.x * FR_WPB;
    uint4 tb = wid < wt.n ? wt.t[wid] : make_uint4(0, 0, 0, 0);            // this tile
    uint4 tn = wid + nw < wt.n ? wt.t[wid + nw] : make_uint4(0, 0, 0, 0);  // the next
    if (wid < wt.n) fr_prefetch<NC>(S, W, rows, uR, tb, fr_buf_at(mine, R));
    cp_async_commit();
    u32 it = 0;
    for (u32 tile = wid; tile < wt.n; tile += nw, it++) {
        const FrBuf cur = fr_buf_at(mine + (it & 1) * bbytes, R);
        if (tile + nw < wt.n) fr_prefetch<NC>(S, W, rows, uR, tn, fr_buf_at(mine + ((it + 1) & 1) * bbytes, R));
        cp_async_commit();
        const uint4 tc = tb;
        tb = tn;
        if (tile + 2 * nw < wt.n) tn = wt.t[tile + 2 * nw];
        cp_async_wait_prior();  // this tile's copies
        __syncwarp();
        const u32 s0 = tc.x, ns = tc.y - tc.x, c0 = tc.z, nc = tc.w - tc.z;
        const u32 E = nc * uR;
        if (lane < nc) {
            u32 sl = 0;
            while (cur.soff[sl + 1] - c0 <= lane) sl++;
            segl[lane] = sl;
        }
        // 1. u of every element, all the lane's gathers in flight together
        {
            double g[NE];
            ElemPos p = first;
#pragma unroll
            for (int k = 0; k < NE; k++) {
                g[k] = 0.0;
                if (p.r < nc) {
#pragma unroll
                    for (int b = 0; b < NC; b++) g[k] += __ldg(x + size_t(cur.code[b * WT + p.r]) * Ru + p.c);
                    if constexpr (NBK == WNB)
                        for (u32 b = WNB; b < S.nb; b++)
                            g[k] += __ldg(x + size_t(__ldg(S.coord + size_t(b) * S.M + c0 + p.r)) * Ru + p.c);
                }
                p.step(q32, r32, uR);
            }
#pragma unroll
            for (int k = 0; k < NE; k++) {
                const u32 e = lane + 32u * u32(k);
                if (e < E) U[e] = g[k];
            }
        }
        __syncwarp();
        // 2. alpha of every (segment, column) pair
        for (u32 pr = lane; pr < ns * uR; pr += 32) {
            const u32 sl = pr / uR, c = pr % uR;
            const u32 i0 = cur.soff[sl] - c0, i1 = cur.soff[sl + 1] - c0;
            double a = 0.0;
            for (u32 i = i0; i < i1; i++) a += (W.cell_w ? cur.cw[i] : 1.0) * U[i * uR + c];
            const double al = (b1[size_t(s0 + sl) * Ru + c] - a) * cur.n1i[sl];
            A[sl * uR + c] = al;
            if (alpha) alpha[size_t(s0 + sl) * Ru + c] = al;
        }
        __syncwarp();
        // 3. the rows
        {
            double* dst = rows + size_t(c0) * Ru;
            ElemPos p = first;
            for (u32 e = lane; e < E; e += 32) {
                __stcs(dst + e, cur.v[e] - (A[segl[p.r] * uR + p.c] + U[e]));
                p.step(q32, r32, uR);
            }
        }
        __syncwarp();
    }
    cp_async_wait_all();
}

}  // namespace fereg
