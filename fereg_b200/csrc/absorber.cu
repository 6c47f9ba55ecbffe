// GpuAbsorber: structure on the host, the solve on the B200.
//
// residualize (solve.rs:1141-1311) runs the rhs pass over the rows (k_seg_rhs + k_pull_rhs),
// lockstep PCG on the reduced system (k_seg_apply + k_pull_apply per matvec; Jacobi / grounded
// dense small-block preconditioner; per-column scalars on the device), and the in-place
// residualization pass (k_residualize). With Precision::F32_REFINED the PCG iterations run in
// FP32 on the correction of an FP64 iterate whose true residual is recomputed in FP64 between
// rounds (iterative refinement); the stopping rule is evaluated on the FP64 quantities.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <type_traits>

#include "absorber.h"
#include "amg.cuh"
#include "amg.h"
#include "dstruct.h"
#include "pcg.cuh"
#include "pcg_driver.h"
#include "weights.cuh"

namespace fereg {

namespace {
constexpr int THREADS = TB;
constexpr int GRID_T = 148 * 6;  // tile kernels: up to 6 resident CTAs per SM
constexpr int GRID_V = 148 * 2;  // vector kernels with per-CTA partials
constexpr int GRID_S = 148 * 4;  // warp-tile kernels (CTAs of WPB warps)
constexpr size_t SMALL_STAGE_MAX = 16 * 1024;  // shared memory for the staged small rows of a chunk
constexpr u32 VSEG_MAX = 256;  // longest segment (cells) a lane group walks in the operator's segment pass
constexpr double REDUNDANT = 1e-12;  // operator.rs:21
// Largest small super-block factored densely on the device. Beyond it the small coordinates keep
// Jacobi, as the reference does when the dense factor costs more than a few PCG iterations
// (solve.rs:541-548 defer_small); the converged answer is the same within the tolerance.
constexpr size_t DENSE_SMALL_MAX = 1024;
// Refinement: an FP32 inner solve stops once its preconditioned residual fell by this factor
// (squared), well above FP32 rounding; the FP64 true residual then restarts it.
constexpr double REFINE_DROP = 1e-9;
constexpr int REFINE_ROUNDS = 30;

void dense_ldlt_inverse(double* a, double* d, int k, double* x, cudaStream_t st, u64& launches);
template <class K>
void allow_smem(K kernel, size_t bytes);

inline int grid_for(size_t total) {
    size_t b = (total + THREADS - 1) / THREADS;
    return int(std::max<size_t>(1, std::min<size_t>(b, size_t(GRID_T) * 4)));
}

struct DevTiles {
    DBuf<u32> k0, k1, e0, e1, fix_k, fix_p0, fix_np;
    DBuf<int> part, fixidx;
    u32 n = 0, nfix = 0, nparts = 0;
    void upload(const TileList& t, cudaStream_t s) {
        k0.upload(t.k0, s);
        k1.upload(t.k1, s);
        e0.upload(t.e0, s);
        e1.upload(t.e1, s);
        part.upload(t.part, s);
        fixidx.upload(t.fixidx, s);
        fix_k.upload(t.fix_k, s);
        fix_p0.upload(t.fix_p0, s);
        fix_np.upload(t.fix_np, s);
        n = u32(t.k0.size());
        nfix = u32(t.fix_k.size());
        nparts = t.nparts;
    }
    TileSet set() const { return TileSet{n, k0.p, k1.p, e0.p, e1.p, part.p, fixidx.p, nfix, fix_k.p, fix_p0.p, fix_np.p, nparts}; }
};

// Warp tiles packed as (k0, k1, e0, e1) in one 16-byte load.
struct DevWarpTiles {
    DBuf<uint4> t;
    u32 n = 0;
    void upload(const WarpTileList& l, cudaStream_t s) {
        std::vector<uint4> h(l.k0.size());
        for (size_t i = 0; i < h.size(); i++) h[i] = make_uint4(l.k0[i], l.k1[i], l.e0[i], l.e1[i]);
        t.upload(h, s);
        n = u32(h.size());
    }
    WarpTiles set() const { return WarpTiles{n, t.p}; }
};

// Dynamic shared memory of the warp-tile kernels for a chunk of Rc columns (per-warp parts, then
// the lane-private small-coordinate slots and column partials).
inline size_t grhs_smem(u32 ms_acc) { return WPB * (size_t(ms_acc) * 64 * 8 + 4 * 32 * 8); }
inline size_t wresid_smem(int Rc) { return WPB * wresid_bytes(Rc); }

inline size_t wpull_smem() { return WPB * pull_bytes(); }

// Calls f(RCP, NBK) as integral constants: RCP the padded width of an Rc-column chunk, NBK the
// block-count key of nb blocks (from MIN_NBK: apply and list kernels never run without blocks).
template <int RCP, int MIN_NBK, class F>
void with_nbk(u32 nb, F&& f) {
    using std::integral_constant;
    switch (std::max(nbk_of(nb), MIN_NBK)) {
        case 0: f(integral_constant<int, RCP>{}, integral_constant<int, 0 < MIN_NBK ? MIN_NBK : 0>{}); break;
        case 1: f(integral_constant<int, RCP>{}, integral_constant<int, 1>{}); break;
        case 2: f(integral_constant<int, RCP>{}, integral_constant<int, 2>{}); break;
        case 3: f(integral_constant<int, RCP>{}, integral_constant<int, 3>{}); break;
        default: f(integral_constant<int, RCP>{}, integral_constant<int, WNB>{}); break;
    }
}
// Lane groups of L lanes (lanes_of(Rc) by default: two columns per lane).
template <int MIN_NBK = 0, class F>
void with_lanes(int Rc, u32 nb, F&& f, int L = 0) {
    switch (L > 0 ? L : lanes_of(Rc)) {
        case 1: with_nbk<1, MIN_NBK>(nb, f); break;
        case 2: with_nbk<2, MIN_NBK>(nb, f); break;
        case 4: with_nbk<4, MIN_NBK>(nb, f); break;
        case 8: with_nbk<8, MIN_NBK>(nb, f); break;
        default: with_nbk<16, MIN_NBK>(nb, f); break;
    }
}
// Lane groups of the padded-vector passes: vlanes_of(Rc) lanes of 4 columns each (1 to 32).
template <class F>
void with_vlanes(int Rc, u32 nb, F&& f) {
    switch (vlanes_of(Rc)) {
        case 1: with_nbk<1, 1>(nb, f); break;
        case 2: with_nbk<2, 1>(nb, f); break;
        case 4: with_nbk<4, 1>(nb, f); break;
        case 8: with_nbk<8, 1>(nb, f); break;
        case 16: with_nbk<16, 1>(nb, f); break;
        default: with_nbk<32, 1>(nb, f); break;
    }
}
// Calls f(NSA) with the small blocks the segment passes sum (0 to WNB) as an integral constant.
template <class F>
void with_nsa(u32 ns, F&& f) {
    using std::integral_constant;
    switch (ns) {
        case 0: f(integral_constant<int, 0>{}); break;
        case 1: f(integral_constant<int, 1>{}); break;
        case 2: f(integral_constant<int, 2>{}); break;
        case 3: f(integral_constant<int, 3>{}); break;
        default: f(integral_constant<int, WNB>{}); break;
    }
}
template <int MIN_NBK = 0, class F>
void with_rcp(int Rc, u32 nb, F&& f) {
    switch (rcp_of(Rc)) {
        case 1: with_nbk<1, MIN_NBK>(nb, f); break;
        case 2: with_nbk<2, MIN_NBK>(nb, f); break;
        case 4: with_nbk<4, MIN_NBK>(nb, f); break;
        case 8: with_nbk<8, MIN_NBK>(nb, f); break;
        case 16: with_nbk<16, MIN_NBK>(nb, f); break;
        default: with_nbk<32, MIN_NBK>(nb, f); break;
    }
}
}  // namespace

// Device form of an escalated block's hierarchy (amg.h) and its V-cycle work vectors.
struct DevAmgBlock {
    u32 off = 0, g = 0;  // the block's coordinates [off, off + g)
    std::vector<DevAmgLevel> lv;
    std::vector<DBuf<u32>> iu;     // CSR index arrays of every level
    std::vector<DBuf<double>> dv;  // CSR values and dinv of every level
    DBuf<double> minv;             // generalized inverse of the coarsest level
    // per level l: right-hand side (l >= 1), output (l >= 1), and the residual / prolongated value
    std::vector<DBuf<double>> wd;
    std::vector<DBuf<float>> wf;
};

template <class T>
std::vector<DBuf<T>>& amg_work(DevAmgBlock& a);
template <>
std::vector<DBuf<double>>& amg_work<double>(DevAmgBlock& a) {
    return a.wd;
}
template <>
std::vector<DBuf<float>>& amg_work<float>(DevAmgBlock& a) {
    return a.wf;
}

struct Scratch {
    // escalated large blocks
    std::vector<DevAmgBlock> amg;
    u64 escalations = 0;
    // structure
    DBuf<u32> seg_off, coord, cell_row, pl_off, pl_cell, pl_seg, pl_other;
    DevTiles seg_tiles, pull_tiles;      // CTA tiles of the long lists
    DevWarpTiles wseg, wpull;            // warp tiles of the short lists
    DBuf<u32> wseg_segs;                 // the segments of the warp tiles, in order
    DBuf<u32> aseg_segs;                 // the operator's lane-group segments (at most VSEG_MAX cells)
    DevTiles aseg_tiles;                 // the operator's CTA tiles (longer segments)
    u32 ms_acc = 0, ns_acc = 0;  // small coordinates / blocks summed in the segment passes
    // weights
    DBuf<double> w_rows, cell_w, n1inv, nr, inv_diag, minv;
    DBuf<double> n1, diag, wpart;  // device weight refresh
    DBuf<u32> pi;                  // the row order (kept observation of each row)
    DBuf<u32> cw_e0, cw_e1, cw_list_off;  // chunks of the coordinate lists (weights.cuh)
    DBuf<double> cw_chunks;
    u32 cw_nchunks = 0;
    // work items of the row-wise small-block assembly (k_small_rows): row, entry range; first
    // item of every row
    DBuf<u32> sr_k, sr_a, sr_b, sr_first;
    u32 sr_n = 0;
    // dense rows of S on the small coordinates (srow, m x ms_acc, transposed) and the work items
    // of their assembly: entry range of every run of a coordinate list, first item per coordinate
    DBuf<double> srow;
    DBuf<u32> si_a, si_b, si_first;
    u32 si_n = 0;
    bool srow_on = false;
    DBuf<uint8_t> red;
    DBuf<int> wflag;
    // solve (FP64)
    DBuf<double> rows, rhs, b1, coefs, r, z, p, q, t, part, cta, cta2, colsum, along, small;
    DBuf<double> rhsv, xv;  // the padded right-hand side and iterate of the PCG
    // inner FP32 buffers of the refined solve
    DBuf<float> fx, fb, fr, fz, fp, fq, ft, fpart, frhs, fx0, fsmall;
    DBuf<double> cg_rho, cg_rho_new, cg_pq, cg_gamma, cg_beta, cg_xb, cg_ss1, cg_floor, cg_ring, cg_xconst, cg_pfloor;
    DBuf<int> cg_active, cg_nactive;
    DBuf<double> cg_ss0;
    int* h_nactive = nullptr;  // pinned: the loop control words (CgLoop::ctl) read back
    double* h_ss0 = nullptr;   // pinned: ss0 read back (h_ss0_n values)
    size_t h_ss0_n = 0;
    // PCG loop state on the device (pcg.cuh) and the captured iteration graphs, each keyed by
    // every address its kernels read or write
    DBuf<int> lp_ctl, lp_act;
    DBuf<double> lp_tol;
    DBuf<unsigned> lp_ticket;
    DBuf<double> lp_rho_from, lp_rho_at;
    struct PcgGraph {
        std::vector<u64> key;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        u64 body_launches = 0;  // kernels of one body
    };
    std::vector<PcgGraph> graphs;
    // grids of the S*P passes chosen by the autotuner, per (padded width, element size)
    struct ApplyGrids {
        int seg = 148 * 4, pull = 148 * 4;
    };
    std::map<std::pair<int, int>, ApplyGrids> grids;
    double tune_us = 0;  // host time of the tuning runs
    u64 graph_launches = 0, graph_captures = 0;
    u64 fp64_finishes = 0;  // FP32-refined solves finished in FP64
    double graph_build_us = 0;  // host time of the captures and instantiations
    void drop_graphs() {
        for (auto& q : graphs) {
            if (q.exec) cudaGraphExecDestroy(q.exec);
            if (q.g) cudaGraphDestroy(q.g);
        }
        graphs.clear();
    }
    // phase timing
    bool prof = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_slot;
    double ms[GpuAbsorber::P_NSLOTS] = {};
    u64 cnt[GpuAbsorber::P_NSLOTS] = {};
    std::vector<cudaEvent_t> pool_;
    u64 launches = 0;

    DevStruct ds(const HostStructure& hs) const {
        DevStruct s{};
        s.M = u32(hs.ncells);
        s.g1 = hs.g1;
        s.nb = u32(hs.nb());
        s.m = u32(hs.m);
        s.ms = u32(hs.m_small);
        s.ms_acc = ms_acc;
        s.ns_acc = ns_acc;
        s.seg_off = seg_off.p;
        s.coord = coord.p;
        s.cell_row = cell_row.p;
        s.pl_off = pl_off.p;
        s.pl_cell = pl_cell.p;
        s.pl_seg = pl_seg.p;
        s.pl_other = pl_other.p;
        s.seg = seg_tiles.set();
        s.pull = pull_tiles.set();
        return s;
    }
    DevWeights dw() const { return DevWeights{w_rows.p, cell_w.p, n1inv.p, nr.p}; }
    CgState cg() {
        return CgState{cg_rho.p, cg_rho_new.p, cg_pq.p,   cg_gamma.p,  cg_beta.p,   cg_xb.p,     cg_ss1.p,
                       cg_floor.p, cg_ring.p, cg_xconst.p, cg_pfloor.p, cg_active.p, cg_nactive.p};
    }
    cudaEvent_t get_event() {
        if (!pool_.empty()) {
            cudaEvent_t e = pool_.back();
            pool_.pop_back();
            return e;
        }
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        return e;
    }
    int begin(int slot, cudaStream_t st) {
        if (!prof) return -1;
        cudaEvent_t a = get_event();
        CK(cudaEventRecord(a, st));
        ev.push_back(a);
        ev.push_back(nullptr);
        ev_slot.push_back(slot);
        return int(ev.size()) - 2;
    }
    void end(int h, cudaStream_t st) {
        if (h < 0) return;
        cudaEvent_t b = get_event();
        CK(cudaEventRecord(b, st));
        ev[size_t(h) + 1] = b;
    }
    void collect() {
        for (size_t i = 0; i + 1 < ev.size(); i += 2) {
            float t = 0;
            if (ev[i + 1]) {
                CK(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
                ms[ev_slot[i / 2]] += t;
                cnt[ev_slot[i / 2]]++;
                pool_.push_back(ev[i + 1]);
            }
            pool_.push_back(ev[i]);
        }
        ev.clear();
        ev_slot.clear();
    }
    ~Scratch() {
        drop_graphs();
        if (h_nactive) cudaFreeHost(h_nactive);
        if (h_ss0) cudaFreeHost(h_ss0);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
        for (auto e : pool_) cudaEventDestroy(e);
    }
};

GpuAbsorber::GpuAbsorber(const std::vector<const u32*>& codes, const std::vector<u32>& g, const double* w, size_t n,
                         const Ctx& ctx, const std::vector<const u32*>* dev_codes)
    : g_(g), ctx_(ctx) {
    check_codes_host(codes, g, n);
    if (w) check_weights_host(w, n);
    hs_ = plan_structure(codes, g, n, SMALL_LIMIT);
    norm_fe1_ = fe1_index(g);
    ctx_.check();
    keep_pool_mapped();
    if (ctx_.priority_level < 0) {
        CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    } else {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        const int prio = std::min(std::max(greatest, least - 1), greatest + ctx_.priority_level);
        CK(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, prio));
    }
    AllocScope alloc_scope(stream_);
    d_ = std::make_unique<Scratch>();
    CK(cudaHostAlloc(&d_->h_nactive, 8 * sizeof(int), cudaHostAllocDefault));
    // the cell structure and coordinate lists, built on the device from device codes
    std::vector<u32> pl_off, pl_seg;
    {
        std::vector<DBuf<u32>> up;
        std::vector<const u32*> dptr;
        if (dev_codes) {
            dptr = *dev_codes;
        } else {
            up.resize(codes.size());
            for (size_t q = 0; q < codes.size(); q++) {
                up[q].upload(codes[q], n, stream_);
                dptr.push_back(up[q].p);
            }
        }
        DeviceStructure ds;
        build_structure_device(dptr, g, hs_, ds, pl_off, pl_seg, stream_);
        d_->pi = std::move(ds.pi);
        d_->seg_off = std::move(ds.seg_off);
        d_->coord = std::move(ds.coord);
        d_->cell_row = std::move(ds.cell_row);
        d_->pl_off = std::move(ds.pl_off);
        d_->pl_cell = std::move(ds.pl_cell);
        d_->pl_seg = std::move(ds.pl_seg);
        d_->pl_other = std::move(ds.pl_other);
        CK(cudaStreamSynchronize(stream_));  // the uploaded codes die here
    }
    {
        // segments weigh max(cells, rows): short ones go to warp tiles, the others to CTA tiles
        std::vector<u32> wgt(hs_.g1);
        for (u32 s = 0; s < hs_.g1; s++) {
            const u32 c0 = hs_.seg_off[s], c1 = hs_.seg_off[s + 1];
            const u32 rows = hs_.trivial() ? c1 - c0 : hs_.cell_row[c1] - hs_.cell_row[c0];
            wgt[s] = std::max(c1 - c0, rows);
        }
        WarpTileList wt;
        TileList ct;
        split_tiles(hs_.seg_off, &wgt, 0, hs_.g1, WT, WT, WSEG, TILE, wt, ct);
        d_->wseg.upload(wt, stream_);
        std::vector<u32> segs;  // the short segments in order (one per lane group in k_vseg_apply)
        for (size_t i = 0; i < wt.k0.size(); i++)
            for (u32 s = wt.k0[i]; s < wt.k1[i]; s++) segs.push_back(s);
        d_->wseg_segs.upload(segs, stream_);
        d_->seg_tiles.upload(ct, stream_);
        // the operator's segment pass: lane groups walk every segment of at most VSEG_MAX cells (in
        // order), CTA tiles take the longer ones
        std::vector<u32> asegs;
        for (u32 s = 0; s < hs_.g1; s++)
            if (hs_.seg_off[s + 1] - hs_.seg_off[s] <= VSEG_MAX) asegs.push_back(s);
        d_->aseg_segs.upload(asegs, stream_);
        d_->aseg_tiles.upload(build_tiles(hs_.seg_off, 0, hs_.g1, TILE, VSEG_MAX), stream_);
        CK(cudaStreamSynchronize(stream_));
    }
    {
        u32 ns = 0;
        for (auto& b : hs_.blocks) ns += b.small;
        if (hs_.m_small > 0 && hs_.m_small <= size_t(SACC_MAX) && ns <= u32(SACC_BLOCKS)) {
            d_->ms_acc = u32(hs_.m_small);
            d_->ns_acc = ns;
        }
    }
    if (hs_.m > 0) {
        {  // chunks of the lists for the device weight refresh (weights.cuh)
            std::vector<u32> e0, e1, loff(hs_.m + 1, 0);
            for (size_t k = 0; k < hs_.m; k++) {
                for (u32 a = pl_off[k]; a < pl_off[k + 1]; a += CW_CHUNK) {
                    e0.push_back(a);
                    e1.push_back(std::min<u32>(pl_off[k + 1], a + CW_CHUNK));
                }
                loff[k + 1] = u32(e0.size());
            }
            d_->cw_nchunks = u32(e0.size());
            d_->cw_e0.upload(e0, stream_);
            d_->cw_e1.upload(e1, stream_);
            d_->cw_list_off.upload(loff, stream_);
        }
        if (hs_.m_small > 0 && hs_.m_small <= DENSE_SMALL_MAX) {
            // runs of each small coordinate's entries, at least `run` long, never splitting a segment
            const u32 es = pl_off[hs_.m_small];
            const u32 run = std::max<u32>(256, es / 4096);
            std::vector<u32> ik, ia, ib, first(hs_.m_small + 1, 0);
            for (u32 k = 0; k < u32(hs_.m_small); k++) {
                first[k] = u32(ik.size());
                for (u32 a = pl_off[k]; a < pl_off[k + 1];) {
                    u32 b = std::min(pl_off[k + 1], a + run);
                    while (b < pl_off[k + 1] && pl_seg[b] == pl_seg[b - 1]) b++;
                    ik.push_back(k);
                    ia.push_back(a);
                    ib.push_back(b);
                    a = b;
                }
            }
            first[hs_.m_small] = u32(ik.size());
            d_->sr_k.upload(ik, stream_);
            d_->sr_a.upload(ia, stream_);
            d_->sr_b.upload(ib, stream_);
            d_->sr_first.upload(first, stream_);
            d_->sr_n = u32(ik.size());
        }
        if (d_->ms_acc > 0) {
            // work items of the dense small rows: runs of at least 256 entries of every list, never
            // splitting a segment's run
            std::vector<u32> ia, ib, first(hs_.m + 1, 0);
            for (u32 f = 0; f < u32(hs_.m); f++) {
                first[f] = u32(ia.size());
                for (u32 a = pl_off[f]; a < pl_off[f + 1];) {
                    u32 b = std::min(pl_off[f + 1], a + 256);
                    while (b < pl_off[f + 1] && pl_seg[b] == pl_seg[b - 1]) b++;
                    ia.push_back(a);
                    ib.push_back(b);
                    a = b;
                }
            }
            first[hs_.m] = u32(ia.size());
            d_->si_a.upload(ia, stream_);
            d_->si_b.upload(ib, stream_);
            d_->si_first.upload(first, stream_);
            d_->si_n = u32(ia.size());
            d_->srow_on = true;
        }
        WarpTileList wt;
        TileList ct;
        split_tiles(pl_off, nullptr, d_->ms_acc, u32(hs_.m), PULL_WARP_MAX, PULL_WARP_MAX, WLIST, PULL_SLICE, wt, ct);
        d_->wpull.upload(wt, stream_);
        d_->pull_tiles.upload(ct, stream_);
        CK(cudaStreamSynchronize(stream_));  // host tables die here
    }
    // the weight state, on the device: kept-order weights gathered into row order
    if (w) {
        DBuf<double> wk, wr;
        wk.upload(w, n, stream_);
        wr.alloc(n);
        k_gather_rows_f64<<<grid_for(n), THREADS, 0, stream_>>>(wk.p, d_->pi.p, n, wr.p);
        d_->launches++;
        set_weights_device(wr.p);
        CK(cudaStreamSynchronize(stream_));
    } else {
        unit_weights_device();
    }
}

// The weight state of unit row weights on the device: cell weights are the cells' row counts
// (none when every cell holds one row), n1 the segments' row counts.
void GpuAbsorber::unit_weights_device() {
    AllocScope alloc_scope(stream_);
    Scratch& d = *d_;
    const size_t M = hs_.ncells, g1 = hs_.g1;
    d.w_rows.release();
    if (hs_.trivial()) {
        d.cell_w.release();
    } else {
        d.cell_w.alloc(M);
        k_cell_counts<<<grid_for(M), THREADS, 0, stream_>>>(d.cell_row.p, u32(M), d.cell_w.p);
        d.launches++;
    }
    d.n1.alloc(g1);
    d.n1inv.alloc(g1);
    k_seg_weights<<<grid_for(g1), THREADS, 0, stream_>>>(d.cell_w.p, d.seg_off.p, u32(g1), d.n1.p, d.n1inv.p);
    d.launches++;
    CK(cudaGetLastError());
    sw_ = double(hs_.n);
    weighted_ = false;
    host_stale_ = true;
    coord_stale_ = hs_.m > 0;
    refresh_coord();
    build_srow();
    pre_fresh_ = false;
    small_stale_ = false;
    amg_stale_ = true;
    CK(cudaStreamSynchronize(stream_));
}

// The host copy of the cells' block coordinates, for the host readers of the structure (the
// multigrid setup, fit_rows), fetched from the device the first time one needs it.
void GpuAbsorber::ensure_host_coord() const {
    const size_t len = hs_.nb() * hs_.ncells;
    if (len == 0 || hs_.coord.size() == len) return;
    hs_.coord.resize(len);
    CK(cudaMemcpyAsync(hs_.coord.data(), d_->coord.p, len * sizeof(u32), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

// Escalation: the reference escalates once, when the probe finds slow contraction (cg.rs:24-37,
// solve.rs:838-876). Every Jacobi-preconditioned block above 2 AMG_COARSE levels (the large
// blocks, and the blocks of a small super-block without its dense factor) gets a hierarchy.
// New weights leave the hierarchies in place as a stale but still symmetric positive
// preconditioner (the reference keeps stale factors across IRLS weights, solve.rs:554
// stale_refresh_pays); they are rebuilt only when a later probe finds slow contraction again.
// A stale hierarchy is rebuilt only on clearly slow contraction (a rebuild costs a host
// assembly; a stale V-cycle still contracts far faster than Jacobi).
constexpr double STALE_AMG_RATIO = 0.85;

bool GpuAbsorber::escalate(double rho_hat) {
    AllocScope alloc_scope(stream_);
    const auto t0 = std::chrono::steady_clock::now();
    struct Clock {  // host wall time of the escalation step into its phase slot
        Scratch& d;
        std::chrono::steady_clock::time_point t0;
        ~Clock() {
            if (!d.prof) return;
            d.ms[GpuAbsorber::P_ESCALATE] +=
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            d.cnt[GpuAbsorber::P_ESCALATE]++;
        }
    } clock{*d_, t0};
    // one step per probe, cheapest first: a stale dense small factor, then stale hierarchies,
    // then new hierarchies
    if (small_stale_) {
        refresh_coord();
        refresh_small();
        return true;
    }
    if (!d_->amg.empty() && amg_stale_) {
        if (rho_hat <= STALE_AMG_RATIO) return false;
        build_amg();
        amg_stale_ = false;
        d_->escalations++;
        return true;
    }
    if (!d_->amg.empty()) return false;  // the hierarchies are current: nothing stronger
    if (d_->amg.empty() && amg_wanted_) return false;    // aggregation stalled before: keep Jacobi
    bool any = false;
    for (auto& b : hs_.blocks) any |= (!b.small || !small_ok_) && b.g > 2 * AMG_COARSE;
    if (!any) return false;
    amg_wanted_ = true;
    build_amg();
    amg_stale_ = false;
    d_->escalations++;
    return !d_->amg.empty();
}

void GpuAbsorber::refresh_small() {
    pre_fresh_ = false;
    ensure_precond();
    small_stale_ = false;
}

constexpr u32 AMG_DENSE_MAX = 2048;  // the largest coarsest level inverted densely

void GpuAbsorber::build_amg() {
    AllocScope alloc_scope(stream_);
    sync_host_weights();
    ensure_host_coord();
    d_->amg.clear();
    for (size_t b = 0; b < hs_.blocks.size(); b++) {
        const Block& B = hs_.blocks[b];
        // large blocks, and the blocks of a small super-block too big for its dense factor
        if ((B.small && small_ok_) || B.g <= 2 * AMG_COARSE) continue;
        AmgHierarchy H =
            amg_build(hs_, b, cell_w_.empty() ? nullptr : cell_w_.data(), n1_.data(), diag_.data(), red_.data());
        const u32 nL = H.levels.back().n;
        if (nL > AMG_DENSE_MAX) continue;  // aggregation stalled: the block keeps Jacobi
        DevAmgBlock A;
        A.off = B.off;
        A.g = B.g;
        const size_t L = H.levels.size();
        auto up_u = [&](const std::vector<u32>& v) {
            A.iu.emplace_back();
            A.iu.back().upload(v, stream_);
            return A.iu.size() - 1;
        };
        auto up_d = [&](const std::vector<double>& v) {
            A.dv.emplace_back();
            A.dv.back().upload(v, stream_);
            return A.dv.size() - 1;
        };
        struct Idx {
            size_t a[3], p[3], t[3], dinv;
        };
        std::vector<Idx> ix(L);
        for (size_t l = 0; l < L; l++) {
            const AmgLevel& Lv = H.levels[l];
            ix[l].a[0] = up_u(Lv.A.ptr);
            ix[l].a[1] = up_u(Lv.A.col);
            ix[l].a[2] = up_d(Lv.A.val);
            ix[l].dinv = up_d(Lv.dinv);
            if (l + 1 < L) {
                ix[l].p[0] = up_u(Lv.P.ptr);
                ix[l].p[1] = up_u(Lv.P.col);
                ix[l].p[2] = up_d(Lv.P.val);
                ix[l].t[0] = up_u(Lv.Pt.ptr);
                ix[l].t[1] = up_u(Lv.Pt.col);
                ix[l].t[2] = up_d(Lv.Pt.val);
            }
        }
        // the pointers, once every upload is in place (the buffer vectors no longer grow)
        for (size_t l = 0; l < L; l++) {
            const Idx& q = ix[l];
            DevAmgLevel dl{};
            dl.n = H.levels[l].n;
            dl.A = DevCsr{A.iu[q.a[0]].p, A.iu[q.a[1]].p, A.dv[q.a[2]].p};
            dl.dinv = A.dv[q.dinv].p;
            if (l + 1 < L) {
                dl.P = DevCsr{A.iu[q.p[0]].p, A.iu[q.p[1]].p, A.dv[q.p[2]].p};
                dl.Pt = DevCsr{A.iu[q.t[0]].p, A.iu[q.t[1]].p, A.dv[q.t[2]].p};
            }
            A.lv.push_back(dl);
        }
        // generalized inverse of the coarsest level: unit-diagonal scaling over the nodes with a
        // positive diagonal, grounded LDL^T, explicit inverse (the small block's kernels)
        std::vector<u32> keep;
        for (u32 i = 0; i < nL; i++)
            if (H.coarse[size_t(i) * nL + i] > 0.0) keep.push_back(i);
        const size_t k = keep.size();
        std::vector<double> scale(k), ak(k * k);
        for (size_t i = 0; i < k; i++) scale[i] = 1.0 / std::sqrt(H.coarse[size_t(keep[i]) * (nL + 1)]);
        for (size_t i = 0; i < k; i++)
            for (size_t j = 0; j < k; j++) ak[i * k + j] = H.coarse[size_t(keep[i]) * nL + keep[j]] * scale[i] * scale[j];
        A.minv.alloc(size_t(nL) * nL);
        CK(cudaMemsetAsync(A.minv.p, 0, size_t(nL) * nL * sizeof(double), stream_));
        if (k > 0) {
            DBuf<double> da, dd, dx, dscale;
            DBuf<u32> dkeep;
            da.upload(ak, stream_);
            dd.alloc(k);
            dx.alloc(k * k);
            dscale.upload(scale, stream_);
            dkeep.upload(keep, stream_);
            dense_ldlt_inverse(da.p, dd.p, int(k), dx.p, stream_, d_->launches);
            k_expand_minv<<<grid_for(k * k), THREADS, 0, stream_>>>(dx.p, dkeep.p, dscale.p, int(k), nL, A.minv.p);
            CK(cudaGetLastError());
            d_->launches++;
            CK(cudaStreamSynchronize(stream_));
        }
        d_->amg.push_back(std::move(A));
    }
    CK(cudaStreamSynchronize(stream_));
}

size_t GpuAbsorber::escalated_blocks() const { return d_->amg.size(); }
u64 GpuAbsorber::escalations() const { return d_->escalations; }

GpuAbsorber::~GpuAbsorber() {
    d_.reset();
    if (stream_) cudaStreamDestroy(stream_);
}

bool GpuAbsorber::weights(double* out) const {
    if (!weighted_) return false;
    sync_host_weights();
    if (out) std::copy(w_rows_.begin(), w_rows_.end(), out);
    return true;
}

// Device form of refresh_weights for row-order weights already in device memory: every array
// of the weight state is computed on the device (weights.cuh); the host mirrors are copied back
// only when a host-side reader needs them.
void GpuAbsorber::set_weights_device(const double* w_dev) {
    AllocScope alloc_scope(stream_);
    ctx_.check();
    const HostStructure& st = hs_;
    const size_t n = st.n, M = st.ncells, g1 = st.g1, m = st.m;
    Scratch& d = *d_;
    d.wflag.alloc(1);
    CK(cudaMemsetAsync(d.wflag.p, 0, sizeof(int), stream_));
    k_check_weights<<<grid_for(n), THREADS, 0, stream_>>>(w_dev, n, d.wflag.p);
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, d.wflag.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    if (bad) throw Error(RC_INVALID_INPUT, "weights must be positive and finite");
    d.w_rows.alloc(n);
    CK(cudaMemcpyAsync(d.w_rows.p, w_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    d.cell_w.alloc(M);
    if (st.trivial()) CK(cudaMemcpyAsync(d.cell_w.p, w_dev, M * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    else k_cell_weights<<<grid_for(M), THREADS, 0, stream_>>>(w_dev, d.cell_row.p, u32(M), d.cell_w.p);
    d.n1.alloc(g1);
    d.n1inv.alloc(g1);
    k_seg_weights<<<grid_for(g1), THREADS, 0, stream_>>>(d.cell_w.p, d.seg_off.p, u32(g1), d.n1.p, d.n1inv.p);
    d.wpart.alloc(GRID_V);
    k_vec_sum<<<GRID_V, 256, 0, stream_>>>(d.n1.p, g1, d.wpart.p);
    d.launches += 4;
    std::vector<double> part(GRID_V);
    CK(cudaMemcpyAsync(part.data(), d.wpart.p, GRID_V * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    CK(cudaGetLastError());
    sw_ = 0.0;
    for (double v : part) sw_ += v;
    weighted_ = true;
    host_stale_ = true;
    // nr is part of the operator (the diagonal of S P), so the coordinate weight state is
    // recomputed now; the dense small factor and the hierarchies of earlier weights stay as
    // stale preconditioners (they change the iteration count, not the operator) until a slow
    // probe asks for a stronger preconditioner (escalate).
    coord_stale_ = m > 0;
    refresh_coord();
    build_srow();
    small_stale_ = small_ok_;
    pre_fresh_ = small_ok_;
    amg_stale_ = true;
}

// nr, diag, redundant and the Jacobi factors on the device for the current cell weights.
void GpuAbsorber::refresh_coord() const {
    if (!coord_stale_) return;
    const size_t m = hs_.m;
    Scratch& d = *d_;
    d.nr.alloc(m);
    d.diag.alloc(m);
    d.red.alloc(m);
    d.inv_diag.alloc(m);
    const u32 nch = d.cw_nchunks;
    d.cw_chunks.alloc(size_t(nch) * sizeof(CwChunk) / sizeof(double));
    CwChunk* ch = reinterpret_cast<CwChunk*>(d.cw_chunks.p);
    k_coord_chunks<<<int(std::min<size_t>((size_t(nch) * 32 + THREADS - 1) / THREADS, size_t(GRID_T) * 8)), THREADS, 0,
                     stream_>>>(d.cw_e0.p, d.cw_e1.p, nch, d.pl_cell.p, d.pl_seg.p, d.cell_w.p, d.n1inv.p, ch);
    k_coord_combine<<<grid_for(m), THREADS, 0, stream_>>>(d.cw_list_off.p, u32(m), ch, d.n1inv.p, d.nr.p, d.diag.p,
                                                          d.red.p, d.inv_diag.p);
    d.launches += 2;
    CK(cudaGetLastError());
    coord_stale_ = false;
}

// Copies the device weight state back into the host mirrors after set_weights_device.
void GpuAbsorber::sync_host_weights() const {
    AllocScope alloc_scope(stream_);
    if (!host_stale_) return;
    refresh_coord();
    const HostStructure& st = hs_;
    const size_t n = st.n, M = st.ncells, g1 = st.g1, m = st.m;
    Scratch& d = *d_;
    // unweighted: no row weights; unit cells: no cell weights (both read as 1)
    w_rows_.resize(d.w_rows.p ? n : 0);
    cell_w_.resize(d.cell_w.p ? M : 0);
    n1_.resize(g1);
    nr_.resize(m);
    diag_.resize(m);
    red_.resize(m);
    if (d.w_rows.p) CK(cudaMemcpyAsync(w_rows_.data(), d.w_rows.p, n * 8, cudaMemcpyDeviceToHost, stream_));
    if (d.cell_w.p) CK(cudaMemcpyAsync(cell_w_.data(), d.cell_w.p, M * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(n1_.data(), d.n1.p, g1 * 8, cudaMemcpyDeviceToHost, stream_));
    if (m > 0) {
        CK(cudaMemcpyAsync(nr_.data(), d.nr.p, m * 8, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(diag_.data(), d.diag.p, m * 8, cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(red_.data(), d.red.p, m, cudaMemcpyDeviceToHost, stream_));
    }
    CK(cudaStreamSynchronize(stream_));
    host_stale_ = false;
}

// The dense rows of S on the small coordinates (weights.cuh) for the current cell weights: part
// of the operator, so rebuilt with every weight state (unlike the preconditioners).
void GpuAbsorber::build_srow() {
    Scratch& d = *d_;
    if (!d.srow_on || d.si_n == 0) return;
    const HostStructure& st = hs_;
    const u32 ms = d.ms_acc, M = u32(st.ncells), g1 = st.g1, m = u32(st.m);
    const int ns = int(d.ns_acc);
    const double* cw = d.cell_w.p;  // null: unit cell weights
    DBuf<double> csk, part;
    csk.alloc(size_t(g1) * ms);
    part.alloc(size_t(d.si_n) * ms);
    d.srow.alloc(size_t(m) * ms);
    k_seg_small_w<<<grid_for(size_t(g1) * ms), THREADS, 0, stream_>>>(d.seg_off.p, d.coord.p, M, g1, ns, ms, cw,
                                                                       csk.p);
    k_srow_items<<<(d.si_n + 7) / 8, 256, 0, stream_>>>(d.coord.p, M, ns, ms, cw, d.n1inv.p, d.pl_cell.p, d.pl_seg.p,
                                                        csk.p, d.si_a.p, d.si_b.p, d.si_n, part.p);
    k_srow_sum<<<grid_for(size_t(m) * ms), THREADS, 0, stream_>>>(part.p, d.si_first.p, m, ms, d.srow.p);
    d.launches += 3;
    CK(cudaGetLastError());
}

void GpuAbsorber::set_weights(const double* w_rows) {
    AllocScope alloc_scope(stream_);
    ctx_.check();
    if (!w_rows) {
        unit_weights_device();
        return;
    }
    DBuf<double> wd;
    wd.upload(w_rows, hs_.n, stream_);
    set_weights_device(wd.p);
    CK(cudaStreamSynchronize(stream_));
}

void GpuAbsorber::weight_state(double* n1, double* nr, double* diag, uint8_t* red, double* sw) const {
    sync_host_weights();
    if (n1) std::copy(n1_.begin(), n1_.end(), n1);
    if (nr) std::copy(nr_.begin(), nr_.end(), nr);
    if (diag) std::copy(diag_.begin(), diag_.end(), diag);
    if (red) std::copy(red_.begin(), red_.end(), red);
    if (sw) *sw = sw_;
}

// Jacobi entries (precond/jacobi.rs:7) and the exact dense factor of the small super-block
// (precond/dense.rs:79-160), both from the device weight state: the Jacobi factors come with the
// coordinate weights (refresh_coord), S_SS is assembled on the device, scaled to unit diagonal
// over the kept coordinates, factored with grounding and inverted.
void GpuAbsorber::ensure_precond() {
    if (pre_fresh_) return;
    const size_t ms = hs_.m_small;
    refresh_coord();
    small_ok_ = false;
    if (ms > 0 && ms <= DENSE_SMALL_MAX) build_small_device();
    pre_fresh_ = true;
}

// The dense small factor from the device assembly of S_SS (weights.cuh) for the device weight
// state: by rows (k_small_rows over the work items built with the coordinate lists), each row's
// items summed in item order.
void GpuAbsorber::build_small_device() {
    const HostStructure& st = hs_;
    const size_t ms = st.m_small, M = st.ncells;
    Scratch& d = *d_;
    int ns = 0;
    for (auto& b : st.blocks) ns += b.small;
    const size_t len = ms * ms;
    DBuf<double> part, a, ak, dd, dx, dscale;
    DBuf<u32> dkeep;
    a.alloc(len);
    if (d.sr_n > 0) {
        part.alloc(size_t(d.sr_n) * ms);
        const size_t shm = size_t(8) * ms * sizeof(double);
        allow_smem(k_small_rows, shm);
        k_small_rows<<<(d.sr_n + 7) / 8, 256, shm, stream_>>>(d.seg_off.p, d.coord.p, u32(M), ns, u32(ms),
                                                               d.cell_w.p, d.n1inv.p, d.pl_cell.p, d.pl_seg.p,
                                                               d.sr_k.p, d.sr_a.p, d.sr_b.p, d.sr_n, part.p);
        k_small_rows_sum<<<u32(ms), 256, 0, stream_>>>(part.p, d.sr_first.p, u32(ms), a.p);
        d.launches += 2;
    } else {  // no small coordinate has a cell
        CK(cudaMemsetAsync(a.p, 0, len * sizeof(double), stream_));
    }
    // kept coordinates (not redundant, positive diagonal) and their unit-diagonal scaling
    std::vector<double> diag(ms);
    std::vector<uint8_t> red(ms);
    CK(cudaMemcpy2DAsync(diag.data(), sizeof(double), a.p, (ms + 1) * sizeof(double), sizeof(double), ms,
                         cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(red.data(), d.red.p, ms, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    std::vector<u32> keep;
    for (size_t i = 0; i < ms; i++)
        if (!red[i] && diag[i] > 0.0) keep.push_back(u32(i));
    const size_t k = keep.size();
    std::vector<double> scale(k);
    for (size_t i = 0; i < k; i++) scale[i] = 1.0 / std::sqrt(diag[keep[i]]);
    d.minv.alloc(len);
    CK(cudaMemsetAsync(d.minv.p, 0, len * sizeof(double), stream_));
    if (k > 0) {
        dkeep.upload(keep, stream_);
        dscale.upload(scale, stream_);
        ak.alloc(k * k);
        dd.alloc(k);
        dx.alloc(k * k);
        k_small_gather<<<grid_for(k * k), THREADS, 0, stream_>>>(a.p, u32(ms), dkeep.p, dscale.p, int(k), ak.p);
        dense_ldlt_inverse(ak.p, dd.p, int(k), dx.p, stream_, d.launches);
        k_expand_minv<<<grid_for(k * k), THREADS, 0, stream_>>>(dx.p, dkeep.p, dscale.p, int(k), u32(ms), d.minv.p);
        d.launches += 2;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    small_ok_ = true;
}

namespace {

// Lets `kernel` take `bytes` of dynamic shared memory (static and dynamic together may pass the
// 48 KB default) through smem_limit (device.cuh): set once per kernel, to the most it can take.
template <class K>
void allow_smem(K kernel, size_t bytes) {
    if (bytes == 0) return;
    if (bytes > size_t(smem_limit(kernel)))
        throw Error(RC_INTERNAL, "fereg: a kernel needs more shared memory than a block can take");
}

// Grounded LDL^T of the k x k row-major `a` (lower triangle read, overwritten) and its inverse
// into x (k x k), on `st`: panels of NB columns (16 up to k = 1024, 8 beyond, so that a panel of
// k rows fits the shared memory of one CTA), each followed by its trailing update.
void dense_ldlt_inverse(double* a, double* d, int k, double* x, cudaStream_t st, u64& launches) {
    if (k <= 0) return;
    auto factor = [&](auto nbc) {
        constexpr int NB = decltype(nbc)::value;
        allow_smem(k_ldlt_panel<NB>, size_t(k) * NB * sizeof(double));
        for (int jb = 0; jb < k; jb += NB) {
            const int nb = std::min(NB, k - jb);
            k_ldlt_panel<NB><<<1, 1024, size_t(k - jb) * NB * sizeof(double), st>>>(a, d, k, jb);
            launches++;
            const int T = (k - jb - nb + 31) / 32;  // trailing tiles per side
            if (T > 0) {
                k_ldlt_trail<NB><<<T * (T + 1) / 2, 256, 0, st>>>(a, d, k, jb, nb);
                launches++;
            }
        }
    };
    if (k <= 1024) factor(std::integral_constant<int, 16>{});
    else factor(std::integral_constant<int, 8>{});
    allow_smem(k_ldlt_inverse, size_t(8) * k * sizeof(double));
    k_ldlt_inverse<<<(k + 7) / 8, 256, size_t(8) * k * sizeof(double), st>>>(a, d, k, x);
    launches++;
    CK(cudaGetLastError());
}

// Per-CTA partial rows of the small coordinates: GRID_S rows of the short-segment kernels, then
// GRID_T rows of the long-segment tiles, then GRID_T rows of the long-segment slices.
inline size_t small_rows() { return size_t(GRID_S) + 2 * size_t(GRID_T); }

template <class T>
void launch_small_reduce(Scratch& d, const DevStruct& S, T* small, int R, T* Y, cudaStream_t st) {
    const u32 len = S.ms_acc * u32(R);
    T* sb = small + size_t(GRID_S) * len;
    T* sc = sb + size_t(GRID_T) * len;
    k_small_reduce<T><<<std::max<u32>(1, std::min<u32>((len + 7) / 8, GRID_V)), THREADS, 0, st>>>(
        small, GRID_S, S.seg.n ? sb : nullptr, GRID_T, S.seg.nfix ? sc : nullptr, GRID_T, len, Y);
    d.launches++;
}

// Y = S P on the PCG's padded vectors (Rv a multiple of 4). Short segments: one lane group per
// segment (k_vseg_apply); long segments: CTA tiles, their slices' partials completed by k_fix.
// Short coordinate lists: warp tiles (k_vpull_apply); long ones: CTA tiles and k_fix. The small
// coordinates' rows (ms_acc > 0) come from the dense rows of S (k_srow_apply), their CTA
// partials added by k_small_reduce.
template <class T>
void launch_apply(Scratch& d, const DevStruct& S, const DevWeights& W, const T* P, int Rv, T* Y, T* t, T* part,
                  T* small, cudaStream_t st) {
    if (Rv % 4 != 0) throw Error(RC_INTERNAL, "fereg: the operator takes padded vectors (a multiple of 4 columns)");
    const bool weighted = W.cell_w != nullptr;
    const auto gi = d.grids.find({Rv, int(sizeof(T))});
    const Scratch::ApplyGrids grid = gi == d.grids.end() ? Scratch::ApplyGrids{} : gi->second;
    int h = d.begin(GpuAbsorber::P_APPLY, st);
    DevStruct SA = S;  // the operator's segment tiles
    SA.seg = d.aseg_tiles.set();
    if (d.aseg_segs.n)
        for (int j0 = 0; j0 < Rv; j0 += VCOLS) {
            const int Rc = std::min(VCOLS, Rv - j0);
            const u32 nsegs = u32(d.aseg_segs.n);
            const size_t sm = small_stage_bytes<T>(S.ms_acc, Rc);
            const int stage = S.ns_acc > 0 && sm <= SMALL_STAGE_MAX;
            auto go = [&](auto lc, auto nbk, auto wc) {
                constexpr int L = decltype(lc)::value, NBK = decltype(nbk)::value;
                constexpr bool WT_ = decltype(wc)::value;
                k_vseg_apply<T, L, NBK, WT_><<<grid.seg, WPB * 32, stage ? sm : 0, st>>>(S, W, d.aseg_segs.p, nsegs,
                                                                                         P, Rv, j0, Rc, t, stage);
            };
            with_vlanes(Rc, S.nb, [&](auto lc, auto nbk) {
                if (weighted) go(lc, nbk, std::true_type{});
                else go(lc, nbk, std::false_type{});
            });
            d.launches++;
        }
    if (SA.seg.n) {
        k_seg_apply<T><<<GRID_T, THREADS, 0, st>>>(SA, W, P, Rv, t, part, false, nullptr);
        d.launches++;
        if (SA.seg.nfix) {
            k_fix<T><<<std::min<u32>(SA.seg.nfix, GRID_T), THREADS, 0, st>>>(SA.seg, W, P, part, Rv, 1, t);
            d.launches++;
        }
    }
    d.end(h, st);
    h = d.begin(GpuAbsorber::P_APPLY_PULL, st);
    if (d.wpull.n)
        for (int j0 = 0; j0 < Rv; j0 += VCOLS) {
            const int Rc = std::min(VCOLS, Rv - j0);
            const size_t sm = small_stage_bytes<T>(S.ms_acc, Rc);
            const int stage = S.ns_acc > 0 && sm <= SMALL_STAGE_MAX;
            auto go = [&](auto lc, auto nbk, auto wc) {
                constexpr int L = decltype(lc)::value, NBK = decltype(nbk)::value;
                constexpr bool WT_ = decltype(wc)::value;
                const size_t shm = WPB * vpull_warp_bytes<NBK - 1, WT_>() + (stage ? sm : 0);
                allow_smem(k_vpull_apply<T, L, NBK, WT_>, shm);
                k_vpull_apply<T, L, NBK, WT_><<<grid.pull, WPB * 32, shm, st>>>(S, W, d.wpull.set(), P, t, Rv, j0, Rc,
                                                                                Y, stage);
            };
            with_vlanes(Rc, S.nb, [&](auto lc, auto nbk) {
                if (weighted) go(lc, nbk, std::true_type{});
                else go(lc, nbk, std::false_type{});
            });
            d.launches++;
        }
    if (S.pull.n) {
        k_pull_apply<T><<<GRID_T, THREADS, 0, st>>>(S, W, P, t, Rv, Y, part);
        d.launches++;
        if (S.pull.nfix) {
            k_fix<T><<<std::min<u32>(S.pull.nfix, GRID_T), THREADS, 0, st>>>(S.pull, W, P, part, Rv, 0, Y);
            d.launches++;
        }
    }
    if (S.ms_acc > 0) {
        if (!d.srow_on) throw Error(RC_INTERNAL, "fereg: the dense small rows are missing");
        const u32 len = S.ms_acc * u32(Rv);
        const u32 grid = std::max<u32>(1, std::min<u32>(4 * GRID_V, (S.m + 31) / 32));
        k_srow_apply<T><<<grid, THREADS, 0, st>>>(d.srow.p, S.m, S.ms_acc, P, Rv, small);
        k_small_reduce<T><<<std::max<u32>(1, std::min<u32>((len + 7) / 8, GRID_V)), THREADS, 0, st>>>(
            small, int(grid), nullptr, 0, nullptr, 0, len, Y);
        d.launches += 2;
    }
    CK(cudaGetLastError());
    d.end(h, st);
}

// The project's autotuner for the S*P passes: the grid of k_vseg_apply and of k_vpull_apply among
// 1, 2, 4, 8 and 16 CTAs per SM (a grid only partitions the lane groups and list tiles, so every
// choice gives the same bits), each timed with CUDA events on the solver's stream (one untimed
// launch, then the shorter of two) on the solve's own vectors. The choice is kept for the process
// under the structure's shape (the powers of two of the cells, segments, coordinates and small
// coordinates; blocks, padded width, element size, weighted), so later sessions of a similar shape
// reuse it. FEREG_AUTOTUNE=0 turns it off (the default grid, 4 CTAs per SM). Passes under 2^20
// cells are not tuned.
std::mutex g_tune_mu;
std::map<std::vector<u64>, Scratch::ApplyGrids> g_tuned;

template <class T>
void autotune_apply(Scratch& d, const DevStruct& S, const DevWeights& W, T* P, int Rv, T* Y, T* t, T* part, T* small,
                    cudaStream_t st) {
    const std::pair<int, int> key{Rv, int(sizeof(T))};
    if (d.grids.count(key) || d.prof || S.M < (1u << 20)) return;
    const char* env = std::getenv("FEREG_AUTOTUNE");
    if (env && env[0] == '0') return;
    // sizes by their power of two: structures of a similar size share a choice (a serving loop's
    // requests each have their own exact sizes)
    auto lg = [](u64 v) { return u64(v ? 64 - __builtin_clzll(v) : 0); };
    const std::vector<u64> shape{lg(S.M), lg(S.g1), lg(S.m), S.nb, lg(S.ms_acc), u64(Rv), sizeof(T),
                                 W.cell_w != nullptr};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        const auto it = g_tuned.find(shape);
        if (it != g_tuned.end()) {
            d.grids[key] = it->second;
            return;
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int cand[] = {148, 296, 592, 1184, 2368};
    Scratch::ApplyGrids best;
    auto time_of = [&]() {
        float mn = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            CK(cudaEventRecord(e0, st));
            launch_apply<T>(d, S, W, P, Rv, Y, t, part, small, st);
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) mn = std::min(mn, ms);
        }
        return mn;
    };
    // the segment pass's grid with the pull pass at its default, then the pull pass's
    for (int pass = 0; pass < 2; pass++) {
        float bt = 1e30f;
        int bg = 148 * 4;
        for (int g : cand) {
            Scratch::ApplyGrids trial = best;
            (pass == 0 ? trial.seg : trial.pull) = g;
            d.grids[key] = trial;
            const float ms = time_of();
            if (ms < bt) {
                bt = ms;
                bg = g;
            }
        }
        (pass == 0 ? best.seg : best.pull) = bg;
    }
    d.grids[key] = best;
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    d.tune_us += std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[shape] = best;
}

// The V-cycle's work vectors of every level for R columns (allocated before a graph capture).
template <class T>
void amg_alloc(DevAmgBlock& A, int R) {
    const size_t L = A.lv.size();
    std::vector<DBuf<T>>& w = amg_work<T>(A);
    if (w.size() != 3 * L) w.resize(3 * L);
    for (size_t l = 0; l < L; l++) {
        const size_t len = size_t(A.lv[l].n) * R;
        if (l > 0) {
            w[3 * l].alloc(len);
            w[3 * l + 1].alloc(len);
        }
        if (l + 1 < L) w[3 * l + 2].alloc(len);
    }
}

// One V(1,1) cycle (amg.cuh) on the block's slice of r into the same slice of z.
template <class T>
void launch_amg(Scratch& d, DevAmgBlock& A, const T* r, T* z, int R, cudaStream_t st) {
    const size_t L = A.lv.size();
    amg_alloc<T>(A, R);
    std::vector<DBuf<T>>& w = amg_work<T>(A);
    std::vector<const T*> rin(L);
    std::vector<T*> zout(L), z1(L);
    rin[0] = r + size_t(A.off) * R;
    zout[0] = z + size_t(A.off) * R;
    for (size_t l = 0; l < L; l++) {
        if (l > 0) {
            rin[l] = w[3 * l].p;
            zout[l] = w[3 * l + 1].p;
        }
        if (l + 1 < L) z1[l] = w[3 * l + 2].p;
    }
    for (size_t l = 0; l + 1 < L; l++) {
        const u32 nc = A.lv[l + 1].n;
        k_amg_resid<T><<<grid_for(size_t(A.lv[l].n) * R), THREADS, 0, st>>>(A.lv[l], rin[l], R, z1[l]);
        k_amg_restrict<T><<<grid_for(size_t(nc) * R), THREADS, 0, st>>>(A.lv[l].Pt, nc, z1[l], R, w[3 * (l + 1)].p);
        d.launches += 2;
    }
    k_amg_dense<T><<<grid_for(size_t(A.lv[L - 1].n) * R), THREADS, 0, st>>>(A.minv.p, A.lv[L - 1].n, rin[L - 1], R,
                                                                          zout[L - 1]);
    d.launches++;
    for (size_t l = L - 1; l-- > 0;) {
        const size_t len = size_t(A.lv[l].n) * R;
        k_amg_up1<T><<<grid_for(len), THREADS, 0, st>>>(A.lv[l], rin[l], zout[l + 1], R, z1[l]);
        k_amg_up2<T><<<grid_for(len), THREADS, 0, st>>>(A.lv[l], rin[l], z1[l], R, zout[l]);
        d.launches += 2;
    }
}

template <class T>
void launch_precond(Scratch& d, const DevStruct& S, bool small_ok, const T* r, T* z, int R, cudaStream_t st) {
    const int h = d.begin(GpuAbsorber::P_PRECOND, st);
    const u32 ms = small_ok ? S.ms : 0;
    if (S.m > ms) {
        k_jacobi<T><<<grid_for(size_t(S.m - ms) * R), THREADS, 0, st>>>(r, z, d.inv_diag.p, ms, S.m, R);
        d.launches++;
    }
    if (ms > 0) {
        k_small_apply<T><<<grid_for(size_t(ms) * R * 32), THREADS, 0, st>>>(d.minv.p, ms, r, z, R);
        d.launches++;
    }
    for (auto& a : d.amg) launch_amg<T>(d, a, r, z, R, st);  // escalated blocks replace their Jacobi values
    CK(cudaGetLastError());
    d.end(h, st);
}

void reduce_cols(Scratch& d, const double* part, int nparts, int ncols, double* out, cudaStream_t st,
                 const double* part2 = nullptr, int nparts2 = 0) {
    k_reduce_cols<<<std::max(1, std::min(GRID_V, (ncols + 7) / 8)), THREADS, 0, st>>>(part, nparts, part2, nparts2,
                                                                                       ncols, out);
    d.launches++;
    CK(cudaGetLastError());
}

// rhs pass: b1 per segment, [sum w v^2, sum w v, sum b1^2/n1] per column into colsum (3R), and
// the reduced right-hand side (small coordinates in the segment passes, the others pulled).
void launch_rhs(Scratch& d, const DevStruct& S, const DevWeights& W, const double* rows, int R, double* b1,
                double* rhs, double* colsum, cudaStream_t st) {
    const bool acc = S.ms_acc > 0;
    const u32 len = S.ms_acc * u32(R);
    double* small = d.small.p;
    int h = d.begin(GpuAbsorber::P_RHS_SEG, st);
    if (d.wseg.n) {
        for (int j0 = 0; j0 < R; j0 += WCOLS) {
            const int Rc = std::min(WCOLS, R - j0);
            const size_t shm = grhs_smem(S.ms_acc);
            with_lanes<WNB>(Rc, WNB, [&](auto c, auto) {
                constexpr int RCP = decltype(c)::value;
                with_nsa(acc ? S.ns_acc : 0u, [&](auto nsa) {
                    constexpr int NSA = decltype(nsa)::value;
                    allow_smem(k_grhs<RCP, NSA>, shm);
                    k_grhs<RCP, NSA><<<GRID_S, WPB * 32, shm, st>>>(S, W, d.wseg_segs.p, u32(d.wseg_segs.n), rows, R,
                                                                     j0, Rc, b1, d.cta2.p, acc ? small : nullptr);
                });
            });
            d.launches++;
        }
    } else {
        CK(cudaMemsetAsync(d.cta2.p, 0, size_t(GRID_S) * 2 * R * sizeof(double), st));
        if (acc) CK(cudaMemsetAsync(small, 0, size_t(GRID_S) * len * sizeof(double), st));
    }
    if (S.seg.n) {
        double* sb = small + size_t(GRID_S) * len;
        k_seg_rhs<<<GRID_T, THREADS, 0, st>>>(S, W, rows, R, b1, d.part.p, d.cta.p, acc ? sb : nullptr);
        d.launches++;
        if (S.seg.nfix) {
            k_fix<double><<<std::min<u32>(S.seg.nfix, GRID_T), THREADS, 0, st>>>(S.seg, W, nullptr, d.part.p, R, 2, b1);
            d.launches++;
            if (acc) {
                k_rhs_small_slices<<<GRID_T, THREADS, 0, st>>>(S, W, rows, b1, R, sb + size_t(GRID_T) * len);
                d.launches++;
            }
        }
    }
    d.end(h, st);
    h = d.begin(GpuAbsorber::P_VECTOR, st);
    reduce_cols(d, d.cta2.p, GRID_S, 2 * R, colsum, st, S.seg.n ? d.cta.p : nullptr, GRID_T);
    k_b1sq<<<GRID_V, THREADS, 0, st>>>(S.g1, b1, W.n1inv, R, d.cta.p);
    d.launches++;
    reduce_cols(d, d.cta.p, GRID_V, R, colsum + 2 * R, st);
    d.end(h, st);
    if (S.m > 0) {
        h = d.begin(GpuAbsorber::P_RHS_PULL, st);
        if (d.wpull.n)
            for (int j0 = 0; j0 < R; j0 += WCOLS) {
                const int Rc = std::min(WCOLS, R - j0);
                with_rcp<WNB>(Rc, WNB, [&](auto c, auto) {
                    constexpr int RCP = decltype(c)::value;
                    k_wpull_rhs<RCP><<<GRID_S, WPB * 32, wpull_smem(), st>>>(S, W, d.wpull.set(), rows, b1, R, j0, Rc,
                                                                              rhs);
                });
                d.launches++;
            }
        if (S.pull.n) {
            k_pull_rhs<<<GRID_T, THREADS, 0, st>>>(S, W, rows, b1, R, rhs, d.part.p);
            d.launches++;
            if (S.pull.nfix) {
                k_fix<double><<<std::min<u32>(S.pull.nfix, GRID_T), THREADS, 0, st>>>(S.pull, W, nullptr, d.part.p, R, 2, rhs);
                d.launches++;
            }
        }
        if (acc) launch_small_reduce<double>(d, S, small, R, rhs, st);
        d.end(h, st);
    }
    CK(cudaGetLastError());
}

// Scratch of the right-hand side pass held outside the handle (the allocation-free entry point):
// per-CTA column partials of the short (cta2) and long (cta) segment kernels, slice partials of
// the long lists (part) and the small coordinates' partial rows (small). Sizes in doubles.
struct RhsScratch {
    double *cta2, *cta, *part, *small;
};
inline size_t rhs_scratch_part(size_t doubles) { return (doubles + 31) / 32 * 32; }  // 256-byte steps
inline size_t rhs_scratch_need(const DevStruct& S, size_t r, u32 ms_acc) {
    return rhs_scratch_part(size_t(GRID_S) * 2 * r) + rhs_scratch_part(size_t(std::max(GRID_T, GRID_V)) * 3 * r) +
           rhs_scratch_part(std::max<size_t>(1, size_t(std::max(S.seg.nparts, S.pull.nparts)) * r)) +
           rhs_scratch_part(std::max<size_t>(1, small_rows() * ms_acc * r));
}
inline RhsScratch rhs_scratch_carve(double* p, const DevStruct& S, size_t r, u32 ms_acc) {
    RhsScratch s;
    s.cta2 = p;
    p += rhs_scratch_part(size_t(GRID_S) * 2 * r);
    s.cta = p;
    p += rhs_scratch_part(size_t(std::max(GRID_T, GRID_V)) * 3 * r);
    s.part = p;
    p += rhs_scratch_part(std::max<size_t>(1, size_t(std::max(S.seg.nparts, S.pull.nparts)) * r));
    s.small = p;
    return s;
}

// The kernels of launch_rhs, in the same order, on the scratch `x` (no phase timing).
void launch_rhs_scratch(Scratch& d, const DevStruct& S, const DevWeights& W, const double* rows, int R, double* b1,
                        double* rhs, double* colsum, const RhsScratch& x, cudaStream_t st) {
    const bool acc = S.ms_acc > 0;
    const u32 len = S.ms_acc * u32(R);
    if (d.wseg.n) {
        for (int j0 = 0; j0 < R; j0 += WCOLS) {
            const int Rc = std::min(WCOLS, R - j0);
            const size_t shm = grhs_smem(S.ms_acc);
            with_lanes<WNB>(Rc, WNB, [&](auto c, auto) {
                constexpr int RCP = decltype(c)::value;
                with_nsa(acc ? S.ns_acc : 0u, [&](auto nsa) {
                    constexpr int NSA = decltype(nsa)::value;
                    allow_smem(k_grhs<RCP, NSA>, shm);
                    k_grhs<RCP, NSA><<<GRID_S, WPB * 32, shm, st>>>(S, W, d.wseg_segs.p, u32(d.wseg_segs.n), rows, R,
                                                                     j0, Rc, b1, x.cta2, acc ? x.small : nullptr);
                });
            });
            d.launches++;
        }
    } else {
        // the short-segment partials start at zero when no short-segment kernel writes them
        CK(cudaMemsetAsync(x.cta2, 0, size_t(GRID_S) * 2 * R * sizeof(double), st));
        if (acc) CK(cudaMemsetAsync(x.small, 0, size_t(GRID_S) * len * sizeof(double), st));
    }
    if (S.seg.n) {
        double* sb = x.small + size_t(GRID_S) * len;
        k_seg_rhs<<<GRID_T, THREADS, 0, st>>>(S, W, rows, R, b1, x.part, x.cta, acc ? sb : nullptr);
        d.launches++;
        if (S.seg.nfix) {
            k_fix<double><<<std::min<u32>(S.seg.nfix, GRID_T), THREADS, 0, st>>>(S.seg, W, nullptr, x.part, R, 2, b1);
            d.launches++;
            if (acc) {
                k_rhs_small_slices<<<GRID_T, THREADS, 0, st>>>(S, W, rows, b1, R, sb + size_t(GRID_T) * len);
                d.launches++;
            }
        }
    }
    reduce_cols(d, x.cta2, GRID_S, 2 * R, colsum, st, S.seg.n ? x.cta : nullptr, GRID_T);
    k_b1sq<<<GRID_V, THREADS, 0, st>>>(S.g1, b1, W.n1inv, R, x.cta);
    d.launches++;
    reduce_cols(d, x.cta, GRID_V, R, colsum + 2 * R, st);
    if (S.m > 0) {
        if (d.wpull.n)
            for (int j0 = 0; j0 < R; j0 += WCOLS) {
                const int Rc = std::min(WCOLS, R - j0);
                with_rcp<WNB>(Rc, WNB, [&](auto c, auto) {
                    constexpr int RCP = decltype(c)::value;
                    k_wpull_rhs<RCP><<<GRID_S, WPB * 32, wpull_smem(), st>>>(S, W, d.wpull.set(), rows, b1, R, j0, Rc,
                                                                              rhs);
                });
                d.launches++;
            }
        if (S.pull.n) {
            k_pull_rhs<<<GRID_T, THREADS, 0, st>>>(S, W, rows, b1, R, rhs, x.part);
            d.launches++;
            if (S.pull.nfix) {
                k_fix<double><<<std::min<u32>(S.pull.nfix, GRID_T), THREADS, 0, st>>>(S.pull, W, nullptr, x.part, R, 2,
                                                                                      rhs);
                d.launches++;
            }
        }
        if (acc) launch_small_reduce<double>(d, S, x.small, R, rhs, st);
    }
    CK(cudaGetLastError());
}

}  // namespace

void GpuAbsorber::apply_host(const double* p, size_t r, double* y) {
    AllocScope alloc_scope(stream_);
    const size_t m = hs_.m, rv = (r + 3) / 4 * 4;  // the PCG's padded layout
    const DevStruct S = d_->ds(hs_);
    d_->p.alloc(m * rv);
    d_->q.alloc(m * rv);
    d_->t.alloc(size_t(hs_.g1) * rv);
    d_->part.alloc(std::max<size_t>(1, size_t(std::max(S.seg.nparts, S.pull.nparts)) * rv));
    d_->small.alloc(std::max<size_t>(1, small_rows() * d_->ms_acc * rv));
    CK(cudaMemsetAsync(d_->p.p, 0, m * rv * 8, stream_));
    CK(cudaMemcpy2DAsync(d_->p.p, rv * 8, p, r * 8, r * 8, m, cudaMemcpyHostToDevice, stream_));
    launch_apply<double>(*d_, S, d_->dw(), d_->p.p, int(rv), d_->q.p, d_->t.p, d_->part.p, d_->small.p, stream_);
    CK(cudaMemcpy2DAsync(y, r * 8, d_->q.p, rv * 8, r * 8, m, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    d_->collect();
}

void GpuAbsorber::precond_host(const double* rr, size_t r, double* z) {
    AllocScope alloc_scope(stream_);
    ensure_precond();
    const size_t m = hs_.m;
    d_->r.alloc(m * r);
    d_->z.alloc(m * r);
    CK(cudaMemcpyAsync(d_->r.p, rr, m * r * 8, cudaMemcpyHostToDevice, stream_));
    launch_precond<double>(*d_, d_->ds(hs_), small_ok_, d_->r.p, d_->z.p, int(r), stream_);
    CK(cudaMemcpyAsync(z, d_->z.p, m * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    d_->collect();
}

void GpuAbsorber::rhs_host(const double* rows, size_t r, double* y, double* b1, double* wsq, double* wsum) {
    AllocScope alloc_scope(stream_);
    const size_t n = hs_.n, m = hs_.m, g1 = hs_.g1;
    const DevStruct S = d_->ds(hs_);
    d_->rows.alloc(n * r);
    d_->rhs.alloc(std::max<size_t>(1, m * r));
    d_->b1.alloc(g1 * r);
    d_->part.alloc(std::max<size_t>(1, size_t(std::max(S.seg.nparts, S.pull.nparts)) * r));
    d_->cta.alloc(size_t(std::max(GRID_T, GRID_V)) * 3 * r);
    d_->cta2.alloc(size_t(GRID_S) * 2 * r);
    d_->colsum.alloc(3 * r);
    d_->small.alloc(std::max<size_t>(1, small_rows() * d_->ms_acc * r));
    CK(cudaMemcpyAsync(d_->rows.p, rows, n * r * 8, cudaMemcpyHostToDevice, stream_));
    launch_rhs(*d_, S, d_->dw(), d_->rows.p, int(r), d_->b1.p, d_->rhs.p, d_->colsum.p, stream_);
    if (m > 0) CK(cudaMemcpyAsync(y, d_->rhs.p, m * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(b1, d_->b1.p, g1 * r * 8, cudaMemcpyDeviceToHost, stream_));
    std::vector<double> cs(3 * r);
    CK(cudaMemcpyAsync(cs.data(), d_->colsum.p, 3 * r * 8, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    d_->collect();
    for (size_t j = 0; j < r; j++) {
        wsq[j] = cs[j];
        wsum[j] = cs[r + j];
    }
}

void GpuAbsorber::rhs_device_scratch(const double* rows, size_t r, double* rhs, double* b1, double* colsum,
                                     double* scratch, size_t cap) {
    if (r == 0) return;
    const DevStruct S = d_->ds(hs_);
    const size_t need = rhs_scratch_need(S, r, d_->ms_acc);
    if (need > cap) {
        std::ostringstream o;
        o << "fereg: the allocation-free rhs pass needs " << need * sizeof(double) << " bytes of scratch for " << r
          << " columns; its static scratch holds " << cap * sizeof(double) << " bytes";
        throw Error(RC_INVALID_INPUT, o.str());
    }
    launch_rhs_scratch(*d_, S, d_->dw(), rows, int(r), b1, rhs, colsum, rhs_scratch_carve(scratch, S, r, d_->ms_acc),
                       stream_);
}

SolveInfo GpuAbsorber::residualize(double* z, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                                   double* coefs, Precision prec) {
    AllocScope alloc_scope(stream_);
    const size_t n = hs_.n;
    d_->rows.alloc(std::max<size_t>(1, n * r));
    int h = d_->begin(P_H2D, stream_);
    CK(cudaMemcpyAsync(d_->rows.p, z, n * r * 8, cudaMemcpyHostToDevice, stream_));
    d_->end(h, stream_);
    SolveInfo info = solve(d_->rows.p, r, tol, maxiter, want_coefs, warm, coefs, prec);
    h = d_->begin(P_D2H, stream_);
    CK(cudaMemcpyAsync(z, d_->rows.p, n * r * 8, cudaMemcpyDeviceToHost, stream_));
    d_->end(h, stream_);
    CK(cudaStreamSynchronize(stream_));
    d_->collect();
    return info;
}

SolveInfo GpuAbsorber::residualize_device_warm_last(double* z_dev, size_t r, double tol, size_t maxiter,
                                                    Precision prec) {
    AllocScope alloc_scope(stream_);
    ctx_.check();
    if (r == 0) return SolveInfo{1, false, true};
    return solve(z_dev, r, tol, maxiter, false, nullptr, nullptr, prec, true);
}

SolveInfo GpuAbsorber::residualize_device(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs,
                                          const double* warm, double* coefs, Precision prec) {
    AllocScope alloc_scope(stream_);
    return solve(z_dev, r, tol, maxiter, want_coefs, warm, coefs, prec);
}

constexpr int PROBE_FROM = 7, PROBE_AT = 12;
constexpr double PROBE_RATIO = 0.6;

// Iterations a graph launch may run at most before the host looks at the loop state again.
constexpr int GRAPH_CAP = 64;

// The operator of a PCG run on the intercept-only structure: q = S p (launch_apply) and
// z = M^-1 r (launch_precond), with the device addresses their launches touch.
template <class T>
struct FeOp {
    Scratch& d;
    const DevStruct& S;
    const DevWeights& W;
    bool small_ok;
    T *t, *part, *small;
    u32 m() const { return S.m; }
    void apply(T* p, int R, T* q, cudaStream_t st) const { launch_apply<T>(d, S, W, p, R, q, t, part, small, st); }
    void precond(T* r, T* z, int R, cudaStream_t st) const { launch_precond<T>(d, S, small_ok, r, z, R, st); }
    void key(std::vector<u64>& k) const {
        auto put = [&](const void* ptr) { k.push_back(u64(reinterpret_cast<uintptr_t>(ptr))); };
        k.push_back(small_ok);
        for (const void* ptr : {(const void*)t, (const void*)part, (const void*)small, (const void*)W.w_rows,
                                (const void*)W.cell_w, (const void*)W.n1inv, (const void*)W.nr, (const void*)d.inv_diag.p,
                                (const void*)d.minv.p, (const void*)d.srow.p})
            put(ptr);
        k.push_back(d.amg.size());
        for (auto& A : d.amg) {
            put(A.minv.p);
            for (auto& b : A.iu) put(b.p);
            for (auto& b : A.dv) put(b.p);
            for (auto& b : amg_work<T>(A)) put(b.p);
        }
    }
    void prepare(int R) const {
        for (auto& A : d.amg) amg_alloc<T>(A, R);
    }
};

// Every device address the iteration body reads or writes, with the body's shape: a captured
// graph is reused only for an identical key.
template <class T, class Op>
std::vector<u64> body_key(Scratch& d, const Op& op, const T* x, const T* rhs_true, const T* x0, const T* r, const T* z,
                          const T* p, const T* q, int R) {
    std::vector<u64> k;
    auto put = [&](const void* ptr) { k.push_back(u64(reinterpret_cast<uintptr_t>(ptr))); };
    k.push_back(sizeof(T));
    k.push_back(u64(R));
    k.push_back(u64(op.m()));
    put(d.lp_tol.p);
    for (const void* ptr : {(const void*)x, (const void*)rhs_true, (const void*)x0, (const void*)r, (const void*)z,
                            (const void*)p, (const void*)q})
        put(ptr);
    for (const void* ptr : {(const void*)d.cta.p, (const void*)d.lp_ctl.p, (const void*)d.lp_ticket.p,
                            (const void*)d.cg_rho.p, (const void*)d.cg_active.p, (const void*)d.cg_ring.p,
                            (const void*)d.cg_xb.p, (const void*)d.cg_beta.p, (const void*)d.cg_gamma.p,
                            (const void*)d.cg_pfloor.p, (const void*)d.cg_xconst.p, (const void*)d.cg_floor.p,
                            (const void*)d.cg_ss1.p, (const void*)d.cg_pq.p, (const void*)d.cg_rho_new.p,
                            (const void*)d.cg_nactive.p, (const void*)d.lp_rho_from.p, (const void*)d.lp_rho_at.p,
                            (const void*)d.lp_act.p})
        put(ptr);
    op.key(k);
    return k;
}

// The iteration body (cg.rs:207-290): q = S p, gamma, x and r (with the stopping rule's dot
// products), z = M^-1 r, rho and the stopping rule, p. In a graph (use_cond) its last kernel sets
// the WHILE condition.
template <class T, class Op>
void enqueue_iteration(Scratch& d, const Op& op, T* x, const T* rhs_true, const T* x0, T* r, T* z, T* p, T* q, int R,
                       const CgState& cg, const CgLoop& lp, cudaGraphConditionalHandle cond, bool use_cond,
                       cudaStream_t st) {
    const u32 m = op.m();
    const size_t tot = size_t(m) * R;
    op.apply(p, R, q, st);
    int h = d.begin(GpuAbsorber::P_VECTOR, st);
    k_pq_gamma<T><<<GRID_V, THREADS, 0, st>>>(p, q, m, R, d.cta.p, cg, lp);
    k_update_xr_sum<T><<<GRID_V, THREADS, 0, st>>>(x, r, p, q, rhs_true, x0, m, R, d.cta.p, cg, lp);
    d.launches += 2;
    d.end(h, st);
    op.precond(r, z, R, st);
    h = d.begin(GpuAbsorber::P_VECTOR, st);
    k_rz_stop<T><<<GRID_V, THREADS, 0, st>>>(r, z, m, R, d.cta.p, cg, lp, PROBE_FROM, PROBE_AT);
    k_update_p_cond<T><<<grid_for(tot), THREADS, 0, st>>>(p, z, cg.beta, cg.active, m, R, lp, cond, use_cond ? 1 : 0);
    d.launches += 2;
    d.end(h, st);
    CK(cudaGetLastError());
}

// The graph of one iteration body under a WHILE node, captured on `st` (the body kernels with
// their current arguments).
template <class T, class Op>
Scratch::PcgGraph capture_iteration(Scratch& d, const Op& op, T* x, const T* rhs_true, const T* x0, T* r, T* z, T* p,
                                    T* q, int R, const CgState& cg, const CgLoop& lp, cudaStream_t st,
                                    std::vector<u64> key) {
    const auto t0 = std::chrono::steady_clock::now();
    Scratch::PcgGraph gr;
    gr.key = std::move(key);
    CK(cudaGraphCreate(&gr.g, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, gr.g, 0, cudaGraphCondAssignDefault));
    // a first node sets the condition from the active count and the launch's cap, so that a launch
    // with no active column runs no iteration (the host need not look before launching)
    CK(cudaStreamBeginCaptureToGraph(st, gr.g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    k_cond_first<<<1, 32, 0, st>>>(cond, cg.n_active, lp);
    CK(cudaStreamEndCapture(st, &gr.g));
    cudaGraphNode_t first = nullptr;
    size_t nn = 1;
    CK(cudaGraphGetNodes(gr.g, &first, &nn));
    if (nn != 1) throw Error(RC_INTERNAL, "fereg: the PCG graph's first node");
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, gr.g, &first, 1, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    const u64 launches0 = d.launches;
    CK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    enqueue_iteration<T>(d, op, x, rhs_true, x0, r, z, p, q, R, cg, lp, cond, true, st);
    CK(cudaStreamEndCapture(st, &body));
    gr.body_launches = d.launches - launches0;
    d.launches = launches0;  // counted when the graph runs
    CK(cudaGraphInstantiate(&gr.exec, gr.g, 0));
    d.graph_captures++;
    d.graph_build_us += std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    return gr;
}

// One PCG run (cg.rs:132-292) on the m x R system S d = b in precision T, from d = 0 unless
// `x_is_start` (then d holds the start and b - S d is formed first). The stopping rule tests the
// FP64 quantities of the full iterate x0 + d: ss_k = ss1 - (x0'rhs + d'rhs + x0'r + d'r), with
// x0'rhs in cg_xconst and x0 (as T) in `x0` (null when d is the whole iterate). With `drop` > 0
// a column also stops (state 2: another refinement round) once its preconditioned residual fell
// by that factor. Returns the iterations run.
// At PROBE_AT iterations after the start (and after a restart) the contraction
// rhohat = (rho_12 / rho_7)^(1/5) of the slowest active column is measured (cg.rs:24-37,
// 254-279); above PROBE_RATIO the system escalates (when `escalate` can) and PCG restarts from
// the current x.
// The iterations run on the device: without phase timing, as launches of a captured graph whose
// WHILE node repeats the body until every column stopped or the launch's cap is reached (the
// host looks at the loop state only between launches: at the probe, at the cap, at the end);
// with phase timing, one body at a time with the host reading the state after each.
template <class T, class Op>
static u64 run_pcg(Scratch& d, const Op& op, T* x, const T* b, const T* rhs_true, const T* x0, T* r, T* z, T* p, T* q,
                   int R, double tol, double drop, u64 iters_done, size_t maxiter, bool x_is_start, const Ctx& ctx,
                   cudaStream_t st, const std::function<bool(double)>& escalate) {
    const size_t m = op.m(), tot = m * size_t(R);
    CgState cg = d.cg();
    d.lp_ctl.alloc(4);
    d.lp_ticket.alloc(4);
    d.lp_rho_from.alloc(size_t(R));
    d.lp_rho_at.alloc(size_t(R));
    d.lp_act.alloc(size_t(R));
    d.lp_tol.alloc(1);
    CK(cudaMemsetAsync(d.lp_ticket.p, 0, 4 * sizeof(unsigned), st));
    std::memcpy(d.h_nactive + 6, &tol, sizeof(double));  // pinned words 6-7
    CK(cudaMemcpyAsync(d.lp_tol.p, d.h_nactive + 6, sizeof(double), cudaMemcpyHostToDevice, st));
    const CgLoop lp{d.lp_ctl.p, d.lp_tol.p, d.lp_ticket.p, d.lp_rho_from.p, d.lp_rho_at.p, d.lp_act.p};
    u64 it = 0;
    std::vector<double> rho_from(R), rho_at(R);
    std::vector<int> act(R);
    int* hc = d.h_nactive;  // pinned [n_active, k, k of the launch, cap]
restart:
    if (x_is_start) {
        op.apply(x, R, q, st);
        k_sub<T><<<grid_for(tot), THREADS, 0, st>>>(r, b, q, tot);
        d.launches++;
    } else {
        CK(cudaMemcpyAsync(r, b, tot * sizeof(T), cudaMemcpyDeviceToDevice, st));
    }
    op.precond(r, z, R, st);
    int h = d.begin(GpuAbsorber::P_VECTOR, st);
    k_dot<T><<<GRID_V, THREADS, 0, st>>>(r, z, u32(m), R, d.cta.p);
    reduce_cols(d, d.cta.p, GRID_V, R, d.cg_rho.p, st);
    k_cg_start<<<1, THREADS, 0, st>>>(cg, R, drop);
    k_mask_copy<T><<<grid_for(tot), THREADS, 0, st>>>(p, z, d.cg_active.p, tot, R);
    d.launches += 3;
    CK(cudaMemsetAsync(d.lp_ctl.p, 0, 4 * sizeof(int), st));  // k = 0 since the (re)start
    CK(cudaMemcpyAsync(hc, d.cg_nactive.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    d.end(h, st);
    // with the body's graph captured already, the graph's first node decides whether the first
    // launch runs an iteration: the host launches it without reading the active count first
    bool look = d.prof || maxiter <= iters_done + it;
    if (!look) {
        op.prepare(R);
        const std::vector<u64> key0 = body_key<T>(d, op, x, rhs_true, x0, r, z, p, q, R);
        look = true;
        for (auto& q_ : d.graphs)
            if (q_.key == key0) look = false;
    }
    if (look) CK(cudaStreamSynchronize(st));
    bool any_active = look ? hc[0] > 0 : true;
    int k = 0;
    bool probed = false;
    while (any_active) {
        ctx.check();
        // iterations this launch may run: up to the probe, the cap and maxiter
        long long cap = GRAPH_CAP;
        if (escalate && !probed && k < PROBE_AT) cap = std::min<long long>(cap, PROBE_AT - k);
        const long long left = (long long)maxiter - (long long)(iters_done + it);
        if (left <= 0) {
            std::ostringstream os;
            os << "convergence not achieved in " << maxiter << " iterations";
            throw Error(RC_CONVERGENCE, os.str());
        }
        cap = std::min(cap, left);
        if (d.prof) cap = 1;  // phase timing: one body per launch, timed by events
        hc[4] = 0;
        hc[5] = int(cap);
        CK(cudaMemcpyAsync(d.lp_ctl.p + 2, hc + 4, 2 * sizeof(int), cudaMemcpyHostToDevice, st));
        const Scratch::PcgGraph* gr = nullptr;
        if (!d.prof) {
            op.prepare(R);
            std::vector<u64> key = body_key<T>(d, op, x, rhs_true, x0, r, z, p, q, R);
            for (auto& q_ : d.graphs)
                if (q_.key == key) gr = &q_;
            if (!gr) {
                // a new body: this batch runs one iteration by launches (first uses of its kernels
                // set their attributes), and the body is captured for the next batches
                enqueue_iteration<T>(d, op, x, rhs_true, x0, r, z, p, q, R, cg, lp, 0, false, st);
                if (d.graphs.size() >= 8) d.drop_graphs();
                d.graphs.push_back(capture_iteration<T>(d, op, x, rhs_true, x0, r, z, p, q, R, cg, lp, st, std::move(key)));
            } else {
                CK(cudaGraphLaunch(gr->exec, st));
                d.graph_launches++;
            }
        } else {
            enqueue_iteration<T>(d, op, x, rhs_true, x0, r, z, p, q, R, cg, lp, 0, false, st);
        }
        CK(cudaMemcpyAsync(hc, d.lp_ctl.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        const int ran_now = hc[2];
        it += u64(ran_now);
        if (gr) d.launches += u64(ran_now) * gr->body_launches;
        k = hc[1];
        any_active = hc[0] > 0;
        if (escalate && any_active && !probed && k >= PROBE_AT) {
            probed = true;
            CK(cudaMemcpyAsync(rho_from.data(), d.lp_rho_from.p, R * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(rho_at.data(), d.lp_rho_at.p, R * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(act.data(), d.lp_act.p, R * sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            double rho_hat = 0.0;
            for (int j = 0; j < R; j++)
                if (act[j] == 1 && rho_from[j] > 0.0)
                    rho_hat = std::max(rho_hat, std::pow(rho_at[j] / rho_from[j], 1.0 / double(PROBE_AT - PROBE_FROM)));
            if (rho_hat > PROBE_RATIO && escalate(rho_hat)) {
                CK(cudaMemsetAsync(d.cg_ring.p, 0, size_t(R) * WINDOW * sizeof(double), st));
                x_is_start = true;
                goto restart;
            }
        }
    }
    return it;
}

// solve.rs:1141-1311 residualize.
SolveInfo GpuAbsorber::solve(double* rows, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                             double* coefs, Precision prec, bool warm_last) {
    SolveInfo info;
    const size_t m = hs_.m, g1 = hs_.g1;
    if (r == 0) {
        wait_write_fence(stream_);
        info.iterations = 1;
        info.exact = true;
        return info;
    }
    ctx_.check();
    ensure_precond();
    // the closed form x + M^-1 (rhs - S x) needs the current factor, not a stale one
    if (small_stale_ && small_ok_ && hs_.m_small == hs_.m) refresh_small();
    const int R = int(r);
    // the PCG runs on padded vectors: row stride rv (a multiple of 4), columns r..rv-1 zero and
    // inactive; the rows' passes keep r
    const size_t rv = (r + 3) / 4 * 4;
    const int RV = int(rv);
    const DevStruct S = d_->ds(hs_);
    const DevWeights W = d_->dw();
    cudaStream_t st = stream_;
    Scratch& d = *d_;
    const size_t nparts = std::max<size_t>(1, size_t(std::max(S.seg.nparts, S.pull.nparts)));
    d.rhs.alloc(std::max<size_t>(1, m * r));
    d.rhsv.alloc(std::max<size_t>(1, m * rv));
    d.xv.alloc(std::max<size_t>(1, m * rv));
    d.b1.alloc(g1 * r);
    d.coefs.alloc((m + g1) * r);
    d.part.alloc(nparts * rv);
    d.cta.alloc(size_t(std::max(GRID_T, GRID_V)) * 3 * rv);
    d.colsum.alloc(3 * r);
    d.t.alloc(g1 * rv);
    d.cta2.alloc(size_t(GRID_S) * 2 * r);
    d.small.alloc(std::max<size_t>(1, small_rows() * d.ms_acc * rv));
    launch_rhs(d, S, W, rows, R, d.b1.p, d.rhs.p, d.colsum.p, st);
    ctx_.check();
    // ss0 and ss1 (solve.rs:1210-1217) and the PCG's start state on the device from the column sums;
    // the host reads ss0 back only where it needs it (an explicit warm start; the exactness test
    // after the PCG, whose launches synchronize the stream), with no round trip here
    std::vector<double> ss0(rv, 0.0);
    if (m > 0) {
        for (auto* b : {&d.cg_ss0, &d.cg_ss1, &d.cg_floor, &d.cg_xconst}) b->alloc(rv);
        d.cg_active.alloc(rv);
        k_ss_prep<<<grid_for(rv), THREADS, 0, st>>>(d.colsum.p, R, RV, sw_, d.cg_ss0.p, d.cg_ss1.p, d.cg_active.p,
                                                    d.cg_floor.p, d.cg_xconst.p);
        d.launches++;
        if (d.h_ss0_n < rv) {
            if (d.h_ss0) CK(cudaFreeHost(d.h_ss0));
            d.h_ss0 = nullptr;
            d.h_ss0_n = 0;
            CK(cudaHostAlloc(&d.h_ss0, rv * sizeof(double), cudaHostAllocDefault));
            d.h_ss0_n = rv;
        }
        CK(cudaMemcpyAsync(d.h_ss0, d.cg_ss0.p, rv * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    auto read_ss0 = [&]() {  // once the stream has passed the copy above
        if (m > 0) std::copy(d.h_ss0, d.h_ss0 + rv, ss0.begin());
    };
    // the padded right-hand side
    if (m > 0) {
        CK(cudaMemsetAsync(d.rhsv.p, 0, m * rv * 8, st));
        CK(cudaMemcpy2DAsync(d.rhsv.p, rv * 8, d.rhs.p, r * 8, r * 8, m, cudaMemcpyDeviceToDevice, st));
    }
    double* x = d.xv.p;  // the padded iterate
    const bool have_last = warm_last && last_r_ == r && m > 0;
    if (have_last) {  // the previous solution, already in place; zero the columns with ss0 = 0
        k_zero_ss0<<<grid_for(m * rv), THREADS, 0, st>>>(x, d.cg_ss0.p, m * rv, RV, R);
        d.launches++;
    } else if (warm) {
        CK(cudaStreamSynchronize(st));
        read_ss0();
        std::vector<double> w0(warm, warm + m * r);
        for (size_t j = 0; j < r; j++)
            if (ss0[j] == 0.0)
                for (size_t i = 0; i < m; i++) w0[i * r + j] = 0.0;
        if (m > 0) {
            CK(cudaMemsetAsync(x, 0, m * rv * 8, st));
            CK(cudaMemcpy2DAsync(x, rv * 8, w0.data(), r * 8, r * 8, m, cudaMemcpyHostToDevice, st));
        }
    } else if (m > 0) {
        CK(cudaMemsetAsync(x, 0, m * rv * 8, st));
    }
    u64 iterations = 1;
    bool exact = true;
    if (m > 0) {
        const size_t tot = m * rv;
        d.r.alloc(tot);
        d.z.alloc(tot);
        d.p.alloc(tot);
        d.q.alloc(tot);
        for (auto* b : {&d.cg_rho, &d.cg_rho_new, &d.cg_pq, &d.cg_gamma, &d.cg_beta, &d.cg_ss1, &d.cg_floor, &d.cg_xconst,
                        &d.cg_pfloor})
            b->alloc(rv);
        d.cg_xb.alloc(3 * rv);
        d.cg_ring.alloc(rv * WINDOW);
        d.cg_nactive.alloc(1);
        std::vector<int> act(rv);
        CK(cudaMemsetAsync(d.cg_ring.p, 0, rv * WINDOW * 8, st));
        const bool exact_pre = small_ok_ && hs_.m_small == hs_.m;
        const std::function<bool(double)> esc = [this](double rho_hat) { return escalate(rho_hat); };
        const FeOp<double> op64{d, S, W, small_ok_, d.t.p, d.part.p, d.small.p};
        if (exact_pre) {
            // x* = x + M^-1 (rhs - S x) (cg.rs:171-198)
            if (warm || have_last) {
                launch_apply<double>(d, S, W, x, RV, d.q.p, d.t.p, d.part.p, d.small.p, st);
                k_sub<double><<<grid_for(tot), THREADS, 0, st>>>(d.r.p, d.rhsv.p, d.q.p, tot);
                d.launches++;
            } else {
                CK(cudaMemcpyAsync(d.r.p, d.rhsv.p, tot * 8, cudaMemcpyDeviceToDevice, st));
            }
            launch_precond<double>(d, S, small_ok_, d.r.p, d.z.p, RV, st);
            k_add_active<double><<<grid_for(tot), THREADS, 0, st>>>(x, d.z.p, d.cg_active.p, tot, RV);
            d.launches++;
            CK(cudaGetLastError());
        } else if (prec == Precision::F64) {
            if (ctx_.autotune) autotune_apply<double>(d, S, W, d.rhsv.p, RV, d.q.p, d.t.p, d.part.p, d.small.p, st);
            iterations = run_pcg<double>(d, op64, x, d.rhsv.p, d.rhsv.p, nullptr, d.r.p, d.z.p, d.p.p, d.q.p, RV, tol,
                                         0.0, 0, maxiter, warm != nullptr || have_last, ctx_, st, esc);
            exact = false;
        } else {
            // FP32 inner PCG on the correction, FP64 true residual between rounds.
            for (auto* b : {&d.fx, &d.fb, &d.fr, &d.fz, &d.fp, &d.fq, &d.frhs, &d.fx0}) b->alloc(tot);
            d.ft.alloc(g1 * rv);
            d.fpart.alloc(nparts * rv);
            d.fsmall.alloc(std::max<size_t>(1, small_rows() * d.ms_acc * rv));
            k_convert<double, float><<<grid_for(tot), THREADS, 0, st>>>(d.rhsv.p, d.frhs.p, tot);
            d.launches++;
            if (ctx_.autotune) autotune_apply<float>(d, S, W, d.frhs.p, RV, d.fq.p, d.ft.p, d.fpart.p, d.fsmall.p, st);
            if (ctx_.autotune) autotune_apply<double>(d, S, W, d.rhsv.p, RV, d.q.p, d.t.p, d.part.p, d.small.p, st);
            iterations = 0;
            std::vector<double> rho64(rv, 0.0), rho_prev(rv, 0.0);
            bool have_r = false;  // d.r holds the FP64 true residual of x
            const bool start_nonzero = warm != nullptr || have_last;
            bool accepted = false;
            for (int round = 0; round < REFINE_ROUNDS && !accepted; round++) {
                // true residual b = rhs - S x in FP64 (kept from the previous round's check), x'rhs,
                // and the FP32 copies
                if (!have_r && start_nonzero) {
                    launch_apply<double>(d, S, W, x, RV, d.q.p, d.t.p, d.part.p, d.small.p, st);
                    k_sub<double><<<grid_for(tot), THREADS, 0, st>>>(d.r.p, d.rhsv.p, d.q.p, tot);
                    d.launches++;
                } else if (!have_r) {
                    CK(cudaMemcpyAsync(d.r.p, d.rhsv.p, tot * 8, cudaMemcpyDeviceToDevice, st));
                }
                k_dot<double><<<GRID_V, THREADS, 0, st>>>(x, d.rhsv.p, u32(m), RV, d.cta.p);
                reduce_cols(d, d.cta.p, GRID_V, RV, d.cg_xconst.p, st);
                k_convert<double, float><<<grid_for(tot), THREADS, 0, st>>>(d.r.p, d.fb.p, tot);
                k_convert<double, float><<<grid_for(tot), THREADS, 0, st>>>(x, d.fx0.p, tot);
                CK(cudaMemsetAsync(d.fx.p, 0, tot * 4, st));
                CK(cudaMemsetAsync(d.cg_ring.p, 0, rv * WINDOW * 8, st));
                d.launches += 3;
                const FeOp<float> op32{d, S, W, small_ok_, d.ft.p, d.fpart.p, d.fsmall.p};
                iterations += run_pcg<float>(d, op32, d.fx.p, d.fb.p, d.frhs.p, d.fx0.p, d.fr.p, d.fz.p, d.fp.p, d.fq.p,
                                             RV, tol, REFINE_DROP, iterations, maxiter, false, ctx_, st, esc);
                k_add_correction<<<grid_for(tot), THREADS, 0, st>>>(x, d.fx.p, tot);
                d.launches++;
                // the round's check in FP64: true residual, its preconditioned norm and ss_k
                launch_apply<double>(d, S, W, x, RV, d.q.p, d.t.p, d.part.p, d.small.p, st);
                k_sub<double><<<grid_for(tot), THREADS, 0, st>>>(d.r.p, d.rhsv.p, d.q.p, tot);
                launch_precond<double>(d, S, small_ok_, d.r.p, d.z.p, RV, st);
                k_dot<double><<<GRID_V, THREADS, 0, st>>>(d.r.p, d.z.p, u32(m), RV, d.cta.p);
                reduce_cols(d, d.cta.p, GRID_V, RV, d.cg_rho.p, st);
                k_dot<double><<<GRID_V, THREADS, 0, st>>>(x, d.rhsv.p, u32(m), RV, d.cta.p);
                reduce_cols(d, d.cta.p, GRID_V, RV, d.cg_xconst.p, st);
                k_dot<double><<<GRID_V, THREADS, 0, st>>>(x, d.r.p, u32(m), RV, d.cta.p);
                reduce_cols(d, d.cta.p, GRID_V, RV, d.cg_pq.p, st);
                k_refine_accept<<<1, THREADS, 0, st>>>(d.cg(), RV, tol);
                d.launches += 5;
                have_r = true;
                CK(cudaMemcpyAsync(d.h_nactive, d.cg_nactive.p, sizeof(int), cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(rho64.data(), d.cg_rho.p, rv * sizeof(double), cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(act.data(), d.cg_active.p, rv * sizeof(int), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                accepted = d.h_nactive[0] == 0;
                // a round that cut no remaining column's FP64 residual norm tenfold is at the limit
                // of FP32 (on an ill-conditioned graph S P of smooth vectors cancels below FP32
                // precision): the remaining columns finish in FP64
                bool progress = round == 0;
                for (size_t j = 0; j < rv && !progress; j++)
                    progress = act[j] == 1 && rho64[j] <= 0.1 * rho_prev[j];
                rho_prev = rho64;
                if (!accepted && !progress) break;
            }
            if (!accepted) {
                // FP64 PCG from the refined iterate on the columns not yet accepted, under the
                // reference's stopping rule on the full iterate (x0 = 0, x'rhs in the rule)
                CK(cudaMemsetAsync(d.cg_xconst.p, 0, rv * 8, st));
                CK(cudaMemsetAsync(d.cg_ring.p, 0, rv * WINDOW * 8, st));
                iterations += run_pcg<double>(d, op64, x, d.rhsv.p, d.rhsv.p, nullptr, d.r.p, d.z.p, d.p.p, d.q.p, RV,
                                              tol, 0.0, iterations, maxiter, true, ctx_, st, esc);
                d.fp64_finishes++;
            }
            iterations = std::max<u64>(iterations, 1);
            exact = false;
        }
        if (!exact) {
            read_ss0();
            bool all0 = true;
            for (double s : ss0) all0 &= s == 0.0;
            exact = all0;
        }
    }
    // the unpadded solution [x; .] for the residualization and the caller
    if (m > 0) CK(cudaMemcpy2DAsync(d.coefs.p, r * 8, d.xv.p, rv * 8, r * 8, m, cudaMemcpyDeviceToDevice, st));
    x = d.coefs.p;
    ctx_.check();
    wait_write_fence(st);
    int h = d.begin(P_RESID, st);
    double* alpha = want_coefs ? x + m * r : nullptr;
    if (d.wseg.n && !S.cell_row && R <= FR_MAXR) {  // one row per cell, narrow rows: pipelined tiles
        const size_t shm = FR_WPB * fresid_bytes(R);
        auto run = [&](auto ne) {
            constexpr int NE = decltype(ne)::value;
            with_nbk<1, 0>(S.nb, [&](auto, auto nbk) {
                constexpr int NBK = decltype(nbk)::value;
                allow_smem(k_fresid<NBK, NE>, shm);
                const int per_sm = resident_ctas(k_fresid<NBK, NE>, FR_WPB * 32, shm);  // shared memory bounds it
                const int grid = 148 * std::max(1, std::min(per_sm, 5));
                k_fresid<NBK, NE><<<grid, FR_WPB * 32, shm, st>>>(S, W, d.wseg.set(), rows, R, x, d.b1.p, alpha);
            });
        };
        using std::integral_constant;
        switch ((R + 3) / 4) {  // a tile holds at most WT R elements: R per lane
            case 1: run(integral_constant<int, 4>{}); break;
            case 2: run(integral_constant<int, 8>{}); break;
            case 3: run(integral_constant<int, 12>{}); break;
            default: run(integral_constant<int, 16>{}); break;
        }
        d.launches++;
    }
    else if (d.wseg.n)
        for (int j0 = 0; j0 < R; j0 += WCOLS) {
            const int Rc = std::min(WCOLS, R - j0);
            const size_t shm = wresid_smem(Rc);
            with_rcp<0>(Rc, S.nb, [&](auto c, auto nbk) {
                constexpr int RCP = decltype(c)::value, NBK = decltype(nbk)::value;
                allow_smem(k_wresid<RCP, NBK>, shm);
                k_wresid<RCP, NBK><<<GRID_S, WPB * 32, shm, st>>>(S, W, d.wseg.set(), rows, R, j0, Rc, x, d.b1.p,
                                                                   alpha);
            });
            d.launches++;
        }
    if (S.seg.nfix) {
        d.along.alloc(size_t(S.seg.nfix) * r);
        k_seg_apply<double><<<GRID_T, THREADS, 0, st>>>(S, W, x, R, d.t.p, d.part.p, true, nullptr);
        k_fix_alpha<<<std::min<u32>(S.seg.nfix, GRID_T), THREADS, 0, st>>>(S.seg, W, d.part.p, d.b1.p, R, d.along.p, alpha);
        d.launches += 2;
    }
    if (S.seg.n) {
        k_residualize<<<GRID_T, THREADS, 0, st>>>(S, W, rows, R, x, d.b1.p, d.along.p, alpha);
        d.launches++;
    }
    d.end(h, st);
    CK(cudaGetLastError());
    if (want_coefs && coefs) CK(cudaMemcpyAsync(coefs, x, (m + g1) * r * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    last_r_ = r;
    d.collect();
    info.iterations = iterations;
    info.exact = exact;
    info.escalated = !d.amg.empty();
    return info;
}

void GpuAbsorber::set_profiling(bool on) {
    AllocScope alloc_scope(stream_);
    d_->prof = on;
    if (on) {
        std::fill(d_->ms, d_->ms + P_NSLOTS, 0.0);
        std::fill(d_->cnt, d_->cnt + P_NSLOTS, u64(0));
    }
}

void GpuAbsorber::phase_times(double* ms, u64* counts) const {
    for (int i = 0; i < P_NSLOTS; i++) {
        if (ms) ms[i] = d_->ms[i];
        if (counts) counts[i] = d_->cnt[i];
    }
}

u64 GpuAbsorber::launches() const { return d_->launches; }

void GpuAbsorber::fe_leverage_device(double* h_dev) {
    AllocScope alloc_scope(stream_);
    ensure_precond();
    if (small_stale_ && small_ok_ && hs_.m_small == hs_.m) refresh_small();  // the current weights' factor
    if (hs_.m > 0 && !(small_ok_ && hs_.m_small == hs_.m))
        throw Error(RC_INVALID_INPUT,
                    "fereg: the exact FE leverage (HC2/HC3) needs a reduced system of at most 1024 coordinates");
    const DevStruct S = d_->ds(hs_);
    k_fe_leverage<<<std::max(1u, std::min<u32>((hs_.g1 + 127) / 128, 148 * 8)), 128, 0, stream_>>>(
        S, d_->dw(), hs_.m ? d_->minv.p : nullptr, h_dev);
    d_->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
}

void GpuAbsorber::solver_stats(u64* o) const {
    o[0] = d_->graph_captures;
    o[1] = d_->graph_launches;
    o[2] = u64(d_->graph_build_us);
    o[3] = d_->fp64_finishes;
}

void GpuAbsorber::fit_rows(const double* coefs, size_t r, size_t col, double* out) const {
    AllocScope alloc_scope(stream_);
    ensure_host_coord();
    const HostStructure& st = hs_;
    const size_t m = st.m, M = st.ncells, nb = st.nb();
    for (u32 s = 0; s < st.g1; s++)
        for (u32 c = st.seg_off[s]; c < st.seg_off[s + 1]; c++) {
            double f = coefs[(m + s) * r + col];
            for (size_t b = 0; b < nb; b++) f += coefs[size_t(st.coord[b * M + c]) * r + col];
            const u32 r0 = st.trivial() ? c : st.cell_row[c], r1 = st.trivial() ? c + 1 : st.cell_row[c + 1];
            for (u32 row = r0; row < r1; row++) out[row] = f;
        }
}

size_t GpuAbsorber::term_values_len() const {
    size_t t = 0;
    for (u32 v : g_) t += v;
    return t;
}

void GpuAbsorber::term_values(const double* coefs, size_t r, size_t col, double* out) const {
    AllocScope alloc_scope(stream_);
    sync_host_weights();
    const HostStructure& st = hs_;
    const size_t nterms = g_.size();
    if (st.fe1 < 0 || norm_fe1_ < 0) return;
    std::vector<std::vector<double>> vals(nterms), lw(nterms);
    vals[size_t(st.fe1)].resize(st.g1);
    for (size_t s = 0; s < st.g1; s++) vals[size_t(st.fe1)][s] = coefs[(st.m + s) * r + col];
    lw[size_t(st.fe1)] = n1_;
    for (auto& b : st.blocks) {
        vals[b.term].resize(b.g);
        lw[b.term].resize(b.g);
        for (size_t l = 0; l < b.g; l++) {
            vals[b.term][l] = coefs[(b.off + l) * r + col];
            lw[b.term][l] = nr_[b.off + l];
        }
    }
    double shift = 0;
    for (size_t t = 0; t < nterms; t++) {
        if (int(t) == norm_fe1_) continue;
        double mean = 0;
        for (size_t l = 0; l < vals[t].size(); l++) mean += vals[t][l] * lw[t][l];
        mean /= sw_;
        for (auto& v : vals[t]) v -= mean;
        shift += mean;
    }
    for (auto& v : vals[size_t(norm_fe1_)]) v += shift;
    size_t o = 0;
    for (size_t t = 0; t < nterms; t++) {
        std::copy(vals[t].begin(), vals[t].end(), out + o);
        o += g_[t];
    }
}

// The operator of a PcgDriver run, seen by the templated loop.
struct VirtOp {
    DevOperator& o;
    u32 m() const { return o.m(); }
    void apply(double* p, int R, double* q, cudaStream_t st) const { o.apply(p, R, q, st); }
    void precond(double* r, double* z, int R, cudaStream_t st) const { o.precond(r, z, R, st); }
    void key(std::vector<u64>& k) const { o.key(k); }
    void prepare(int) const {}
};

PcgDriver::PcgDriver() : d_(std::make_unique<Scratch>()) {
    CK(cudaHostAlloc(&d_->h_nactive, 8 * sizeof(int), cudaHostAllocDefault));
}
PcgDriver::~PcgDriver() = default;

u64 PcgDriver::run(DevOperator& op, double* x, const double* b, int R, const std::vector<double>& ss0,
                   const std::vector<double>& ss1, double tol, size_t maxiter, bool x_is_start, const Ctx& ctx,
                   cudaStream_t st) {
    Scratch& d = *d_;
    const size_t m = op.m(), rv = size_t(R);
    if (R % 4 != 0 || ss0.size() != rv || ss1.size() != rv) throw Error(RC_INTERNAL, "fereg: PCG driver shapes");
    if (m == 0) return 0;
    const size_t tot = m * rv;
    d.r.alloc(tot);
    d.z.alloc(tot);
    d.p.alloc(tot);
    d.q.alloc(tot);
    d.cta.alloc(size_t(std::max(GRID_T, GRID_V)) * 3 * rv);
    for (auto* buf : {&d.cg_rho, &d.cg_rho_new, &d.cg_pq, &d.cg_gamma, &d.cg_beta, &d.cg_ss1, &d.cg_floor, &d.cg_xconst,
                      &d.cg_pfloor})
        buf->alloc(rv);
    d.cg_xb.alloc(3 * rv);
    d.cg_ring.alloc(rv * WINDOW);
    d.cg_active.alloc(rv);
    d.cg_nactive.alloc(1);
    std::vector<int> act(rv);
    std::vector<double> fl(rv);
    for (size_t j = 0; j < rv; j++) {
        act[j] = ss0[j] > 0.0;
        fl[j] = 1e-26 * ss0[j];
    }
    CK(cudaMemcpyAsync(d.cg_active.p, act.data(), rv * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d.cg_ss1.p, ss1.data(), rv * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d.cg_floor.p, fl.data(), rv * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d.cg_xconst.p, 0, rv * 8, st));
    CK(cudaMemsetAsync(d.cg_pfloor.p, 0, rv * 8, st));
    CK(cudaMemsetAsync(d.cg_ring.p, 0, rv * WINDOW * 8, st));
    const VirtOp vo{op};
    const u64 it = run_pcg<double>(d, vo, x, b, b, nullptr, d.r.p, d.z.p, d.p.p, d.q.p, R, tol, 0.0, 0, maxiter,
                                   x_is_start, ctx, st, std::function<bool(double)>());
    CK(cudaStreamSynchronize(st));  // the host vectors above stay alive until the copies ran
    return it;
}

void PcgDriver::col_sums(const double* part, int nparts, int ncols, double* out, cudaStream_t st) {
    reduce_cols(*d_, part, nparts, ncols, out, st);
}

u64 PcgDriver::launches() const { return d_->launches; }

void PcgDriver::stats(u64* o) const {
    o[0] = d_->graph_captures;
    o[1] = d_->graph_launches;
    o[2] = u64(d_->graph_build_us);
    o[3] = 0;
}

}  // namespace fereg
