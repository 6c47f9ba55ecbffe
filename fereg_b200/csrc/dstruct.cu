// The cell structure on the device (dstruct.h; kernels in dstruct.cuh).
//
// Row order: when the rows are not already in key order, stable LSD radix sorts of the row ids by
// the block codes (last block first), then by the FE1 code, each over the bits its level count
// needs; equal keys keep observation order, as in the host build's counting sorts. Cells: a row
// opens a cell when its key differs from the previous row's (flags, exclusive scan). Coordinate
// lists: the entries of every block (cells in order, keyed by their coordinate) sorted stably by
// coordinate, so each list holds its cells in cell order.
#include "dstruct.h"

#include <algorithm>

#include "dstruct.cuh"
#include "prep.h"

namespace fereg {

namespace {

int ds_grid(size_t n) { return int(std::max<size_t>(1, std::min<size_t>((n + DS_TB - 1) / DS_TB, 148 * 16))); }

// Bits that hold every value up to v.
int bits_for(u64 v) {
    int b = 0;
    for (; v; v >>= 1) b++;
    return b;
}

__global__ void k_ds_set(u32* p, u32 v) { *p = v; }

template <class T>
void to_host(std::vector<T>& h, const T* d, size_t count, cudaStream_t st) {
    h.resize(count);
    if (count) CK(cudaMemcpyAsync(h.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost, st));
}

}  // namespace

void build_structure_device(const std::vector<const u32*>& dcodes, const std::vector<u32>& g, HostStructure& hs,
                            DeviceStructure& ds, std::vector<u32>& pl_off_host, std::vector<u32>& pl_seg_host,
                            cudaStream_t st) {
    const size_t n = hs.n, nb = hs.nb();
    const u32 g1 = hs.g1;
    DBuf<int> flag;
    flag.alloc(1);
    CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    for (size_t q = 0; q < dcodes.size(); q++)
        if (n) k_ds_check<<<ds_grid(n), DS_TB, 0, st>>>(dcodes[q], n, g[q], flag.p);
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (bad) throw Error(RC_INVALID_INPUT, "term code out of range of its level count");

    // terms in key order: FE1, then the blocks
    std::vector<const u32*> tptr;
    std::vector<u32> toff, tg;
    const int has_fe1 = hs.fe1 >= 0 ? 1 : 0;
    if (has_fe1) {
        tptr.push_back(dcodes[size_t(hs.fe1)]);
        toff.push_back(0);
        tg.push_back(g1);
    }
    for (const Block& b : hs.blocks) {
        tptr.push_back(dcodes[b.term]);
        toff.push_back(b.off);
        tg.push_back(b.g);
    }
    const int nt = int(tptr.size());
    DBuf<const u32*> dt;
    DBuf<u32> doff;
    dt.upload(tptr, st);
    doff.upload(toff, st);
    const TermCodes tc{dt.p, doff.p, nt, has_fe1};

    // row order
    ds.pi.alloc(n);
    if (n) k_ds_iota<<<ds_grid(n), DS_TB, 0, st>>>(ds.pi.p, n);
    int unsorted = 0;
    if (n > 1 && nt > 0) {
        CK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
        k_ds_unsorted<<<ds_grid(n), DS_TB, 0, st>>>(tc, n, flag.p);
        CK(cudaMemcpyAsync(&unsorted, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    if (unsorted) {
        DBuf<u64> k1, k2;
        DBuf<u32> v2;
        k1.alloc(n);
        k2.alloc(n);
        v2.alloc(n);
        u32* cur = ds.pi.p;
        u32* alt = v2.p;
        for (int q = nt - 1; q >= 0; q--) {
            k_ds_gather_key<<<ds_grid(n), DS_TB, 0, st>>>(tptr[size_t(q)], cur, n, k1.p);
            u64* keys = k1.p;
            u32* vals = cur;
            device_sort_pairs(keys, vals, k2.p, alt, n, bits_for(tg[size_t(q)] - 1), st);
            if (vals != cur) std::swap(cur, alt);
        }
        if (cur != ds.pi.p) CK(cudaMemcpyAsync(ds.pi.p, cur, n * sizeof(u32), cudaMemcpyDeviceToDevice, st));
        CK(cudaStreamSynchronize(st));  // v2 and the keys die here
    }

    // cells and segments
    DBuf<u32> flags, cell_of;
    flags.alloc(n);
    cell_of.alloc(n);
    u32 M = 0;
    if (n) {
        k_ds_cell_flags<<<ds_grid(n), DS_TB, 0, st>>>(tc, ds.pi.p, n, flags.p);
        M = device_excl_scan(flags.p, n, cell_of.p, st);
    }
    hs.ncells = M;
    const bool trivial = size_t(M) == n;
    ds.cseg.alloc(M);
    ds.coord.alloc(size_t(nb) * M);
    if (!trivial) ds.cell_row.alloc(size_t(M) + 1);
    if (n)
        k_ds_cells<<<ds_grid(n), DS_TB, 0, st>>>(tc, ds.pi.p, n, flags.p, cell_of.p, M,
                                                 trivial ? nullptr : ds.cell_row.p, ds.cseg.p, ds.coord.p);
    if (!trivial) k_ds_set<<<1, 1, 0, st>>>(ds.cell_row.p + M, u32(n));
    ds.seg_off.alloc(size_t(g1) + 1);
    k_ds_seg_off<<<ds_grid(size_t(M) + 1), DS_TB, 0, st>>>(ds.cseg.p, M, g1, ds.seg_off.p);
    CK(cudaGetLastError());
    to_host(hs.pi, ds.pi.p, n, st);
    to_host(hs.seg_off, ds.seg_off.p, size_t(g1) + 1, st);
    if (!trivial) to_host(hs.cell_row, ds.cell_row.p, size_t(M) + 1, st);
    else hs.cell_row.clear();
    hs.coord.clear();
    CK(cudaStreamSynchronize(st));

    // coordinate-sorted cell lists
    const size_t m = hs.m, E = size_t(M) * nb, no = nb > 0 ? nb - 1 : 0;
    ds.pl_off.alloc(m + 1);
    ds.pl_seg.alloc(E);
    ds.pl_other.alloc(E * no);
    hs.small_work = 0;
    if (E == 0) {
        CK(cudaMemsetAsync(ds.pl_off.p, 0, (m + 1) * sizeof(u32), st));
        ds.pl_cell.alloc(0);
        pl_off_host.assign(m + 1, 0);
        pl_seg_host.clear();
        CK(cudaStreamSynchronize(st));
        return;
    }
    DBuf<u64> ek, ek2;
    DBuf<u32> ev, ev2, cnt, boff;
    ek.alloc(E);
    ek2.alloc(E);
    ev.alloc(E);
    ev2.alloc(E);
    k_ds_entries<<<ds_grid(E), DS_TB, 0, st>>>(ds.coord.p, M, int(nb), ek.p, ev.p);
    u64* keys = ek.p;
    u32* vals = ev.p;
    device_sort_pairs(keys, vals, ek2.p, ev2.p, E, bits_for(m - 1), st);
    cnt.alloc(m + 1);
    CK(cudaMemsetAsync(cnt.p, 0, (m + 1) * sizeof(u32), st));
    k_ds_count<<<ds_grid(E), DS_TB, 0, st>>>(ds.coord.p, E, cnt.p);
    device_excl_scan(cnt.p, m + 1, ds.pl_off.p, st);
    std::vector<u32> hb(nb + 1);
    for (size_t k = 0; k < nb; k++) hb[k] = hs.blocks[k].off;
    hb[nb] = u32(m);
    boff.upload(hb, st);
    k_ds_pull_rest<<<ds_grid(E), DS_TB, 0, st>>>(keys, vals, E, ds.cseg.p, ds.coord.p, M, int(nb), boff.p, ds.pl_seg.p,
                                                 ds.pl_other.p);
    CK(cudaGetLastError());
    to_host(pl_off_host, ds.pl_off.p, m + 1, st);
    to_host(pl_seg_host, ds.pl_seg.p, E, st);
    CK(cudaStreamSynchronize(st));

    // dense small-block work sum_s d_s^2 (structure.rs:521-525)
    if (hs.m_small > 0) {
        const size_t es = pl_off_host[hs.m_small];
        DBuf<u32> d;
        DBuf<unsigned long long> tot;
        d.alloc(g1);
        tot.alloc(1);
        CK(cudaMemsetAsync(d.p, 0, size_t(g1) * sizeof(u32), st));
        CK(cudaMemsetAsync(tot.p, 0, sizeof(unsigned long long), st));
        if (es) k_ds_small_pairs<<<ds_grid(es), DS_TB, 0, st>>>(keys, ds.pl_seg.p, es, d.p);
        k_ds_sq_sum<<<ds_grid(g1), DS_TB, 0, st>>>(d.p, g1, tot.p);
        unsigned long long work = 0;
        CK(cudaMemcpyAsync(&work, tot.p, sizeof(work), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        hs.small_work = u64(work);
        if (hs.small_work > 64 * u64(M)) {
            for (auto& b : hs.blocks) b.small = false;
            hs.m_small = 0;
        }
    }
    // the sorted cells are the lists' cells
    ds.pl_cell = vals == ev.p ? std::move(ev) : std::move(ev2);
    CK(cudaStreamSynchronize(st));
}

}  // namespace fereg
