// The cell structure built on the device (structure.rs:356-527): the same arrays as the host
// build (build_structure + build_pull_table in structure.cpp), element for element.
#pragma once

#include <cuda_runtime.h>

#include "common.h"
#include "device.cuh"

namespace fereg {

// Device arrays of the structure; the host keeps the small ones it reads (see build_structure_device).
struct DeviceStructure {
    DBuf<u32> pi;        // n: kept observation of each row
    DBuf<u32> seg_off;   // g1 + 1
    DBuf<u32> coord;     // nb x M, block-major
    DBuf<u32> cell_row;  // M + 1, empty when every cell holds one row
    DBuf<u32> cseg;      // M: segment of each cell
    DBuf<u32> pl_off;    // m + 1
    DBuf<u32> pl_cell, pl_seg, pl_other;  // E, E, E x (nb - 1)
};

// Builds the structure planned in `hs` (plan_structure: FE1, the blocks and their offsets) from
// the session's term codes in device memory (dcodes[q] for term q, n rows), on `st`. Checks every
// code against its level count (198). Fills hs.ncells, hs.small_work (and the demotion of the small
// blocks, structure.rs:521-525) and the host copies hs.pi, hs.seg_off, hs.cell_row; hs.coord stays
// empty (the device holds it). pl_off_host / pl_seg_host receive the lists' offsets and segments
// for the host's tile builders.
void build_structure_device(const std::vector<const u32*>& dcodes, const std::vector<u32>& g, HostStructure& hs,
                            DeviceStructure& ds, std::vector<u32>& pl_off_host, std::vector<u32>& pl_seg_host,
                            cudaStream_t st);

}  // namespace fereg
