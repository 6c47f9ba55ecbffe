// Shared host-side definitions of the B200 fixed-effects solver.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace fereg {

using u32 = uint32_t;
using u64 = uint64_t;

// Return codes of the C ABI: the reference's `RfError::rc` (error.rs:24-34), so a Stata or Rust
// caller maps them without a table.
enum Rc : int {
    RC_OK = 0,
    RC_INTERRUPTED = 1,
    RC_INVALID_INPUT = 198,
    RC_CONVERGENCE = 430,
    RC_NOT_IDENTIFIED = 481,
    RC_OUT_OF_MEMORY = 909,
    RC_TOO_FEW_OBS = 2001,
    RC_INTERNAL = 9999,
};

// An error carrying its return code; caught at the C ABI and never crossing it.
struct Error : std::runtime_error {
    int rc;
    Error(int rc_, const std::string& msg) : std::runtime_error(msg), rc(rc_) {}
};

void set_last_error(const std::string& msg);
const char* last_error();

// One non-eliminated term: a block of the reduced system (structure.rs:27-37).
struct Block {
    u32 term;   // session term index
    u32 g;      // levels
    u32 off;    // offset of level 0 in the reduced coordinates
    bool small; // in the dense small super-block
};

// Host form of the cell structure (structure.rs:55-92): rows sorted by (FE1, block codes, obs),
// cells = runs of equal code tuples, segments = the cells of one FE1 level.
struct HostStructure {
    size_t n = 0;
    int fe1 = -1;                 // eliminated term (-1: no absorb terms, one synthetic level)
    u32 g1 = 1;
    std::vector<u32> pi;          // kept observation of each row
    std::vector<u32> seg_off;     // g1 + 1
    std::vector<u32> cell_row;    // M + 1 first rows (empty when every cell holds one row)
    size_t ncells = 0;
    std::vector<Block> blocks;
    std::vector<u32> coord;       // nb x M, block-major: global reduced coordinate of each cell
    size_t m = 0, m_small = 0;
    u64 small_work = 0;
    size_t nb() const { return blocks.size(); }
    bool trivial() const { return cell_row.empty(); }
};

// structure.rs:23 SMALL_LIMIT.
constexpr size_t SMALL_LIMIT = 4096;

// The eliminated term, the blocks and their coordinate offsets (structure.rs:247-378), without the
// per-row arrays.
HostStructure plan_structure(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n,
                             size_t small_limit);
HostStructure build_structure(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n,
                              size_t small_limit);
int fe1_index(const std::vector<u32>& g);
// Every code below its term's level count, every weight positive and finite (198 otherwise).
void check_codes_host(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n);
void check_weights_host(const double* w, size_t n);

// Coordinate-sorted cell lists of every block (the transpose of the cell structure): for each
// reduced coordinate k, the cells whose code in k's block is k, ascending. With the segment of
// each cell and the cell's coordinates in the other blocks stored beside it, a pull over these
// lists sums per-cell values by coordinate without a scatter.
struct PullTable {
    std::vector<u32> off;    // m + 1
    std::vector<u32> cell;   // E = M * nb
    std::vector<u32> seg;    // E
    std::vector<u32> other;  // E * (nb - 1), other-block coordinates (block order, k's block skipped)
};
PullTable build_pull_table(const HostStructure& st);

// Load-balanced tiles over the lists of a CSR-like array (segments -> cells, coordinates ->
// entries) longer than `min_len`: each tile covers whole consecutive lists [k0, k1) with at most
// `cap` entries, or a `cap`-sized slice of one longer list, which writes a partial sum completed
// by a fix-up in slice order.
struct TileList {
    std::vector<u32> k0, k1, e0, e1;   // per tile
    std::vector<int32_t> part;         // partial slot, -1 when the tile writes its lists
    std::vector<int32_t> fixidx;       // index of the tile's long list in fix_*, -1 otherwise
    std::vector<u32> fix_k;            // lists completed from partials
    std::vector<u32> fix_p0, fix_np;   // first partial slot and count per long list
    u32 nparts = 0;
};
TileList build_tiles(const std::vector<u32>& off, u32 k_begin, u32 k_end, u32 cap, u32 min_len);

// Warp tiles: whole consecutive lists [k0, k1) covering entries [e0, e1).
struct WarpTileList {
    std::vector<u32> k0, k1, e0, e1;
};

// Splits the lists [k_begin, k_end) of a CSR-like array by weight (`weight[k]`, or the entry
// count when null): lists of weight <= warp_max go to warp tiles, packed consecutively while the
// summed weight stays <= pack and the tile holds at most max_lists lists; the others go to CTA
// tiles of at most cta_cap entries (slices of longer lists write partials).
void split_tiles(const std::vector<u32>& off, const std::vector<u32>* weight, u32 k_begin, u32 k_end, u32 warp_max,
                 u32 pack, u32 max_lists, u32 cta_cap, WarpTileList& wt, TileList& ct);

}  // namespace fereg
