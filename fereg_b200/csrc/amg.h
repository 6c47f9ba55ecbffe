// Escalated preconditioner of a large block: an aggregation multigrid hierarchy of the block's
// exact Schur-complement Laplacian S_bb.
//
// The reference escalates a large block whose Jacobi-preconditioned PCG contracts slowly
// (cg.rs:24-37: at iteration 12, rhohat = (rho_12 / rho_7)^(1/5) > 0.6) to an exact factor of
// S_bb (operator.rs:2054 assemble_block; precond/sparse_chol.rs: AMD + supernodal LDL^T). A
// triangular solve with such a factor is a chain of dependent steps (on a ring or band firm
// graph the elimination tree is a path of ~1e5 levels), so here the escalated block gets a
// multigrid V-cycle instead: every step of it is a parallel sparse pass. The preconditioner
// changes only the iteration count, not the converged answer.
//
// S_bb (block b, g levels) is assembled from the cell structure and the weight state:
//   S_bb[k][l] = -sum_s c_{s,k} c_{s,l} / n1_s  (k != l),  S_bb[k][k] = diag_k,
// with c_{s,k} the weight of the cells of segment s whose block-b level is k (operator.rs:2054).
// Levels: smoothed aggregation. Plain aggregates (strong neighbours |a_ij| >= 0.25 max_l |a_il|,
// at most 8 nodes an aggregate) give the piecewise-constant P0; the prolongation is
// P = (I - (2/3) D^-1 A) P0 (one damped-Jacobi smoothing of P0; D^-1 A of a Laplacian has its
// spectrum in [0, 2]) and the coarse operator A_c = P^T A P, until at most AMG_COARSE nodes
// remain. P0 and P both keep the constants, so every level is again a Laplacian. The coarsest
// level is inverted densely with the grounded LDL^T of the small block (pivots below 1e-10 of the
// unit-scaled diagonal grounded, precond/dense.rs:1-38), which handles the null space.
// Redundant coordinates (operator.rs:21) are left out (their preconditioned value is 0, as under
// Jacobi). On ring and band firm graphs the smoothed hierarchy keeps PCG at ~15 iterations
// independent of size, where Jacobi needs thousands.
#pragma once

#include <vector>

#include "common.h"

namespace fereg {

constexpr u32 AMG_COARSE = 384;   // the coarsest level is dense at or below this size
constexpr double AMG_OMEGA = 0.6;  // Jacobi damping of the smoother (< 1: the V-cycle stays SPD)

// Row-major CSR.
struct Csr {
    u32 nr = 0, nc = 0;
    std::vector<u32> ptr, col;
    std::vector<double> val;
};

struct AmgLevel {
    u32 n = 0;
    Csr A;                     // the level's operator (diagonal included)
    std::vector<double> dinv;  // AMG_OMEGA / a_ii (0: left out)
    Csr P, Pt;                 // prolongation to this level from the next (n x n_c) and its transpose
};

struct AmgHierarchy {
    u32 block = 0;                 // index into HostStructure::blocks
    std::vector<AmgLevel> levels;  // levels[0] is S_bb
    std::vector<double> coarse;    // the coarsest level's matrix, dense (n x n)
    size_t nnz() const {
        size_t t = 0;
        for (auto& l : levels) t += l.A.col.size() + 2 * l.P.col.size();
        return t;
    }
};

// cell_w: cell weights (null: 1 per cell); n1: segment weights; diag, red: the coordinate
// weight state (global coordinates).
AmgHierarchy amg_build(const HostStructure& hs, size_t block, const double* cell_w, const double* n1,
                       const double* diag, const uint8_t* red);

}  // namespace fereg
