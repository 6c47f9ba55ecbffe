// sm_100a kernels of the fixed-effects solve.
//
// Layout in HBM (one absorber):
//   seg_off[g1+1]       cells of each FE1 level (segment), cells sorted by (FE1, codes, obs)
//   coord[nb*M]         block-major global reduced coordinate of every cell
//   cell_row[M+1]       first row of each cell (absent when every cell holds one row)
//   pl_off[m+1], pl_cell/pl_seg[E], pl_other[E*(nb-1)]
//                       coordinate-sorted cell lists (transpose of coord) with each cell's
//                       segment and other-block coordinates beside it
//   rows[n*R]           the caller's row-major column block (FP64), rows in row order
//   reduced vectors     m x R row-major
//
// Every kernel is deterministic: per-cell values are never scattered; sums by coordinate are
// pulls over the coordinate-sorted lists in list order (tiles.cuh), and column sums combine
// fixed per-CTA partials in CTA order. No floating-point atomics.
#pragma once

#include "short.cuh"

namespace fereg {

__device__ __forceinline__ int gwarp() { return int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }
__device__ __forceinline__ int nwarps() { return int((gridDim.x * blockDim.x) >> 5); }
__device__ __forceinline__ int lane_id() { return int(threadIdx.x & 31); }

// ---------------------------------------------------------------------------------------------
// PCG vector work on m x R blocks (cg.rs), column sums as per-CTA partials (gridDim x R).
template <class T>
__global__ void __launch_bounds__(TB) k_dot(const T* __restrict__ a, const T* __restrict__ b, u32 m, int R,
                                            double* __restrict__ cta_part) {
    __shared__ double red[TB];
    for (int j0 = 0; j0 < R; j0 += RC_MAX) {
        const ColMap cm = colmap(R, j0);
        double acc = 0.0;
        if (cm.on)
            for (u32 i = blockIdx.x * u32(cm.nslot) + u32(cm.slot); i < m; i += gridDim.x * u32(cm.nslot)) {
                const size_t o = size_t(i) * R + j0 + cm.col;
                acc += double(a[o]) * double(b[o]);
            }
        red[threadIdx.x] = acc;
        __syncthreads();
        if (int(threadIdx.x) < cm.Rc) {
            double s = 0.0;
            for (int sl = 0; sl < cm.nslot; sl++) s += red[sl * cm.Rc + threadIdx.x];
            cta_part[size_t(blockIdx.x) * R + j0 + threadIdx.x] = s;
        }
        __syncthreads();
    }
}

// Column sums of [nparts x ncols] partials (plus a second array when given) in a fixed order:
// one warp per column, lane l sums parts l, l+32, ..., then a fixed butterfly.
__global__ void k_reduce_cols(const double* __restrict__ part, int nparts, const double* __restrict__ part2,
                              int nparts2, int ncols, double* __restrict__ out) {
    const int lane = lane_id();
    for (int col = gwarp(); col < ncols; col += nwarps()) {
        double acc = 0.0;
        for (int p = lane; p < nparts; p += 32) acc += part[size_t(p) * ncols + col];
        if (part2)
            for (int p = lane; p < nparts2; p += 32) acc += part2[size_t(p) * ncols + col];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
        if (lane == 0) out[col] = acc;
    }
}

// Per-column PCG state (cg.rs:132-292), kept on the device. active: 1 iterating, 0 stopped by
// the reference's rules, 2 stopped at the FP32 precision floor of a refinement round.
struct CgState {
    double* rho;
    double* rho_new;
    double* pq;
    double* gamma;
    double* beta;
    double* xb;      // d'rhs, d'r, x0'r (3R)
    double* ss1;
    double* floor_;  // 1e-26 * ss0
    double* ring;    // R x WINDOW
    double* xconst;  // x0'rhs
    double* pfloor;  // precision floor of the preconditioned residual (0: none)
    int* active;
    int* n_active;
};

constexpr int WINDOW = 5;

// After rho = r'z of a (re)start: columns with rho <= 0 stop (cg.rs:201-205); the precision
// floor is drop * rho; counts the active columns. Single block.
__global__ void k_cg_start(CgState st, int R, double drop) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int local = 0;
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
        if (st.active[j] == 1 && !(st.rho[j] > 0.0)) st.active[j] = 0;
        st.pfloor[j] = drop * st.rho[j];
        local += st.active[j] == 1;
    }
    atomicAdd(&cnt, local);  // integer count: order independent
    __syncthreads();
    if (threadIdx.x == 0) *st.n_active = cnt;
}

// End of an FP32 refinement round, on the FP64 quantities of the refined iterate x: rho = r'M^-1 r
// of its true residual, xconst = x'rhs, pq = x'r. A column is accepted (state 0) only when
// rho <= max(tol^2 ss_k, floor) with ss_k = ss1 - x'(rhs + r), whether the round ended it by the
// FP32 window rule (whose recursive residual can fall below the true one) or at the FP32 floor;
// otherwise it goes another round (state 1). Columns without variation (floor 0) stay stopped.
__global__ void k_refine_accept(CgState st, int R, double tol) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int local = 0;
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
        if (st.floor_[j] > 0.0) {
            const double ssk = st.ss1[j] - (st.xconst[j] + st.pq[j]);
            const double thr = fmax(tol * tol * ssk, st.floor_[j]);
            const bool ok = st.rho[j] <= thr;
            st.active[j] = ok ? 0 : 1;
        }
        local += st.active[j] == 1;
    }
    atomicAdd(&cnt, local);  // integer count: order independent
    __syncthreads();
    if (threadIdx.x == 0) *st.n_active = cnt;
}

template <class Src, class Dst>
__global__ void k_convert(const Src* __restrict__ a, Dst* __restrict__ b, size_t total) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x)
        b[i] = Dst(a[i]);
}

// x += d (the FP32 correction of a refinement round).
__global__ void k_add_correction(double* __restrict__ x, const float* __restrict__ d, size_t total) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x)
        x[i] += double(d[i]);
}

// r = a - b
template <class T>
__global__ void k_sub(T* __restrict__ r, const T* __restrict__ a, const T* __restrict__ b, size_t total) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x)
        r[i] = a[i] - b[i];
}

// p = z masked by the active columns.
template <class T>
__global__ void k_mask_copy(T* __restrict__ p, const T* __restrict__ z, const int* __restrict__ active, size_t total, int R) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x)
        p[i] = active[i % R] == 1 ? z[i] : T(0);
}

// x = 0 on the columns whose mask is 1 (warm starts of zero columns, solve.rs:1209-1217).
__global__ void k_zero_masked(double* __restrict__ x, const int* __restrict__ mask, size_t total, int R) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x)
        if (mask[i % R]) x[i] = 0.0;
}

// The solve's column scalars from the rhs pass's column sums cs = [sum w v^2, sum w v, sum b1^2/n1]
// (solve.rs:1210-1217): ss0 = the weighted centered sum of squares (0 below 1e-15 of the sum of
// squares), ss1 = sum w v^2 - sum b1^2/n1, and the PCG's start state: active = ss0 > 0, the floor
// 1e-26 ss0, x'rhs of the start 0. Columns r..rv-1 (padding) get zeros.
__global__ void k_ss_prep(const double* __restrict__ cs, int r, int rv, double sw, double* __restrict__ ss0,
                          double* __restrict__ ss1, int* __restrict__ active, double* __restrict__ floor_,
                          double* __restrict__ xconst) {
    for (int j = int(blockIdx.x * blockDim.x + threadIdx.x); j < rv; j += int(gridDim.x * blockDim.x)) {
        double s0 = 0.0, s1 = 0.0;
        if (j < r) {
            const double wsq = cs[j], wsum = cs[r + j], b1sq = cs[2 * r + j];
            const double s = wsq - wsum * wsum / sw;
            s0 = s > 1e-15 * wsq ? s : 0.0;
            s1 = wsq - b1sq;
        }
        ss0[j] = s0;
        ss1[j] = s1;
        active[j] = s0 > 0.0;
        floor_[j] = 1e-26 * s0;
        xconst[j] = 0.0;
    }
}

// x = 0 on the columns j < r whose ss0 is 0 (a warm start of zero columns, solve.rs:1209-1217).
__global__ void k_zero_ss0(double* __restrict__ x, const double* __restrict__ ss0, size_t total, int R, int r) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int j = int(i % size_t(R));
        if (j < r && ss0[j] == 0.0) x[i] = 0.0;
    }
}

// x += z on the active columns (exact preconditioner, cg.rs:171-198).
template <class T>
__global__ void k_add_active(T* __restrict__ x, const T* __restrict__ z, const int* __restrict__ active, size_t total, int R) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x)
        if (active[i % R] == 1) x[i] += z[i];
}

// The small coordinates' rows of Y = S P from the dense rows of S (srow, weights.cuh): CTA b
// takes the coordinates f of its chunk; with at most TB (k, j) pairs the threads are (slot, pair)
// and slot s adds srow[f][k] P[f][j] over the chunk's f = s, s + slots, ... (loads unrolled),
// the slots' sums are then added in slot order into part[b][k * R + j]; with more pairs each
// thread takes pairs in turn over the whole chunk. k_small_reduce adds the CTAs' partials in CTA
// order.
template <class T>
__global__ void __launch_bounds__(TB) k_srow_apply(const double* __restrict__ srow, u32 m, u32 ms,
                                                   const T* __restrict__ P, int R, T* __restrict__ part) {
    __shared__ T red[TB];
    const u32 npairs = ms * u32(R);
    const u32 chunk = (m + gridDim.x - 1) / gridDim.x;
    const u32 f0 = min(m, blockIdx.x * chunk), f1 = min(m, f0 + chunk);
    if (npairs <= u32(TB)) {
        const u32 nslot = u32(TB) / npairs, slot = threadIdx.x / npairs, pi = threadIdx.x % npairs;
        const u32 k = pi / u32(R), j = pi % u32(R);
        T acc = T(0);
        if (slot < nslot) {
#pragma unroll 4
            for (u32 f = f0 + slot; f < f1; f += nslot) acc += T(srow[size_t(f) * ms + k]) * P[size_t(f) * R + j];
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        if (threadIdx.x < npairs) {
            T sum = T(0);
            for (u32 sl = 0; sl < nslot; sl++) sum += red[sl * npairs + threadIdx.x];
            part[size_t(blockIdx.x) * npairs + threadIdx.x] = sum;
        }
        return;
    }
    for (u32 pi = threadIdx.x; pi < npairs; pi += blockDim.x) {
        const u32 k = pi / u32(R), j = pi % u32(R);
        T acc = T(0);
#pragma unroll 4
        for (u32 f = f0; f < f1; f++) acc += T(srow[size_t(f) * ms + k]) * P[size_t(f) * R + j];
        part[size_t(blockIdx.x) * npairs + pi] = acc;
    }
}

// Jacobi on coordinates [k0, m): z = inv_diag .* r (precond/jacobi.rs:12-42).
template <class T>
__global__ void k_jacobi(const T* __restrict__ r, T* __restrict__ z, const double* __restrict__ inv_diag, u32 k0, u32 m, int R) {
    const size_t total = size_t(m - k0) * R;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const size_t o = size_t(k0) * R + i;
        z[o] = T(inv_diag[k0 + i / R]) * r[o];
    }
}

// Small super-block: z[0..ms) = Minv r[0..ms) with the expanded, scaled generalized inverse.
// z = minv r on the small coordinates (ms x R), one warp per output element: lane l adds the
// products of entries l, l + 32, ... in order, combined by a fixed butterfly.
template <class T>
__global__ void k_small_apply(const double* __restrict__ minv, u32 ms, const T* __restrict__ r, T* __restrict__ z, int R) {
    const size_t total = size_t(ms) * R;
    const u32 lane = threadIdx.x % 32;
    const size_t nw = size_t(gridDim.x) * blockDim.x / 32;
    for (size_t i = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; i < total; i += nw) {
        const u32 row = u32(i / R);
        const int col = int(i % R);
        const double* mr = minv + size_t(row) * ms;
        double acc = 0.0;
        for (u32 l = lane; l < ms; l += 32) acc += mr[l] * double(r[size_t(l) * R + col]);
#pragma unroll
        for (int o = 16; o > 0; o /= 2) acc += __shfl_xor_sync(FULL, acc, o);
        if (lane == 0) z[i] = T(acc);
    }
}

// ---------------------------------------------------------------------------------------------
// Grounded LDL^T of the unit-diagonal-scaled small block (precond/dense.rs:26-38, 79-100): a
// pivot at or below PIVOT_TOL is replaced by GROUND. `a` is k x k row-major and only its lower
// triangle is read; its strict lower part becomes the unit-lower factor L, its strict upper part
// L^T (for the inverse's backward pass), `d` the pivots. Blocked right-looking: a panel of NB
// columns is factored by one CTA in shared memory (k_ldlt_panel), then every CTA of
// k_ldlt_trail subtracts the panel's rank-NB update from one 32 x 32 tile of the trailing lower
// triangle. Column by column the arithmetic is the unblocked one (a[i][l] -= a[i][j] a[l][j] / d_j
// with the pivots taken in order); only the order of the trailing sums differs.
constexpr double PIVOT_TOL = 1e-10;
constexpr double GROUND = 1e30;

template <int NB>
__global__ void __launch_bounds__(1024) k_ldlt_panel(double* __restrict__ a, double* __restrict__ d, int k, int jb) {
    extern __shared__ double P[];  // rows jb..k-1 of the panel columns jb..jb+NB-1, NB per row
    const int nb = min(NB, k - jb), rows = k - jb;
    for (int idx = threadIdx.x; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        P[idx] = (c < nb && r >= c) ? a[size_t(jb + r) * k + jb + c] : 0.0;
    }
    for (int jj = 0; jj < nb; jj++) {
        __syncthreads();
        double dj = P[jj * NB + jj];
        if (dj <= PIVOT_TOL) dj = GROUND;
        if (threadIdx.x == 0) d[jb + jj] = dj;
        // the panel's later columns: P[r][l] -= P[r][jj] P[l][jj] / dj for jj < l <= r
        for (int idx = threadIdx.x; idx < (rows - jj - 1) * NB; idx += blockDim.x) {
            const int r = jj + 1 + idx / NB, l = idx % NB;
            if (l > jj && l < nb && l <= r) P[r * NB + l] -= P[r * NB + jj] * P[l * NB + jj] / dj;
        }
        __syncthreads();
        for (int r = jj + 1 + int(threadIdx.x); r < rows; r += blockDim.x) P[r * NB + jj] /= dj;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        if (c < nb && r > c) {
            a[size_t(jb + r) * k + jb + c] = P[idx];
            a[size_t(jb + c) * k + jb + r] = P[idx];
        }
    }
}

// Tile (ti, tl), tl <= ti, of the trailing lower triangle (rows and columns from jb + nb): a[i][l]
// -= sum over the panel's columns p of L[i][p] d_p L[l][p], for l <= i.
template <int NB>
__global__ void __launch_bounds__(256) k_ldlt_trail(double* __restrict__ a, const double* __restrict__ d, int k, int jb,
                                                    int nb) {
    __shared__ double Li[32][NB + 1], Ll[32][NB + 1];
    const int t0 = jb + nb, b = int(blockIdx.x);
    int ti = int((sqrt(8.0 * b + 1.0) - 1.0) / 2.0);
    while ((ti + 1) * (ti + 2) / 2 <= b) ti++;
    while (ti * (ti + 1) / 2 > b) ti--;
    const int tl = b - ti * (ti + 1) / 2;
    const int i0 = t0 + 32 * ti, l0 = t0 + 32 * tl;
    for (int idx = threadIdx.x; idx < 32 * NB; idx += blockDim.x) {
        const int r = idx / NB, p = idx % NB;
        Li[r][p] = (i0 + r < k && p < nb) ? a[size_t(i0 + r) * k + jb + p] : 0.0;
        Ll[r][p] = (l0 + r < k && p < nb) ? a[size_t(l0 + r) * k + jb + p] * d[jb + p] : 0.0;
    }
    __syncthreads();
    const int tx = int(threadIdx.x % 32), ty = int(threadIdx.x / 32);
    const int l = l0 + tx;
    for (int rr = ty; rr < 32; rr += int(blockDim.x / 32)) {
        const int i = i0 + rr;
        if (i < k && l < k && l <= i) {
            double s = 0.0;
#pragma unroll
            for (int p = 0; p < NB; p++) s += Li[rr][p] * Ll[tx][p];
            a[size_t(i) * k + l] -= s;
        }
    }
}

// X = L^-T D^-1 L^-1, one warp per column of X (8 per block), the column held in shared memory:
// forward over L's rows (strict lower part), the pivots, backward over L^T's rows (strict upper
// part), each step a warp-wide dot product combined by a fixed butterfly.
__global__ void __launch_bounds__(256) k_ldlt_inverse(const double* __restrict__ a, const double* __restrict__ d, int k,
                                                      double* __restrict__ x) {
    extern __shared__ double xs[];
    const int w = int(threadIdx.x / 32), lane = int(threadIdx.x % 32);
    const int col = int(blockIdx.x) * 8 + w;
    if (col >= k) return;  // whole warps
    double* v = xs + size_t(w) * k;
    for (int i = lane; i < k; i += 32) v[i] = i == col ? 1.0 : 0.0;
    __syncwarp();
    for (int i = col + 1; i < k; i++) {
        const double* Li = a + size_t(i) * k;
        double s = 0.0;
        for (int p = col + lane; p < i; p += 32) s += Li[p] * v[p];
#pragma unroll
        for (int o = 16; o > 0; o /= 2) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) v[i] = -s;
        __syncwarp();
    }
    for (int i = lane; i < k; i += 32) v[i] /= d[i];
    __syncwarp();
    for (int i = k - 2; i >= 0; i--) {
        const double* Ui = a + size_t(i) * k;
        double s = 0.0;
        for (int p = i + 1 + lane; p < k; p += 32) s += Ui[p] * v[p];
#pragma unroll
        for (int o = 16; o > 0; o /= 2) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) v[i] -= s;
        __syncwarp();
    }
    for (int i = lane; i < k; i += 32) x[size_t(i) * k + col] = v[i];
}

// minv (ms x ms, zero outside the kept coordinates) = S^-1 X S^-1 scattered to the kept rows/cols.
__global__ void k_expand_minv(const double* __restrict__ x, const u32* __restrict__ keep, const double* __restrict__ scale,
                              int k, u32 ms, double* __restrict__ minv) {
    const size_t total = size_t(k) * k;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int a = int(i / k), b = int(i % k);
        minv[size_t(keep[a]) * ms + keep[b]] = scale[a] * x[i] * scale[b];
    }
}

}  // namespace fereg
