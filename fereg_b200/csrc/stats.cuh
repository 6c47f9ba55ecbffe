// Device passes of the OLS call around the solve (stats.rs, ols.rs, vcov.rs, dof.rs):
//   - column statistics of the raw rows (stats.rs:40 col_stats, two passes: sums, then sums of
//     squares about the means);
//   - weighted outer-product sums sum_i w_i a_i a_i^T over selected, shifted columns of a row
//     block (the Gram of stats.rs:195, the robust meat of vcov.rs:292, and S^T S of the cluster
//     scores of vcov.rs:320);
//   - residuals e = y - X b with their weighted sum of squares;
//   - cluster score sums over rows grouped by cluster (a stable cluster permutation);
//   - connected components of two FE terms (dof.rs:222 mobility_groups) by lock-free
//     union-find, and the nested-within check (dof.rs:184).
// Every floating-point sum is a per-CTA partial combined in a fixed order: results do not depend
// on timing.
#pragma once

#include <cstdint>

#include "bulk.cuh"
#include "device.cuh"
#include "scan.cuh"

namespace fereg {

constexpr int ST_TB = 256;          // threads per CTA of the stats passes
constexpr int ST_GRID = 148 * 4;    // CTAs of the row passes (4 per SM: 32 warps)
// Rows per chunk and chunks in flight per CTA of the passes that stream the block by bulk copies
constexpr int CS_ROWS = 128, CS_STAGES = 4;
constexpr int OP_ROWS = 32;         // rows staged per tile of the outer-product pass
constexpr int OP_PPT = 8;           // pairs per thread of one outer-product launch
constexpr int OP_MAXP = ST_TB * OP_PPT;  // pairs of one launch
constexpr int OP_MAXM = 64;         // largest staged vector length (msz) of one launch

// ---------------------------------------------------------------------------------------------
// Column statistics. Lane = (group, column) over a column chunk [j0, j0 + Rc), Rc <= 32; rows are
// dealt to the groups of all warps in turn. Pass 1: [sum x, sum w x, sum x^2, sum w x^2] per
// column; pass 2: [sum (x - mean)^2, sum w (x - wmean)^2]. part[cta][col][NV].
template <int NV>
__device__ __forceinline__ void colstat_add(double x, double w, int pass, const double* mean, const double* wmean,
                                            int col, double* a) {
    if (pass == 1) {
        a[0] += x;
        a[1] += w * x;
        a[2] += x * x;
        a[3] += w * x * x;
    } else {
        const double d = x - mean[col], dw = x - wmean[col];
        a[0] += d * d;
        a[1] += w * dw * dw;
    }
}

template <int NV>
__global__ void __launch_bounds__(ST_TB) k_colstats(const double* __restrict__ rows, size_t n, int R, int j0, int Rc,
                                                    const double* __restrict__ w, int pass,
                                                    const double* __restrict__ mean,
                                                    const double* __restrict__ wmean, double* __restrict__ part) {
    __shared__ double red[ST_TB / 32][32][NV];
    int rcp = 1;
    while (rcp < Rc) rcp <<= 1;
    const int G = 32 / rcp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / rcp, j = lane % rcp;
    const bool on = j < Rc;
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) a[v] = 0.0;
    const size_t gw = size_t(blockIdx.x) * (ST_TB / 32) + warp, nw = size_t(gridDim.x) * (ST_TB / 32);
    if (on)
        for (size_t r = gw * G + g; r < n; r += nw * G) {
            const double x = rows[r * R + j0 + j];
            colstat_add<NV>(x, w ? w[r] : 1.0, pass, mean, wmean, j0 + j, a);
        }
#pragma unroll
    for (int v = 0; v < NV; v++) red[warp][lane][v] = on ? a[v] : 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < Rc * NV; i += ST_TB) {
        const int col = i / NV, v = i % NV;
        double s = 0.0;
        for (int wp = 0; wp < ST_TB / 32; wp++)
            for (int gg = 0; gg < G; gg++) s += red[wp][gg * rcp + col][v];
        part[(size_t(blockIdx.x) * R + j0 + col) * NV + v] = s;
    }
}

// Sum of `parts` rows of length len, one warp per element: lane l adds rows l, l + 32, ... in
// order, then the lanes' sums are combined by a fixed butterfly (the same order every call).
__global__ void k_sum_parts(const double* __restrict__ part, int parts, int len, double* __restrict__ out) {
    const int i = blockIdx.x * (blockDim.x / 32) + int(threadIdx.x / 32);
    const int lane = int(threadIdx.x % 32);
    if (i >= len) return;  // whole warps leave together
    double s = 0.0;
    for (int p = lane; p < parts; p += 32) s += part[size_t(p) * len + i];
#pragma unroll
    for (int o = 16; o > 0; o /= 2) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[i] = s;
}
// Launch shape of k_sum_parts for len elements (8 warps per block).
inline unsigned sum_parts_blocks(int len) { return unsigned((len + 7) / 8); }

// Sum of the weights (sum w, and the count) over rows.
__global__ void __launch_bounds__(ST_TB) k_sum_w(const double* __restrict__ w, size_t n, double* __restrict__ part) {
    __shared__ double red[ST_TB];
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * ST_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * ST_TB) s += w[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = ST_TB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------------------------
// Weighted outer products: sum_i om_i a_i a_i^T, a_i[p] = x_i[col[p]] + shift[p] for p < k and
// a_i[k] = 1 when cst. Pairs (a, b), a <= b, in row-major upper-triangle order, pairs
// [p0, p0 + np) of this launch (np <= OP_MAXP); ssq: also sum_i x_i[col[p]]^2 (unweighted) for
// p < k. part[cta][np (+ k)].
struct OpSpec {
    const double* rows;   // n x R row-major
    size_t n;
    int R;
    const int* col;       // k column indices (device)
    const double* shift;  // k shifts (device) or null
    int k, cst, msz;      // msz = k + cst
    const double* om;     // per-row weight or null (= 1)
    const int* perm;      // row i of the pass is rows[perm[i]] (null = identity)
    int p0, np;
    int ssq;
};

__global__ void __launch_bounds__(ST_TB) k_outer(OpSpec s, double* __restrict__ part) {
    __shared__ double tile[OP_ROWS][OP_MAXM + 1];
    __shared__ double tom[OP_ROWS];
    __shared__ short pa[OP_MAXP], pb[OP_MAXP];
    for (int q = threadIdx.x; q < s.np; q += ST_TB) {
        // pair p0 + q -> (a, b): row a holds msz - a pairs
        int p = s.p0 + q, a = 0;
        while (p >= s.msz - a) {
            p -= s.msz - a;
            a++;
        }
        pa[q] = short(a);
        pb[q] = short(a + p);
    }
    double acc[OP_PPT];
#pragma unroll
    for (int t = 0; t < OP_PPT; t++) acc[t] = 0.0;
    double sq = 0.0;  // thread tid < k: sum x^2 of column tid
    const size_t ntile = (s.n + OP_ROWS - 1) / OP_ROWS;
    for (size_t tl = blockIdx.x; tl < ntile; tl += gridDim.x) {
        __syncthreads();
        const size_t r0 = tl * OP_ROWS;
        const int nr = int((s.n - r0 < size_t(OP_ROWS) ? s.n - r0 : size_t(OP_ROWS)));
        for (int e = threadIdx.x; e < nr * s.msz; e += ST_TB) {
            const int i = e / s.msz, p = e % s.msz;
            const size_t row = s.perm ? size_t(s.perm[r0 + i]) : r0 + i;
            tile[i][p] = p < s.k ? s.rows[row * s.R + s.col[p]] + (s.shift ? s.shift[p] : 0.0) : 1.0;
        }
        for (int i = threadIdx.x; i < nr; i += ST_TB) {
            const size_t row = s.perm ? size_t(s.perm[r0 + i]) : r0 + i;
            tom[i] = s.om ? s.om[row] : 1.0;
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < OP_PPT; t++) {
            const int q = threadIdx.x + t * ST_TB;
            if (q < s.np) {
                const int a = pa[q], b = pb[q];
                double v = acc[t];
                for (int i = 0; i < nr; i++) v += tom[i] * tile[i][a] * tile[i][b];
                acc[t] = v;
            }
        }
        if (s.ssq && threadIdx.x < s.k) {
            const double sh = s.shift ? s.shift[threadIdx.x] : 0.0;
            for (int i = 0; i < nr; i++) {
                const double x = tile[i][threadIdx.x] - sh;
                sq += x * x;
            }
        }
    }
    const int len = s.np + (s.ssq ? s.k : 0);
#pragma unroll
    for (int t = 0; t < OP_PPT; t++) {
        const int q = threadIdx.x + t * ST_TB;
        if (q < s.np) part[size_t(blockIdx.x) * len + q] = acc[t];
    }
    if (s.ssq && threadIdx.x < s.k) part[size_t(blockIdx.x) * len + s.np + threadIdx.x] = sq;
}

// Outer products for msz <= 32 (the common case): lane = (group g, column j) of a chunk padded
// to RCP; each group holds one row's vector a_i, and lane j accumulates row j of the matrix,
// om_i a_i[j] a_i[b] for every b, taking a_i[b] from lane (g, b) by shuffle. Rows come U groups
// at a time with their loads batched. Sums: per lane in row order, then groups and warps in a
// fixed order into the CTA's partial part[cta][msz * msz (+ k)].
template <int RCP>
__global__ void __launch_bounds__(ST_TB) k_outer_small(OpSpec s, double* __restrict__ part) {
    constexpr int G = 32 / RCP;
    constexpr int U = RCP >= 32 ? 2 : 4;
    __shared__ double red[RCP * RCP + RCP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / RCP, j = lane % RCP;
    const bool on = j < s.msz;
    const int colj = j < s.k ? s.col[j] : -1;
    const double shj = (j < s.k && s.shift) ? s.shift[j] : 0.0;
    for (int i = threadIdx.x; i < RCP * RCP + RCP; i += ST_TB) red[i] = 0.0;
    double acc[RCP];
#pragma unroll
    for (int b = 0; b < RCP; b++) acc[b] = 0.0;
    double sq = 0.0;
    const size_t gw = size_t(blockIdx.x) * (ST_TB / 32) + warp, nw = size_t(gridDim.x) * (ST_TB / 32);
    for (size_t base = gw * U * G; base < s.n; base += nw * U * G) {
        double x[U], om[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const size_t r = base + size_t(u) * G + g;
            x[u] = 0.0;
            om[u] = 0.0;
            if (r < s.n) {
                const size_t row = s.perm ? size_t(s.perm[r]) : r;
                if (on) x[u] = colj >= 0 ? s.rows[row * s.R + colj] + shj : 1.0;
                om[u] = s.om ? s.om[row] : 1.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const double wx = om[u] * x[u];
            if (s.ssq && colj >= 0) {
                const double d = x[u] - shj;
                sq += d * d;
            }
#pragma unroll
            for (int b = 0; b < RCP; b++) acc[b] += wx * __shfl_sync(FULL, x[u], g * RCP + b);
        }
    }
    // groups in order (lane (0, j) ends with the warp's row j), then warps in order
#pragma unroll
    for (int b = 0; b < RCP; b++) {
        double t = 0.0;
#pragma unroll
        for (int gg = 0; gg < G; gg++) t += __shfl_sync(FULL, acc[b], gg * RCP + j);
        acc[b] = t;
    }
    double tq = 0.0;
#pragma unroll
    for (int gg = 0; gg < G; gg++) tq += __shfl_sync(FULL, sq, gg * RCP + j);
    __syncthreads();
    for (int w = 0; w < ST_TB / 32; w++) {
        if (warp == w && g == 0 && on) {
#pragma unroll
            for (int b = 0; b < RCP; b++) red[j * RCP + b] += acc[b];
            red[RCP * RCP + j] += tq;
        }
        __syncthreads();
    }
    const int mm = s.msz * s.msz;
    const int len = mm + (s.ssq ? s.k : 0);
    for (int i = threadIdx.x; i < len; i += ST_TB)
        part[size_t(blockIdx.x) * len + i] = i < mm ? red[(i / s.msz) * RCP + i % s.msz] : red[RCP * RCP + (i - mm)];
}

// Outer products on the FP64 tensor cores (mma.sync m8n8k4, f64 in and out), msz <= 8 NB: the
// matrix is tiled by 8 x 8 blocks (bi <= bj). A warp takes 4 rows per MMA step: lane l holds
// a_i[8 b + (l >> 2)] of row 4 t + (l & 3) for each column block b, which is both its A fragment
// (scaled by om_i: A[m][k] = om a[8 bi + m] of row k) and its B fragment (B[k][n] =
// a[8 bj + n] of row k). Each warp accumulates its rows in MMA order, then warps are added in a
// fixed order into the CTA's partial part[cta][msz * msz (+ k)] (upper blocks filled).
__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <int NB>
__global__ void __launch_bounds__(ST_TB, NB <= 2 ? 4 : 2) k_outer_mma(OpSpec s, double* __restrict__ part) {
    constexpr int NT = NB * (NB + 1) / 2, U = 4, W = 8 * NB;
    __shared__ double red[W * W + W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kr = lane & 3, cj = lane >> 2;
    // column source of each block: >= 0 a row column, -1 the constant, -2 padding
    int csrc[NB];
    double csh[NB];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int c = 8 * b + cj;
        csrc[b] = c < s.k ? s.col[c] : (c < s.msz ? -1 : -2);
        csh[b] = (c < s.k && s.shift) ? s.shift[c] : 0.0;
    }
    for (int i = threadIdx.x; i < W * W + W; i += ST_TB) red[i] = 0.0;
    double acc[NT][2];
#pragma unroll
    for (int t = 0; t < NT; t++) acc[t][0] = acc[t][1] = 0.0;
    double sq[NB];
#pragma unroll
    for (int b = 0; b < NB; b++) sq[b] = 0.0;
    const size_t gw = size_t(blockIdx.x) * (ST_TB / 32) + warp, nw = size_t(gridDim.x) * (ST_TB / 32);
    for (size_t base = gw * U * 4; base < s.n; base += nw * U * 4) {
        double v[U][NB], om[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const size_t r = base + size_t(u) * 4 + kr;
            om[u] = 0.0;
#pragma unroll
            for (int b = 0; b < NB; b++) v[u][b] = 0.0;
            if (r < s.n) {
                const size_t row = s.perm ? size_t(s.perm[r]) : r;
                om[u] = s.om ? s.om[row] : 1.0;
#pragma unroll
                for (int b = 0; b < NB; b++)
                    v[u][b] = csrc[b] >= 0 ? s.rows[row * s.R + csrc[b]] + csh[b] : (csrc[b] == -1 ? 1.0 : 0.0);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (s.ssq) {
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    const double x = csrc[b] >= 0 ? v[u][b] - csh[b] : 0.0;
                    sq[b] += x * x;
                }
            }
            int t = 0;
#pragma unroll
            for (int bi = 0; bi < NB; bi++) {
                const double a = om[u] * v[u][bi];
#pragma unroll
                for (int bj = bi; bj < NB; bj++, t++) dmma884(acc[t][0], acc[t][1], a, v[u][bj]);
            }
        }
    }
    // sums of squares: the 4 lanes of a column (l & 3 = 0..3) in order
#pragma unroll
    for (int b = 0; b < NB; b++) {
        double q = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) q += __shfl_sync(FULL, sq[b], (cj << 2) + k);
        sq[b] = q;
    }
    __syncthreads();
    for (int w = 0; w < ST_TB / 32; w++) {
        if (warp == w) {
            int t = 0;
#pragma unroll
            for (int bi = 0; bi < NB; bi++)
#pragma unroll
                for (int bj = bi; bj < NB; bj++, t++) {
                    const int rr = 8 * bi + cj, cc = 8 * bj + 2 * kr;
                    red[rr * W + cc] += acc[t][0];
                    red[rr * W + cc + 1] += acc[t][1];
                }
            if (kr == 0)
#pragma unroll
                for (int b = 0; b < NB; b++) red[W * W + 8 * b + cj] += sq[b];
        }
        __syncthreads();
    }
    const int mm = s.msz * s.msz;
    const int len = mm + (s.ssq ? s.k : 0);
    for (int i = threadIdx.x; i < len; i += ST_TB)
        part[size_t(blockIdx.x) * len + i] = i < mm ? red[(i / s.msz) * W + i % s.msz] : red[W * W + (i - mm)];
}

// k_outer_mma with the rows streamed through shared memory by bulk copies (the ring of
// k_colstats_bulk, whose constants it uses): for a contiguous block (no permutation), R <= 32
// columns, starting on a 16-byte boundary. A chunk of CS_ROWS rows is one MMA step of every warp
// (16 rows each); CTA 0 takes the rows past the last whole chunk by direct loads. A wait that runs
// out sets *err and the CTA returns after its copies in flight, without writing its partial.
template <int NB>
__global__ void __launch_bounds__(ST_TB, NB <= 2 ? 3 : 2) k_outer_mma_bulk(OpSpec s, double* __restrict__ part,
                                                                          int* __restrict__ err) {
    constexpr int NT = NB * (NB + 1) / 2, U = 4, W = 8 * NB, NWARP = ST_TB / 32;
    static_assert(NWARP * U * 4 == CS_ROWS, "one MMA step of every warp per chunk");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) u64 bar[CS_STAGES];
    __shared__ double red[W * W + W];
    double* buf = reinterpret_cast<double*>(smem_raw);  // CS_STAGES x CS_ROWS x R
    const int R = s.R;
    const u32 chunk = u32(CS_ROWS) * u32(R);
    const size_t nchunks = s.n / CS_ROWS;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kr = lane & 3, cj = lane >> 2;
    int csrc[NB];
    double csh[NB];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int c = 8 * b + cj;
        csrc[b] = c < s.k ? s.col[c] : (c < s.msz ? -1 : -2);
        csh[b] = (c < s.k && s.shift) ? s.shift[c] : 0.0;
    }
    for (int i = threadIdx.x; i < W * W + W; i += ST_TB) red[i] = 0.0;
    double acc[NT][2];
#pragma unroll
    for (int t = 0; t < NT; t++) acc[t][0] = acc[t][1] = 0.0;
    double sq[NB];
#pragma unroll
    for (int b = 0; b < NB; b++) sq[b] = 0.0;
    auto mma_step = [&](const double (&v)[U][NB], const double (&om)[U]) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (s.ssq) {
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    const double x = csrc[b] >= 0 ? v[u][b] - csh[b] : 0.0;
                    sq[b] += x * x;
                }
            }
            int t = 0;
#pragma unroll
            for (int bi = 0; bi < NB; bi++) {
                const double a = om[u] * v[u][bi];
#pragma unroll
                for (int bj = bi; bj < NB; bj++, t++) dmma884(acc[t][0], acc[t][1], a, v[u][bj]);
            }
        }
    };
    const size_t mine = blockIdx.x < nchunks ? (nchunks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    auto issue = [&](size_t i) {  // thread 0: chunk i of this CTA into buffer i mod CS_STAGES
        const int sb = int(i % CS_STAGES);
        const size_t q = blockIdx.x + i * gridDim.x;
        mbar_expect_tx(&bar[sb], chunk * 8u);
        bulk_load(buf + size_t(sb) * chunk, s.rows + q * chunk, chunk * 8u, &bar[sb]);
    };
    if (threadIdx.x == 0) {
        for (int sb = 0; sb < CS_STAGES; sb++) mbar_init(&bar[sb], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (size_t i = 0; i < mine && i < size_t(CS_STAGES); i++) issue(i);
    size_t failed = mine;
    for (size_t i = 0; i < mine; i++) {
        const int sb = int(i % CS_STAGES);
        const bool late = !mbar_wait(&bar[sb], u32((i / CS_STAGES) & 1), MBAR_WAIT_LIMIT);
        if (__syncthreads_or(late)) {
            failed = i;
            break;
        }
        const double* cb = buf + size_t(sb) * chunk;
        const size_t r0 = (blockIdx.x + i * gridDim.x) * CS_ROWS;
        double v[U][NB], om[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int rr = warp * (U * 4) + u * 4 + kr;
            om[u] = s.om ? s.om[r0 + rr] : 1.0;
#pragma unroll
            for (int b = 0; b < NB; b++)
                v[u][b] = csrc[b] >= 0 ? cb[rr * R + csrc[b]] + csh[b] : (csrc[b] == -1 ? 1.0 : 0.0);
        }
        mma_step(v, om);
        __syncthreads();  // every thread is done with buffer sb
        if (threadIdx.x == 0 && i + CS_STAGES < mine) issue(i + CS_STAGES);
    }
    if (failed < mine) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            for (size_t i = failed; i < mine && i < failed + CS_STAGES; i++)
                mbar_wait(&bar[i % CS_STAGES], u32((i / CS_STAGES) & 1), MBAR_WAIT_LIMIT);
        }
        __syncthreads();
        return;
    }
    if (blockIdx.x == 0)  // the rows past the last whole chunk (a whole warp per base: MMA is warp-wide)
        for (size_t base = nchunks * CS_ROWS + size_t(warp) * U * 4; base < s.n; base += size_t(NWARP) * U * 4) {
            double v[U][NB], om[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const size_t r = base + size_t(u) * 4 + kr;
                om[u] = 0.0;
#pragma unroll
                for (int b = 0; b < NB; b++) v[u][b] = 0.0;
                if (r < s.n) {
                    om[u] = s.om ? s.om[r] : 1.0;
#pragma unroll
                    for (int b = 0; b < NB; b++)
                        v[u][b] = csrc[b] >= 0 ? s.rows[r * R + csrc[b]] + csh[b] : (csrc[b] == -1 ? 1.0 : 0.0);
                }
            }
            mma_step(v, om);
        }
#pragma unroll
    for (int b = 0; b < NB; b++) {
        double q = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) q += __shfl_sync(FULL, sq[b], (cj << 2) + k);
        sq[b] = q;
    }
    __syncthreads();
    for (int w = 0; w < NWARP; w++) {
        if (warp == w) {
            int t = 0;
#pragma unroll
            for (int bi = 0; bi < NB; bi++)
#pragma unroll
                for (int bj = bi; bj < NB; bj++, t++) {
                    const int rr = 8 * bi + cj, cc = 8 * bj + 2 * kr;
                    red[rr * W + cc] += acc[t][0];
                    red[rr * W + cc + 1] += acc[t][1];
                }
            if (kr == 0)
#pragma unroll
                for (int b = 0; b < NB; b++) red[W * W + 8 * b + cj] += sq[b];
        }
        __syncthreads();
    }
    const int mm = s.msz * s.msz;
    const int len = mm + (s.ssq ? s.k : 0);
    for (int i = threadIdx.x; i < len; i += ST_TB)
        part[size_t(blockIdx.x) * len + i] = i < mm ? red[(i / s.msz) * W + i % s.msz] : red[W * W + (i - mm)];
}

// Column statistics in one pass, about a shift c per column (the column's first value):
// [sum (x-c), sum (x-c)^2, sum w (x-c), sum w (x-c)^2, sum x^2, sum w x^2] per column; the means
// and the sums of squares about them follow exactly up to rounding (m2 = S2 - S1^2 / n).
// Lane = (group, column) over a column chunk [j0, j0 + Rc) padded to RCP; rows U groups at a time.
template <int RCP>
__global__ void __launch_bounds__(ST_TB, 4) k_colstats1(const double* __restrict__ rows, size_t n, int R, int j0, int Rc,
                                                     const double* __restrict__ w, double* __restrict__ part) {
    constexpr int G = 32 / RCP, U = 4, NV = 6;
    __shared__ double red[ST_TB / 32][32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / RCP, j = lane % RCP;
    const bool on = j < Rc;
    const double c = on ? rows[j0 + j] : 0.0;
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) a[v] = 0.0;
    const size_t gw = size_t(blockIdx.x) * (ST_TB / 32) + warp, nw = size_t(gridDim.x) * (ST_TB / 32);
    if (on)
        for (size_t base = gw * U * G; base < n; base += nw * U * G) {
            double x[U], wv[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const size_t r = base + size_t(u) * G + g;
                x[u] = r < n ? rows[r * R + j0 + j] : c;
                wv[u] = r < n ? (w ? w[r] : 1.0) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (base + size_t(u) * G + g >= n) continue;
                const double d = x[u] - c;
                a[0] += d;
                a[1] += d * d;
                a[2] += wv[u] * d;
                a[3] += wv[u] * d * d;
                a[4] += x[u] * x[u];
                a[5] += wv[u] * x[u] * x[u];
            }
        }
#pragma unroll
    for (int v = 0; v < NV; v++) red[warp][lane][v] = on ? a[v] : 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < Rc * NV; i += ST_TB) {
        const int col = i / NV, v = i % NV;
        double t = 0.0;
        for (int wp = 0; wp < ST_TB / 32; wp++)
            for (int gg = 0; gg < G; gg++) t += red[wp][gg * RCP + col][v];
        part[(size_t(blockIdx.x) * R + j0 + col) * NV + v] = t;
    }
}

// The same statistics of all R <= 32 columns, the block streamed through shared memory by bulk
// copies: CTA b takes the chunks of CS_ROWS whole rows b, b + grid, ... into a ring of CS_STAGES
// buffers, thread 0 issuing the copies (one mbarrier per buffer, its phase expecting the chunk's
// bytes) and every thread reading a buffer once its phase completes; lanes are (group, column)
// pairs over the buffer's rows. CTA 0 reads the rows past the last whole chunk directly. A wait
// that runs out (never expected) sets *err; the CTA then waits, bounded, for its copies in flight
// and returns without writing its partial. The block must start on a 16-byte boundary (each chunk
// is 1024 R bytes).
template <int RCP>
__global__ void __launch_bounds__(ST_TB, 4) k_colstats_bulk(const double* __restrict__ rows, size_t n, int R,
                                                          const double* __restrict__ w, double* __restrict__ part,
                                                          int* __restrict__ err) {
    constexpr int G = 32 / RCP, NV = 6, NWARP = ST_TB / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) u64 bar[CS_STAGES];
    __shared__ double red[NWARP][32][NV];
    double* buf = reinterpret_cast<double*>(smem_raw);  // CS_STAGES x CS_ROWS x R
    const u32 chunk = u32(CS_ROWS) * u32(R);
    const size_t nchunks = n / CS_ROWS;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / RCP, j = lane % RCP;
    const bool on = j < R;
    const double c = on ? rows[j] : 0.0;
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) a[v] = 0.0;
    auto add = [&](double x, double wv) {
        const double d = x - c;
        a[0] += d;
        a[1] += d * d;
        a[2] += wv * d;
        a[3] += wv * d * d;
        a[4] += x * x;
        a[5] += wv * x * x;
    };
    const size_t mine = blockIdx.x < nchunks ? (nchunks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    auto issue = [&](size_t i) {  // thread 0: chunk i of this CTA into buffer i mod CS_STAGES
        const int sb = int(i % CS_STAGES);
        const size_t q = blockIdx.x + i * gridDim.x;
        mbar_expect_tx(&bar[sb], chunk * 8u);
        bulk_load(buf + size_t(sb) * chunk, rows + q * chunk, chunk * 8u, &bar[sb]);
    };
    if (threadIdx.x == 0) {
        for (int sb = 0; sb < CS_STAGES; sb++) mbar_init(&bar[sb], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (size_t i = 0; i < mine && i < size_t(CS_STAGES); i++) issue(i);
    size_t failed = mine;
    for (size_t i = 0; i < mine; i++) {
        const int sb = int(i % CS_STAGES);
        const bool late = !mbar_wait(&bar[sb], u32((i / CS_STAGES) & 1), MBAR_WAIT_LIMIT);
        if (__syncthreads_or(late)) {
            failed = i;
            break;
        }
        const double* cb = buf + size_t(sb) * chunk;
        const size_t r0 = (blockIdx.x + i * gridDim.x) * CS_ROWS;
        if (on)
            for (int rr = warp * G + g; rr < CS_ROWS; rr += NWARP * G) add(cb[rr * R + j], w ? w[r0 + rr] : 1.0);
        __syncthreads();  // every thread is done with buffer sb
        if (threadIdx.x == 0 && i + CS_STAGES < mine) issue(i + CS_STAGES);
    }
    if (failed < mine) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            for (size_t i = failed; i < mine && i < failed + CS_STAGES; i++)
                mbar_wait(&bar[i % CS_STAGES], u32((i / CS_STAGES) & 1), MBAR_WAIT_LIMIT);
        }
        __syncthreads();
        return;
    }
    if (blockIdx.x == 0 && on)
        for (size_t r = nchunks * CS_ROWS + size_t(warp * G + g); r < n; r += NWARP * G)
            add(rows[r * R + j], w ? w[r] : 1.0);
#pragma unroll
    for (int v = 0; v < NV; v++) red[warp][lane][v] = on ? a[v] : 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < R * NV; i += ST_TB) {
        const int col = i / NV, v = i % NV;
        double t = 0.0;
        for (int wp = 0; wp < NWARP; wp++)
            for (int gg = 0; gg < G; gg++) t += red[wp][gg * RCP + col][v];
        part[(size_t(blockIdx.x) * R + col) * NV + v] = t;
    }
}

// ---------------------------------------------------------------------------------------------
// Residuals: e_i = y_i - sum_p beta[p] x_i[col[p]] (y = column 0, or 0 when y_zero); per-CTA
// partials of sum om_i e_i^2.
__global__ void __launch_bounds__(ST_TB, 4) k_resid_e(const double* __restrict__ rows, size_t n, int R,
                                                   const int* __restrict__ col, const double* __restrict__ beta, int k,
                                                   int y_zero, const double* __restrict__ om, double* __restrict__ e,
                                                   double* __restrict__ part) {
    __shared__ double red[ST_TB];
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * ST_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * ST_TB) {
        const double* row = rows + i * R;
        double v = y_zero ? 0.0 : row[0];
        for (int p = 0; p < k; p++) v -= beta[p] * row[col[p]];
        e[i] = v;
        s += (om ? om[i] : 1.0) * v * v;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = ST_TB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Robust meat weights (vcov.rs:292): e^2 (no weights), e^2 w (fweights), (e w)^2 (aweights,
// pweights); cluster score weights: e w.
__global__ void k_meat_weights(const double* __restrict__ e, const double* __restrict__ w, size_t n, int kind,
                               int cluster, double* __restrict__ om) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double wi = w ? w[i] : 1.0, ei = e[i];
        if (cluster) om[i] = ei * wi;
        else if (!w) om[i] = ei * ei;
        else if (kind == 2) om[i] = ei * ei * wi;
        else om[i] = (ei * wi) * (ei * wi);
    }
}

// Cluster scores: S[g][p] = sum over the rows of cluster g (perm[coff[g]..coff[g+1]], in order)
// of om_i a_i[p]; a warp per cluster, lanes over p.
__global__ void __launch_bounds__(ST_TB) k_cluster_scores(const double* __restrict__ rows, int R,
                                                          const int* __restrict__ col,
                                                          const double* __restrict__ shift, int k, int cst,
                                                          const double* __restrict__ om, const int* __restrict__ perm,
                                                          const u32* __restrict__ coff, u32 G, double* __restrict__ S) {
    const int lane = threadIdx.x & 31;
    const int msz = k + cst;
    const size_t gw = size_t(blockIdx.x) * (ST_TB / 32) + (threadIdx.x >> 5), nw = size_t(gridDim.x) * (ST_TB / 32);
    for (size_t g = gw; g < G; g += nw) {
        for (int p0 = 0; p0 < msz; p0 += 32) {
            const int p = p0 + lane;
            double s = 0.0;
            if (p < msz)
                for (u32 q = coff[g]; q < coff[g + 1]; q++) {
                    const size_t row = size_t(perm[q]);
                    const double a = p < k ? rows[row * R + col[p]] + (shift ? shift[p] : 0.0) : 1.0;
                    s += om[row] * a;
                }
            if (p < msz) S[g * msz + p] = s;
        }
    }
}

// Row gather of kept-order columns into the row-order block: rows[i R + j] = cols[j n + pi[i]]
// (the reference's Session::gather, session.rs, on the device). A warp per row chunk: lanes over
// consecutive rows i read the index pi[i] once and write R values each.
__global__ void k_gather_cols(const double* __restrict__ cols, const u32* __restrict__ pi, size_t n, int R,
                              double* __restrict__ rows) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const size_t src = pi[i];
        for (int j = 0; j < R; j++) rows[i * R + j] = cols[size_t(j) * n + src];
    }
}

__global__ void k_zero_col(double* __restrict__ rows, size_t n, int R, int c) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        rows[i * R + c] = 0.0;
}

// ---------------------------------------------------------------------------------------------
// Connected components of the bipartite graph of two terms (vertices: a-levels 0..ga-1, then
// b-levels ga..ga+gb-1). Linking always hangs the larger root below the smaller one, so a
// component's root is its smallest vertex: its smallest a-level (every b-level meets some
// a-level). The partition is unique, so labels do not depend on timing.
__global__ void k_uf_init(u32* __restrict__ parent, u32 nv) {
    for (u32 v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) parent[v] = v;
}

__device__ __forceinline__ u32 uf_find(u32* parent, u32 v) {
    // Path halving. Parents only decrease (a link sets parent[hi] = lo < hi; halving sets an
    // ancestor), so the walk strictly descends and ends at a vertex that was a root when its
    // entry was read. The reads go through L1 and may be stale under concurrent links: a stale
    // entry still names an ancestor, so two walks that end at the same vertex prove one
    // component, and a link attempted on a vertex that is no longer a root fails its CAS (at L2)
    // and retries from the parent the CAS returns. Caching keeps the root of a large component,
    // which every walk ends at, out of a single hot L2 line.
    u32 p = __ldca(parent + v);
    while (p != v) {
        const u32 gp = __ldca(parent + p);
        if (gp != p) parent[v] = gp;  // benign race: any ancestor is a valid parent
        v = p;
        p = __ldca(parent + v);
    }
    return v;
}

// err: set to 1 if a union step ran out of its retry budget (never expected).
__global__ void k_uf_union(const u32* __restrict__ a, const u32* __restrict__ b, u32 ga, size_t n, u32* parent,
                           int* err) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        u32 u = a[i], v = ga + b[i];
        for (int it = 0; it < (1 << 20); it++) {
            u = uf_find(parent, u);
            v = uf_find(parent, v);
            if (u == v) break;
            const u32 lo = min(u, v), hi = max(u, v);
            const u32 old = atomicCAS(parent + hi, hi, lo);
            if (old == hi) break;  // linked
            u = lo;
            v = old;  // hi already had a new parent: retry from there
            if (it == (1 << 20) - 1) atomicExch(err, 1);
        }
    }
}

__global__ void k_uf_flatten(u32* parent, u32 nv) {
    for (u32 v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        parent[v] = uf_find(parent, v);
}

// flags[l] = 1 when a-level l is its component's root.
__global__ void k_uf_roots(const u32* __restrict__ parent, u32 ga, u32* __restrict__ flags) {
    for (u32 l = blockIdx.x * blockDim.x + threadIdx.x; l < ga; l += gridDim.x * blockDim.x)
        flags[l] = parent[l] == l ? 1u : 0u;
}

// groupvar[i] = 1-based component number of row i (components numbered by their smallest
// a-level): id = exclusive scan of the root flags + 1.
__global__ void k_uf_label(const u32* __restrict__ a, size_t n, const u32* __restrict__ parent,
                           const u32* __restrict__ scan, u32* __restrict__ gv) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        gv[i] = scan[parent[a[i]]] + 1u;
}

// Nested within (dof.rs:184): map[level] takes the first cluster value seen; any other value
// marks the term as not nested (flag = 1). Rows in any order give the same verdict.
__global__ void k_nested(const u32* __restrict__ codes, const u32* __restrict__ cl, size_t n, u32* map, int* flag) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const u32 old = atomicCAS(map + codes[i], 0xffffffffu, cl[i]);
        if (old != 0xffffffffu && old != cl[i]) atomicExch(flag, 1);
    }
}

// ---------------------------------------------------------------------------------------------
// Exclusive scan of u32 (three passes: block sums, a scan of the block sums in one CTA, block
// scans plus their offsets). total (device) receives the sum.
}  // namespace fereg
