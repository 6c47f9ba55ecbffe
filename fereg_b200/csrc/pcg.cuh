// The PCG iteration's vector steps (cg.rs:132-292) as four kernels, each reducing its column sums
// in the same launch: every CTA writes its partials, and the CTA that finishes last (a ticket
// counter, after a memory fence) adds them in CTA order with the fixed order of k_reduce_cols and
// applies the iteration's scalar step. Results are independent of which CTA finishes last.
//
// The iteration counter lives on the device, so the same kernels run launched one by one or as
// the body of a captured CUDA graph whose WHILE node repeats them: k_update_p_cond ends every
// iteration by setting the loop condition (columns still active and fewer than the launch's cap
// iterations run). Its counter rises on every execution of the body, so a graph launch ends
// after at most `cap` iterations whatever the stopping rule does.
#pragma once

#include "kernels.cuh"

namespace fereg {

// Device state of the iteration loop.
struct CgLoop {
    int* ctl;             // [n_active (mirrors CgState::n_active), k since the (re)start, k of this launch, cap]
    const double* tol;    // the stopping rule's tolerance (set per solve, so that one graph serves every tolerance)
    unsigned* ticket;     // last-CTA counters of the three reducing kernels
    double* rho_from;     // rho after iteration PROBE_FROM (cg.rs:24-37 probe)
    double* rho_at;       // rho after iteration PROBE_AT
    int* act_at;          // the column states after iteration PROBE_AT
};

// True in the CTA that finishes last; its loads of the other CTAs' partials must bypass L1.
__device__ __forceinline__ bool last_cta(unsigned* ticket) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) % gridDim.x) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Above WIDE_R columns the vector kernels give each thread whole columns (coalesced across the
// threads), and the last CTA sums a column's partials with one thread, in part order.
constexpr int WIDE_R = 64;

// Column sums of [nparts x ncols] partials by one CTA in a fixed order: up to WIDE_R columns (the
// order of k_reduce_cols) warp w takes columns w, w + warps, ..., lane l adds parts l, l + 32, ...,
// then a fixed butterfly; wider, thread t adds the parts of columns t, t + threads, ... in order.
__device__ __forceinline__ void cta_col_sums(const double* part, int nparts, int ncols, int R, double* out) {
    if (R > WIDE_R) {
        for (int col = threadIdx.x; col < ncols; col += blockDim.x) {
            double acc = 0.0;
            for (int p = 0; p < nparts; p++) acc += __ldcg(part + size_t(p) * ncols + col);
            out[col] = acc;
        }
        return;
    }
    const int lane = int(threadIdx.x & 31), w = int(threadIdx.x >> 5), nw = int(blockDim.x >> 5);
    for (int col = w; col < ncols; col += nw) {
        double acc = 0.0;
        for (int p = lane; p < nparts; p += 32) acc += __ldcg(part + size_t(p) * ncols + col);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
        if (lane == 0) out[col] = acc;
    }
}

// Per-CTA partials of a'b per column (the layout of k_dot); above WIDE_R columns thread t takes
// columns t, t + threads, ... over the CTA's rows.
template <class T>
__device__ __forceinline__ void dot_partials(const T* __restrict__ a, const T* __restrict__ b, u32 m, int R,
                                             double* __restrict__ cta_part, double* red) {
    if (R > WIDE_R) {
        for (int c = threadIdx.x; c < R; c += blockDim.x) {
            double acc = 0.0;
            for (u32 i = blockIdx.x; i < m; i += gridDim.x) {
                const size_t o = size_t(i) * R + c;
                acc += double(a[o]) * double(b[o]);
            }
            cta_part[size_t(blockIdx.x) * R + c] = acc;
        }
        return;
    }
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

// p'q, then gamma = rho / p'q on the active columns (a non-positive or non-finite p'q deactivates).
template <class T>
__global__ void __launch_bounds__(TB) k_pq_gamma(const T* __restrict__ p, const T* __restrict__ q, u32 m, int R,
                                                 double* __restrict__ cta_part, CgState st, CgLoop lp) {
    __shared__ double red[TB];
    dot_partials(p, q, m, R, cta_part, red);
    if (!last_cta(lp.ticket)) return;
    cta_col_sums(cta_part, int(gridDim.x), R, R, st.pq);
    __syncthreads();
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
        double g = 0.0;
        if (st.active[j] == 1) {
            const double pq = st.pq[j];
            if (pq > 0.0 && isfinite(pq)) g = st.rho[j] / pq;
            else st.active[j] = st.pfloor[j] > 0.0 ? 2 : 0;  // inner rounds: FP64 restart, not a stop
        }
        st.gamma[j] = g;
    }
    if (threadIdx.x == 0) lp.ticket[0] = 0;
}

// x += gamma p, r -= gamma q, and x'rhs, x'r, x0'r (x0 null: 0) into st.xb.
template <class T>
__global__ void __launch_bounds__(TB) k_update_xr_sum(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                                                      const T* __restrict__ q, const T* __restrict__ rhs,
                                                      const T* __restrict__ x0, u32 m, int R,
                                                      double* __restrict__ cta_part, CgState st, CgLoop lp) {
    __shared__ double red[3 * TB];
    if (R > WIDE_R) {
        for (int c = threadIdx.x; c < R; c += blockDim.x) {
            const T g = T(st.gamma[c]);
            double xb = 0.0, xr = 0.0, x0r = 0.0;
            for (u32 i = blockIdx.x; i < m; i += gridDim.x) {
                const size_t o = size_t(i) * R + c;
                const T xv = x[o] + g * p[o];
                const T rv = r[o] - g * q[o];
                x[o] = xv;
                r[o] = rv;
                xb += double(xv) * double(rhs[o]);
                xr += double(xv) * double(rv);
                if (x0) x0r += double(x0[o]) * double(rv);
            }
            double* o = cta_part + size_t(blockIdx.x) * 3 * R + c;
            o[0] = xb;
            o[R] = xr;
            o[2 * R] = x0r;
        }
    } else
    for (int j0 = 0; j0 < R; j0 += RC_MAX) {
        const ColMap cm = colmap(R, j0);
        double xb = 0.0, xr = 0.0, x0r = 0.0;
        if (cm.on) {
            const T g = T(st.gamma[j0 + cm.col]);
            for (u32 i = blockIdx.x * u32(cm.nslot) + u32(cm.slot); i < m; i += gridDim.x * u32(cm.nslot)) {
                const size_t o = size_t(i) * R + j0 + cm.col;
                const T xv = x[o] + g * p[o];
                const T rv = r[o] - g * q[o];
                x[o] = xv;
                r[o] = rv;
                xb += double(xv) * double(rhs[o]);
                xr += double(xv) * double(rv);
                if (x0) x0r += double(x0[o]) * double(rv);
            }
        }
        red[threadIdx.x] = xb;
        red[TB + threadIdx.x] = xr;
        red[2 * TB + threadIdx.x] = x0r;
        __syncthreads();
        if (int(threadIdx.x) < cm.Rc) {
            double a = 0.0, b = 0.0, c = 0.0;
            for (int sl = 0; sl < cm.nslot; sl++) {
                a += red[sl * cm.Rc + threadIdx.x];
                b += red[TB + sl * cm.Rc + threadIdx.x];
                c += red[2 * TB + sl * cm.Rc + threadIdx.x];
            }
            double* o = cta_part + size_t(blockIdx.x) * 3 * R + j0 + threadIdx.x;
            o[0] = a;
            o[R] = b;
            o[2 * R] = c;
        }
        __syncthreads();
    }
    if (!last_cta(lp.ticket + 1)) return;
    cta_col_sums(cta_part, int(gridDim.x), 3 * R, R, st.xb);
    if (threadIdx.x == 0) lp.ticket[1] = 0;
}

// rho_new = r'z, then the stopping rule (cg.rs:239-253) and beta with the device iteration counter;
// the probe's contraction inputs are recorded at PROBE_FROM and PROBE_AT.
template <class T>
__global__ void __launch_bounds__(TB) k_rz_stop(const T* __restrict__ r, const T* __restrict__ z, u32 m, int R,
                                                double* __restrict__ cta_part, CgState st, CgLoop lp, int probe_from,
                                                int probe_at) {
    __shared__ double red[TB];
    __shared__ int cnt, kk;
    dot_partials(r, z, m, R, cta_part, red);
    if (!last_cta(lp.ticket + 2)) return;
    cta_col_sums(cta_part, int(gridDim.x), R, R, st.rho_new);
    if (threadIdx.x == 0) {
        cnt = 0;
        kk = ++lp.ctl[1];
    }
    __syncthreads();
    const int k = kk;
    const double tol = *lp.tol;
    int local = 0;
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
        double beta = 0.0;
        if (st.active[j] == 1) {
            double* ring = st.ring + size_t(j) * WINDOW;
            ring[(k - 1) % WINDOW] = st.gamma[j] * st.rho[j];
            const double ssk = st.ss1[j] - (st.xconst[j] + st.xb[j] + st.xb[R + j] + st.xb[2 * R + j]);
            const double thr = fmax(tol * tol * ssk, st.floor_[j]);
            double sum = 0.0;
            for (int w = 0; w < WINDOW; w++) sum += ring[w];
            const double rn = st.rho_new[j];
            const bool done = k >= WINDOW && sum <= thr;
            const bool at_roundoff = rn <= st.floor_[j];
            // In an FP32 round (pfloor > 0) a breakdown or the FP32 round-off floor ends the round
            // with another FP64 restart (state 2); only the window rule stops the column.
            if (done) st.active[j] = 0;
            else if (at_roundoff || !(rn > 0.0)) st.active[j] = st.pfloor[j] > 0.0 ? 2 : 0;
            else if (rn <= st.pfloor[j]) st.active[j] = 2;
            else beta = rn / st.rho[j];
        }
        st.beta[j] = beta;
        st.rho[j] = st.rho_new[j];
        if (k == probe_from) lp.rho_from[j] = st.rho[j];
        if (k == probe_at) {
            lp.rho_at[j] = st.rho[j];
            lp.act_at[j] = st.active[j];
        }
        local += st.active[j] == 1;
    }
    atomicAdd(&cnt, local);  // integer count: order independent
    __syncthreads();
    if (threadIdx.x == 0) {
        *st.n_active = cnt;
        lp.ctl[0] = cnt;
        lp.ticket[2] = 0;
    }
}

// The first condition of a graph launch's WHILE node (a node before it): iterate while some
// column is active and the launch's cap allows one iteration.
__global__ void k_cond_first(cudaGraphConditionalHandle cond, const int* __restrict__ n_active, CgLoop lp) {
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, (*n_active > 0 && lp.ctl[3] > 0) ? 1u : 0u);
}

// p = z + beta p on the active columns, 0 on the others; then the iteration's end: the launch's
// iteration count rises and, in a graph, the WHILE condition is set for the next iteration.
template <class T>
__global__ void k_update_p_cond(T* __restrict__ p, const T* __restrict__ z, const double* __restrict__ beta,
                                const int* __restrict__ active, u32 m, int R, CgLoop lp,
                                cudaGraphConditionalHandle cond, int use_cond) {
    const size_t total = size_t(m) * R;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int j = int(i % R);
        p[i] = active[j] == 1 ? z[i] + T(beta[j]) * p[i] : T(0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int kl = ++lp.ctl[2];
        if (use_cond) cudaGraphSetConditional(cond, (lp.ctl[0] > 0 && kl < lp.ctl[3]) ? 1u : 0u);
    }
}

}  // namespace fereg
