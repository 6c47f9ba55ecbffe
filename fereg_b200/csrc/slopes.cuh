// Device passes of the heterogeneous-slope absorber (slopes.h): the segment pass over the
// levels of the eliminated term E (slopes.rs:1025-1137 seg_task, 1161-1262 resid_task), the
// coordinate pass over the coordinate-sorted slot lists, and the block-Jacobi preconditioner
// (slopes.rs:1996 SPre::apply on its Jacobi blocks). One thread per (level or coordinate or
// unit, column) with the rows in order: every sum has a fixed order.
#pragma once

#include "device.cuh"

namespace fereg {

constexpr int SL_BE_MAX = 8;  // width (intercept + slopes) of the eliminated term
constexpr int SL_B_MAX = 8;   // width of the other terms
constexpr int SL_TB = 256;

struct SlopeDev {
    u32 n, ge, k, m, be, e_ns;
    int e_icpt;
    const u32* seg_off;  // ge + 1
    const u32* sc;       // n x k
    const double* sv;    // n x k
    const double* he;    // n x e_ns
    const double* w;     // n, or null (1)
    const double* minv;  // ge x be^2
};

enum SlMode { SL_APPLY = 0, SL_RHS = 1, SL_RESID = 2 };

// Design value l of E in row i: (1?, slopes...).
__device__ __forceinline__ double sl_he(const SlopeDev& D, u32 i, int l) {
    if (D.e_icpt) return l == 0 ? 1.0 : D.he[size_t(i) * D.e_ns + (l - 1)];
    return D.he[size_t(i) * D.e_ns + l];
}

// The loaded value of row i in column j: APPLY u_i = sum_slots v P[c] (P = src, m x lds); RHS the
// row (src, n x lds); RESID d_i = v_i - u_i(x) (x: m x ldx, or null when m = 0).
template <int MODE>
__device__ __forceinline__ double sl_load(const SlopeDev& D, u32 i, int j, const double* __restrict__ src, int lds,
                                          const double* __restrict__ x, int ldx) {
    if constexpr (MODE == SL_RHS) {
        return src[size_t(i) * lds + j];
    } else {
        const double* P = MODE == SL_APPLY ? src : x;
        const int ld = MODE == SL_APPLY ? lds : ldx;
        double u = 0.0;
        if (P)
            for (u32 t = 0; t < D.k; t++) {
                const size_t e = size_t(i) * D.k + t;
                u += D.sv[e] * P[size_t(D.sc[e]) * ld + j];
            }
        if constexpr (MODE == SL_APPLY) return u;
        else return src[size_t(i) * lds + j] - u;
    }
}

// The segment pass over levels s of E and columns j < C:
//   t = M_s^+ sum_i w_i h_E,i y_i,  e_i = y_i - h_E,i' t,
// APPLY / RHS: Z[i, j] = w_i e_i (n x ldz); RHS also the per-level partials [sum w y^2, sum w y,
// sum w e^2] (part: ge x 3C); RESID: the row becomes e_i (in place) and alpha[s be + l, j] = t_l.
template <int MODE>
__global__ void __launch_bounds__(SL_TB) k_sl_seg(SlopeDev D, const double* src, int lds, int C,
                                                   const double* __restrict__ x, int ldx, double* __restrict__ Z,
                                                   int ldz, double* rows_out, double* __restrict__ alpha, int lda,
                                                   double* __restrict__ part) {
    const size_t total = size_t(D.ge) * C;
    const int be = int(D.be);
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const u32 s = u32(q / C);
        const int j = int(q % C);
        const u32 r0 = D.seg_off[s], r1 = D.seg_off[s + 1];
        double a[SL_BE_MAX], t[SL_BE_MAX];
#pragma unroll
        for (int l = 0; l < SL_BE_MAX; l++) a[l] = 0.0;
        double swv2 = 0.0, swv = 0.0, swe2 = 0.0;
        for (u32 i = r0; i < r1; i++) {
            const double y = sl_load<MODE>(D, i, j, src, lds, x, ldx);
            const double wi = D.w ? D.w[i] : 1.0;
#pragma unroll
            for (int l = 0; l < SL_BE_MAX; l++)
                if (l < be) a[l] += wi * sl_he(D, i, l) * y;
            if constexpr (MODE == SL_RHS) {
                swv2 += wi * y * y;
                swv += wi * y;
            }
        }
        const double* mv = D.minv + size_t(s) * be * be;
#pragma unroll
        for (int l = 0; l < SL_BE_MAX; l++) {
            double v = 0.0;
            if (l < be)
                for (int l2 = 0; l2 < be; l2++) {
                    const double c = mv[l * be + l2];
                    if (c != 0.0) v += c * a[l2];
                }
            t[l] = v;
        }
        for (u32 i = r0; i < r1; i++) {
            const double y = sl_load<MODE>(D, i, j, src, lds, x, ldx);
            double e = y;
#pragma unroll
            for (int l = 0; l < SL_BE_MAX; l++)
                if (l < be) e -= sl_he(D, i, l) * t[l];
            if constexpr (MODE == SL_RESID) {
                rows_out[size_t(i) * lds + j] = e;
            } else {
                const double wi = D.w ? D.w[i] : 1.0;
                Z[size_t(i) * ldz + j] = wi * e;
                if constexpr (MODE == SL_RHS) swe2 += wi * e * e;
            }
        }
        if constexpr (MODE == SL_RESID) {
            if (alpha)
                for (int l = 0; l < be; l++) alpha[(size_t(s) * be + l) * lda + j] = t[l];
        }
        if constexpr (MODE == SL_RHS) {
            double* pp = part + size_t(s) * 3 * C;
            pp[j] = swv2;
            pp[C + j] = swv;
            pp[2 * C + j] = swe2;
        }
    }
}

// The coordinate pass: Y[c, j] = sum over the list of coordinate c of v Z[row, j], c < m, j < C.
__global__ void __launch_bounds__(SL_TB) k_sl_pull(u32 m, int C, const u32* __restrict__ pl_off,
                                                    const u32* __restrict__ pl_row, const double* __restrict__ pl_val,
                                                    const double* __restrict__ Z, int ldz, double* __restrict__ Y,
                                                    int ldy) {
    const size_t total = size_t(m) * C;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const u32 c = u32(q / C);
        const int j = int(q % C);
        double acc = 0.0;
        for (u32 e = pl_off[c]; e < pl_off[c + 1]; e++) acc += pl_val[e] * Z[size_t(pl_row[e]) * ldz + j];
        Y[size_t(c) * ldy + j] = acc;
    }
}

// z = J r per block-Jacobi unit (b consecutive coordinates from c0, inverse at joff, b x b).
__global__ void __launch_bounds__(SL_TB) k_sl_jacobi(u32 nunits, int C, const u32* __restrict__ c0,
                                                      const u32* __restrict__ bw, const u32* __restrict__ joff,
                                                      const double* __restrict__ J, const double* __restrict__ r,
                                                      double* __restrict__ z, int ld) {
    const size_t total = size_t(nunits) * C;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const u32 u = u32(q / C);
        const int j = int(q % C);
        const u32 b = bw[u], base = c0[u];
        const double* Ju = J + joff[u];
        double rr[SL_B_MAX];
#pragma unroll
        for (int a = 0; a < SL_B_MAX; a++) rr[a] = a < int(b) ? r[size_t(base + a) * ld + j] : 0.0;
        for (u32 a = 0; a < b; a++) {
            double v = 0.0;
#pragma unroll
            for (int bb = 0; bb < SL_B_MAX; bb++)
                if (bb < int(b)) v += Ju[a * b + bb] * rr[bb];
            z[size_t(base + a) * ld + j] = v;
        }
    }
}

}  // namespace fereg
