// Row passes of the variances beyond CRV1: the CRV3 jackknife's per-cluster Gram of the
// residualized columns for its closed form (crv3.rs:226-426), and the HC2 / HC3 meat weights.
#pragma once

#include "device.cuh"

namespace fereg {

// out[g][a][b] = sum over cluster g's rows (perm order) of w_i a_i[col[a]] a_i[col[b]], one CTA
// per cluster at a time, one thread per entry (the rows in order).
__global__ void k_cluster_grams(const double* __restrict__ rows, int R, const int* __restrict__ col, int k,
                                const double* __restrict__ w, const int* __restrict__ perm,
                                const u32* __restrict__ coff, u32 G, double* __restrict__ out) {
    for (u32 g = blockIdx.x; g < G; g += gridDim.x)
        for (int q = threadIdx.x; q < k * k; q += blockDim.x) {
            const int a = col[q / k], b = col[q % k];
            double s = 0.0;
            for (u32 t = coff[g]; t < coff[g + 1]; t++) {
                const size_t i = size_t(perm[t]);
                s += (w ? w[i] : 1.0) * rows[i * R + a] * rows[i * R + b];
            }
            out[size_t(g) * k * k + q] = s;
        }
}

// dst row t = columns col[0..k) of src row idx[t] (src R columns), dst k columns.
__global__ void k_gather_cols(const double* __restrict__ src, int R, const u32* __restrict__ idx, size_t m,
                              const int* __restrict__ col, int k, double* __restrict__ dst) {
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < m * k; q += size_t(gridDim.x) * blockDim.x) {
        const size_t t = q / k;
        dst[q] = src[size_t(idx[t]) * R + col[q % k]];
    }
}

// The regress HC2 / HC3 meat weights (ols.rs:456-470, ols/stata_vce.rs:156-167): h = h_fe +
// w_v x~'A x~ over the kept columns col[0..k) (A the raw (X~'WX~)^-1), s = e w_v, tau = w_v with
// fweights else 1; HC2 s^2 / (tau - h), HC3 tau s^2 / (tau - h)^2, 0 when tau - h <= sqrt(eps) tau.
__global__ void k_hc_weights(const double* __restrict__ rows, int R, const int* __restrict__ col, int k,
                             const double* __restrict__ A, const double* __restrict__ e, const double* __restrict__ wv,
                             const double* __restrict__ hfe, int fw, int hc3, size_t n, double* __restrict__ om) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double* row = rows + i * R;
        double q = 0.0;
        for (int p = 0; p < k; p++) {
            double acc = 0.0;
            for (int c = 0; c < k; c++) acc += A[p * k + c] * row[col[c]];
            q += row[col[p]] * acc;
        }
        const double w = wv ? wv[i] : 1.0;
        const double h = hfe[i] + w * q;
        const double s = e[i] * w;
        const double tau = fw ? w : 1.0;
        const double d = tau - h;
        om[i] = d <= 1.4901161193847656e-08 * tau ? 0.0 : (hc3 ? tau * s * s / (d * d) : s * s / d);
    }
}

}  // namespace fereg
