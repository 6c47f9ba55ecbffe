// Row passes of the ReLU separation check (glm/separation.rs:61-196, ppmlhdfe 2.3.3
// relu_fix_separation): the working block [u, X / sd], the weights of the method of weighting,
// the column norms of X on either sample, and one step's prediction, thresholds and counts. Per-CTA
// partials combined in a fixed order on the host.
#pragma once

#include "glm.cuh"

namespace fereg {

// Partials per CTA of one ReLU step (k_relu_step): boundary rows with a negative prediction,
// with a positive one, the smallest boundary residual, and the sum of the negative predictions.
constexpr int RELU_PARTS = 4;

// Unweighted sums of x and x^2 per regressor (columns 1..R-1 of the raw block), per CTA
// (part[cta][2 (R - 1)]): the standard deviations of the standardization (glm/mod.rs:4-6).
__global__ void __launch_bounds__(GLM_TB) k_relu_colsums(const double* __restrict__ raw, size_t n, int R,
                                                         double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    const int k = R - 1;
    for (int j = 0; j < k; j++)
        for (int pw = 1; pw <= 2; pw++) {
            double s = 0.0;
            for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
                const double x = raw[i * R + 1 + j];
                s += pw == 1 ? x : x * x;
            }
            const double t = glm_block_sum(s, red);
            if (threadIdx.x == 0) part[size_t(blockIdx.x) * 2 * k + (pw - 1) * k + j] = t;
            __syncthreads();
        }
}

// The standardized regressors X / sd (n x k), the weights (M on y > 0, 1 on y = 0), the start
// u = 1[y = 0], and per CTA the sums of |x / sd| per column over the non-boundary and the
// boundary rows (part[cta][2 k]: Mata norm(X, 1) of either sample).
__global__ void __launch_bounds__(GLM_TB) k_relu_init(const double* __restrict__ raw, size_t n, int R,
                                                      const double* __restrict__ sd, double big_m,
                                                      double* __restrict__ xs, double* __restrict__ w,
                                                      double* __restrict__ u, double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    const int k = R - 1;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const bool bd = raw[i * R] == 0.0;
        w[i] = bd ? 1.0 : big_m;
        u[i] = bd ? 1.0 : 0.0;
        for (int j = 0; j < k; j++) xs[i * k + j] = raw[i * R + 1 + j] / sd[j];
    }
    for (int j = 0; j < k; j++)
        for (int smp = 0; smp < 2; smp++) {
            double s = 0.0;
            for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB)
                if ((raw[i * R] == 0.0) == (smp == 1)) s += fabs(raw[i * R + 1 + j] / sd[j]);
            const double t = glm_block_sum(s, red);
            if (threadIdx.x == 0) part[size_t(blockIdx.x) * 2 * k + smp * k + j] = t;
            __syncthreads();
        }
}

// The block of one step: B = [u, X / sd] (n x R), and per CTA sum u^2.
__global__ void __launch_bounds__(GLM_TB) k_relu_block(const double* __restrict__ u, const double* __restrict__ xs,
                                                       size_t n, int R, double* __restrict__ B,
                                                       double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    const int k = R - 1;
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double v = u[i];
        B[i * R] = v;
        for (int j = 0; j < k; j++) B[i * R + 1 + j] = xs[i * k + j];
        s += v * v;
    }
    const double t = glm_block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// One step on the residualized block Bt: resid = u~ - X~ b, xbd = u - resid, 0 off the boundary
// and inside [-0.1 delta, delta]; per CTA [boundary rows with xbd < 0, with xbd > 0, min over the
// boundary of resid (0 within zero_tol), sum of -xbd over the negative boundary rows].
__global__ void __launch_bounds__(GLM_TB) k_relu_step(const double* __restrict__ raw, const double* __restrict__ Bt,
                                                      const double* __restrict__ u, size_t n, int R, int rawR,
                                                      const double* __restrict__ b, const int* __restrict__ kept,
                                                      int nk, double delta, double zero_tol,
                                                      double* __restrict__ resid, double* __restrict__ xbd,
                                                      double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double neg = 0.0, pos = 0.0, mn = INFINITY, negsum = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        double e = Bt[i * R];
        for (int a = 0; a < nk; a++) e -= b[a] * Bt[i * R + kept[a]];
        const bool bd = raw[i * rawR] == 0.0;
        double x = u[i] - e;
        if (!bd || (-0.1 * delta <= x && x <= delta)) x = 0.0;
        xbd[i] = x;
        const double ez = fabs(e) <= zero_tol ? 0.0 : e;
        resid[i] = ez;
        if (bd) {
            neg += x < 0.0;
            pos += x > 0.0;
            mn = fmin(mn, ez);
            if (x < 0.0) negsum += -x;
        }
    }
    double v[RELU_PARTS] = {neg, pos, mn, negsum};
    for (int q = 0; q < RELU_PARTS; q++) {
        red[threadIdx.x] = v[q];
        __syncthreads();
        for (int h = GLM_TB / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h)
                red[threadIdx.x] = q == 2 ? fmin(red[threadIdx.x], red[threadIdx.x + h]) : red[threadIdx.x] + red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[size_t(blockIdx.x) * RELU_PARTS + q] = red[0];
        __syncthreads();
    }
}

// No negative boundary residual: boundary rows whose residual exceeds delta leave the
// certificate; per CTA the boundary rows with xbd > 0 that remain.
__global__ void __launch_bounds__(GLM_TB) k_relu_trim(const double* __restrict__ raw, size_t n, int rawR,
                                                      const double* __restrict__ resid, double delta,
                                                      double* __restrict__ xbd, double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double pos = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        if (raw[i * rawR] != 0.0) continue;
        if (resid[i] > delta) xbd[i] = 0.0;
        pos += xbd[i] > 0.0;
    }
    const double t = glm_block_sum(pos, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// The ReLU update of the working variable on the boundary: u = max(xbd, 0).
__global__ void k_relu_update(const double* __restrict__ raw, size_t n, int rawR, const double* __restrict__ xbd,
                              double* __restrict__ u) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        if (raw[i * rawR] == 0.0) u[i] = fmax(xbd[i], 0.0);
}

// The outputs: separated (boundary with xbd > 0) and the certificate (xbd there, 0 elsewhere).
__global__ void k_relu_out(const double* __restrict__ raw, size_t n, int rawR, const double* __restrict__ xbd,
                           uint8_t* __restrict__ sep, double* __restrict__ cert) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const bool s = raw[i * rawR] == 0.0 && xbd[i] > 0.0;
        sep[i] = s ? 1 : 0;
        cert[i] = s ? xbd[i] : 0.0;
    }
}

}  // namespace fereg
