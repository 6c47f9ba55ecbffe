// Row passes of the Poisson PML IRLS (glm/irls.rs:367-560, glm/family.rs): start values, the
// working variable and weights, the linear-predictor update with the deviance, and the
// log-likelihood. Per-CTA partials combined in a fixed order.
#pragma once

#include "device.cuh"

namespace fereg {

constexpr int GLM_TB = 256;

__device__ __forceinline__ double glm_block_sum(double v, double* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int h = GLM_TB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    return red[0];
}

// Partials of sum y and the count of negative y (y = column 0 of the raw block [y, X]).
__global__ void __launch_bounds__(GLM_TB) k_glm_ysum(const double* __restrict__ raw, size_t n, int R,
                                                     double* __restrict__ part, int* neg) {
    __shared__ double red[GLM_TB];
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double y = raw[i * R];
        if (!(y >= 0.0)) atomicExch(neg, 1);
        s += y;
    }
    const double t = glm_block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Start (ppmlhdfe `simple` guess): mu = (y + mean y) / 2, eta = log mu.
__global__ void k_glm_start(const double* __restrict__ raw, size_t n, int R, double ybar, double* __restrict__ mu,
                            double* __restrict__ eta) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double m = 0.5 * (raw[i * R] + ybar);
        mu[i] = m;
        eta[i] = log(m);
    }
}

// Poisson working variable z = eta - 1 + y / mu and weight w = mu; the block B = [z, X] (R
// columns) takes z and a fresh copy of X from the raw block `raw` ([y, X], R columns).
__global__ void k_glm_work(const double* __restrict__ raw, size_t n, int R, const double* __restrict__ mu,
                           const double* __restrict__ eta, double* __restrict__ B, double* __restrict__ z,
                           double* __restrict__ w) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double m = mu[i], zi = eta[i] - 1.0 + raw[i * R] / m;
        z[i] = zi;
        w[i] = m;
        B[i * R] = zi;
        for (int j = 1; j < R; j++) B[i * R + j] = raw[i * R + j];
    }
}

// eta = z - e (the fitted linear predictor of the weighted regression), mu = exp(eta); partials
// of the deviance 2 sum [y log(y / mu) - (y - mu)] (the y log y term is 0 at y = 0).
__global__ void __launch_bounds__(GLM_TB) k_glm_update(const double* __restrict__ raw, size_t n, int R,
                                                       const double* __restrict__ z, const double* __restrict__ e,
                                                       double* __restrict__ eta, double* __restrict__ mu,
                                                       double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double dev = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double et = z[i] - e[i], m = exp(et), y = raw[i * R];
        eta[i] = et;
        mu[i] = m;
        dev += 2.0 * ((y > 0.0 ? y * (log(y) - et) : 0.0) - (y - m));
    }
    const double s = glm_block_sum(dev, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Partials of the Poisson log-likelihood sum [y eta - mu - lgamma(y + 1)].
__global__ void __launch_bounds__(GLM_TB) k_glm_ll(const double* __restrict__ raw, size_t n, int R,
                                                   const double* __restrict__ eta, const double* __restrict__ mu,
                                                   double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double ll = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double y = raw[i * R];
        ll += y * eta[i] - mu[i] - lgamma(y + 1.0);
    }
    const double s = glm_block_sum(ll, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Score weights of the sandwich: om = (e w)^2 (robust) or e w (cluster scores).
__global__ void k_glm_score(const double* __restrict__ e, const double* __restrict__ w, size_t n, int squared,
                            double* __restrict__ om) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double s = e[i] * w[i];
        om[i] = squared ? s * s : s;
    }
}

}  // namespace fereg
