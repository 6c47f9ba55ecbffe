// Row passes of the GLM IRLS (glm/irls.rs:367-560, glm/family.rs) for Poisson and logit: start values, the
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

// Partials of sum y; flag = 1 when a y is out of the family's range (Poisson: y >= 0; logit:
// y in {0, 1}).
__global__ void __launch_bounds__(GLM_TB) k_glm_ysum(const double* __restrict__ raw, size_t n, int R, int fam,
                                                     double* __restrict__ part, int* flag) {
    __shared__ double red[GLM_TB];
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double y = raw[i * R];
        if (fam == 0 ? !(y >= 0.0) : !(y == 0.0 || y == 1.0)) atomicExch(flag, 1);
        s += y;
    }
    const double t = glm_block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Lower bound of mu (100 machine epsilons); logit also caps mu at 1 - GLM_MU_MIN (family.rs:13).
constexpr double GLM_MU_MIN = 100.0 * 2.220446049250313e-16;

// Families (glm/family.rs): 0 Poisson (log link), 1 logit (logit link).
__device__ __forceinline__ double glm_link(int fam, double m) { return fam == 0 ? log(m) : log(m / (1.0 - m)); }

// ln(1 + e^x) without overflow.
__device__ __forceinline__ double glm_softplus(double x) { return fmax(x, 0.0) + log1p(exp(-fabs(x))); }

// mu of a row from eta, clamped (family.rs:103-113), and the row's term of the deviance / 2:
// Poisson (mu - y) + y (ln y - eta) (the second term 0 at y = 0), logit softplus(eta) - y eta
// (on the unclamped eta, irls.rs:252-266).
__device__ __forceinline__ double glm_mu_dev(int fam, double et, double y, double& m) {
    if (fam == 0) {
        const double x = exp(et);
        m = x >= GLM_MU_MIN ? x : GLM_MU_MIN;
        return (m - y) + (y > 0.0 ? y * (log(y) - et) : 0.0);
    }
    const double p = 1.0 / (1.0 + exp(-et));
    m = fmin(fmax(p, GLM_MU_MIN), 1.0 - GLM_MU_MIN);
    return glm_softplus(et) - y * et;
}

// Start: Poisson (the `simple` guess) mu = (y + mean y) / 2, logit mu = (y + 1/2) / 2
// (glm/mod.rs:816-820); `center` is mean y or 1/2. eta = link(mu).
__global__ void k_glm_start(const double* __restrict__ raw, size_t n, int R, double center, int fam,
                            double* __restrict__ mu, double* __restrict__ eta) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double m = 0.5 * (raw[i * R] + center);
        mu[i] = m;
        eta[i] = glm_link(fam, m);
    }
}

// Working variable and weight (family.rs irls_weight / working): Poisson w = mu,
// z = eta - 1 + y / mu; logit w = mu (1 - mu), z = eta + (y - mu) / w. The block B = [z, X]
// (R columns) takes z and a fresh copy of X from the raw block `raw` ([y, X], R columns).
__global__ void k_glm_work(const double* __restrict__ raw, size_t n, int R, int fam, const double* __restrict__ mu,
                           const double* __restrict__ eta, double* __restrict__ B, double* __restrict__ z,
                           double* __restrict__ w) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double m = mu[i], y = raw[i * R];
        const double wi = fam == 0 ? m : m * (1.0 - m);
        const double zi = fam == 0 ? eta[i] - 1.0 + y / m : eta[i] + (y - m) / wi;
        z[i] = zi;
        w[i] = wi;
        B[i * R] = zi;
        for (int j = 1; j < R; j++) B[i * R + j] = raw[i * R + j];
    }
}

// eta = z - e (the fitted linear predictor of the weighted regression), mu from eta, and partials
// of the deviance / 2 (glm_mu_dev); `old` (non-null) saves the previous eta first.
__global__ void __launch_bounds__(GLM_TB) k_glm_update(const double* __restrict__ raw, size_t n, int R, int fam,
                                                       const double* __restrict__ z, const double* __restrict__ e,
                                                       double* __restrict__ eta, double* __restrict__ old,
                                                       double* __restrict__ mu, double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double dev = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double et = z[i] - e[i];
        if (old) old[i] = eta[i];
        double m;
        dev += glm_mu_dev(fam, et, raw[i * R], m);
        eta[i] = et;
        mu[i] = m;
    }
    const double s = glm_block_sum(dev, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// One step halving toward the previous eta (irls.rs:739-748): eta = (eta + old) / 2, mu and the
// deviance partials again.
__global__ void __launch_bounds__(GLM_TB) k_glm_halve(const double* __restrict__ raw, size_t n, int R, int fam,
                                                      const double* __restrict__ old, double* __restrict__ eta,
                                                      double* __restrict__ mu, double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double dev = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double et = 0.5 * (eta[i] + old[i]);
        double m;
        dev += glm_mu_dev(fam, et, raw[i * R], m);
        eta[i] = et;
        mu[i] = m;
    }
    const double s = glm_block_sum(dev, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Partials of the log-likelihood: Poisson sum [y eta - mu - lgamma(y + 1)], logit
// sum [y eta - softplus(eta)] (family.rs:143-147).
__global__ void __launch_bounds__(GLM_TB) k_glm_ll(const double* __restrict__ raw, size_t n, int R, int fam,
                                                   const double* __restrict__ eta, const double* __restrict__ mu,
                                                   double* __restrict__ part) {
    __shared__ double red[GLM_TB];
    double ll = 0.0;
    for (size_t i = size_t(blockIdx.x) * GLM_TB + threadIdx.x; i < n; i += size_t(gridDim.x) * GLM_TB) {
        const double y = raw[i * R];
        if (fam == 0) ll += y * eta[i] - mu[i] - lgamma(y + 1.0);
        else ll += y * eta[i] - glm_softplus(eta[i]);
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
