// Device kernels of the wild cluster bootstrap (WCR11, wildboot/ols.rs:243-650).
//
// A tile of bt draws b0..b0+bt-1 is one n x bt block: column b holds v_{g(i),b} e_r,i, the
// restricted residuals flipped by the draw's cluster signs. The absorber residualizes the block
// (all draws as columns of one block PCG). The slopes need no solve: by linearity
// beta*_b - beta_r = A sum_g v_{g,b} phi_g, phi_g = sum_{i in g} w_i e_r,i x~_i. The variance of
// coefficient j needs the residualized draws only through the cluster sums
// T1[g][b] = sum_{i in g} w_i c_i z~_{i,b}, c_i = a' x~_i (a = row j of A):
// V_b = scale * sum over cluster subsets s (sign_s) of sum_g (T1_s[g][b] - psi_{s,g}' d_b)^2,
// d_b = beta*_b - beta_r, psi_{s,g} = sum_{i in g} w_i c_i x~_i.
// Every sum has a fixed order.
#pragma once

#include "device.cuh"

namespace fereg {

constexpr int BOOT_TB = 256;
constexpr int BOOT_MAX_SUB = 8;

// SplitMix64 (rng.rs:4-31). Draw b reads the stream (seed, b) of rng.rs `stream`: state seed ^
// b * 0xD1B54A32D192ED03, one output skipped; its w-th used 64-bit word is therefore the output
// at state + (w + 2) * 0x9E3779B97F4A7C15.
__device__ __forceinline__ u64 splitmix_out(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// W[col][w]: the sign bits of draw b0 + col for clusters 64w..64w+63 (bit set = -1), from the
// draw's stream (weights.rs:65-79, LSB first) or, under full enumeration, the bits of b.
__global__ void k_boot_words(u64 seed, u64 b0, u32 bt, u32 nwords, int full_enum, u64* __restrict__ W) {
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < size_t(bt) * nwords;
         idx += size_t(gridDim.x) * blockDim.x) {
        const u64 b = b0 + idx / nwords, w = idx % nwords;
        if (full_enum) {
            W[idx] = w == 0 ? b : 0ull;
        } else {
            const u64 st = seed ^ (b * 0xD1B54A32D192ED03ull);
            W[idx] = splitmix_out(st + (w + 2) * 0x9E3779B97F4A7C15ull);
        }
    }
}

__device__ __forceinline__ double boot_sign(const u64* W, u32 nwords, u32 col, u32 g) {
    return (W[size_t(col) * nwords + (g >> 6)] >> (g & 63)) & 1ull ? -1.0 : 1.0;
}

// Z[i][col] = v_{g(i), b0 + col} e_r[i] (row order, n x bt row-major).
__global__ void k_boot_gen(size_t n, u32 bt, const double* __restrict__ er, const u32* __restrict__ bcode,
                           const u64* __restrict__ W, u32 nwords, double* __restrict__ Z) {
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < n * bt; idx += size_t(gridDim.x) * blockDim.x) {
        const size_t i = idx / bt;
        const u32 col = u32(idx % bt);
        Z[idx] = boot_sign(W, nwords, col, bcode[i]) * er[i];
    }
}

// U[col][p] = sum_g v_{g,col} Phi[g][p] (g in order); one thread per (col, p).
__global__ void k_boot_u(u32 bt, u32 G, int k, const u64* __restrict__ W, u32 nwords, const double* __restrict__ Phi,
                         double* __restrict__ U) {
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < size_t(bt) * k;
         idx += size_t(gridDim.x) * blockDim.x) {
        const u32 col = u32(idx / k);
        const int p = int(idx % k);
        double s = 0.0;
        for (u32 g = 0; g < G; g++) s += boot_sign(W, nwords, col, g) * Phi[size_t(g) * k + p];
        U[idx] = s;
    }
}

// D[col][p] = sum_q A[p][q] U[col][q].
__global__ void k_boot_delta(u32 bt, int k, const double* __restrict__ A, const double* __restrict__ U,
                             double* __restrict__ D) {
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < size_t(bt) * k;
         idx += size_t(gridDim.x) * blockDim.x) {
        const size_t col = idx / k;
        const int p = int(idx % k);
        double s = 0.0;
        for (int q = 0; q < k; q++) s += A[p * k + q] * U[col * k + q];
        D[idx] = s;
    }
}

// T1[g][col] = sum over the rows of cluster g (perm[coff[g] .. coff[g+1]], in order) of
// cw[row] Z[row][col]; a warp per (cluster, 32 columns), lane = column.
__global__ void k_boot_t1(const double* __restrict__ Z, u32 bt, const double* __restrict__ cw,
                          const int* __restrict__ perm, const u32* __restrict__ coff, u32 G, double* __restrict__ T1) {
    const u32 chunks = (bt + 31) / 32;
    const u32 lane = threadIdx.x & 31;
    const size_t gw = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5, nw = (size_t(gridDim.x) * blockDim.x) >> 5;
    for (size_t t = gw; t < size_t(G) * chunks; t += nw) {
        const u32 g = u32(t / chunks), col = u32(t % chunks) * 32 + lane;
        if (col >= bt) continue;
        double s = 0.0;
        for (u32 q = coff[g]; q < coff[g + 1]; q++) {
            const size_t row = size_t(perm[q]);
            s += cw[row] * Z[row * bt + col];
        }
        T1[size_t(g) * bt + col] = s;
    }
}

struct BootSubsets {
    const double* T1[BOOT_MAX_SUB];   // G_s x bt
    const double* Psi[BOOT_MAX_SUB];  // G_s x k
    u32 G[BOOT_MAX_SUB];
    double sign[BOOT_MAX_SUB];
    int n;
};

// t[col] = D[col][j] / sqrt(scale * V_col), V as above; a CTA per draw, clusters dealt to the
// threads in turn and combined by a fixed tree. NaN when V is not positive.
__global__ void __launch_bounds__(BOOT_TB) k_boot_var(u32 bt, BootSubsets subs, const double* __restrict__ D, int k,
                                                      int j, double scale, double* __restrict__ t) {
    __shared__ double red[BOOT_TB];
    for (u32 col = blockIdx.x; col < bt; col += gridDim.x) {
        double v = 0.0;
        for (int s = 0; s < subs.n; s++) {
            double acc = 0.0;
            for (u32 g = threadIdx.x; g < subs.G[s]; g += BOOT_TB) {
                double d = subs.T1[s][size_t(g) * bt + col];
                for (int p = 0; p < k; p++) d -= subs.Psi[s][size_t(g) * k + p] * D[size_t(col) * k + p];
                acc += d * d;
            }
            red[threadIdx.x] = acc;
            __syncthreads();
            for (int h = BOOT_TB / 2; h > 0; h >>= 1) {
                if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
                __syncthreads();
            }
            v += subs.sign[s] * red[0];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const double var = scale * v;
            t[col] = var > 0.0 ? D[size_t(col) * k + j] / sqrt(var) : __longlong_as_double(0x7ff8000000000000ll);
        }
    }
}

// out[i] = a[i] * b[i] (b null: a[i]).
__global__ void k_mul(const double* __restrict__ a, const double* __restrict__ b, size_t n, double* __restrict__ out) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = b ? a[i] * b[i] : a[i];
}

}  // namespace fereg
