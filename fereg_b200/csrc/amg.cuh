// Device V-cycle of an escalated block (hierarchy built on the host, amg.h). Vectors are
// n_level x R row-major in the solve's precision T; matrix values stay FP64. One V(1,1) cycle
// from a zero start, four passes per level:
//   resid:    t_i  = r_i - sum_e a_ie dinv_c r_c           (Jacobi pre-smooth from 0, residual)
//   restrict: rc_I = sum_e Pt_Ie t_e                      (P^T t)
//   up1:      z1_i = dinv_i r_i + sum_e P_ie zc_e          (pre-smoothed value + prolongation)
//   up2:      z_i  = z1_i + dinv_i (r_i - sum_e a_ie z1_c)  (Jacobi post-smooth)
// and the coarsest level zc = Minv rc with its dense generalized inverse. Each pass reads only
// its own inputs, so no pass races with itself; every sum runs in a fixed order.
#pragma once

#include "device.cuh"

namespace fereg {

struct DevCsr {
    const u32* ptr;
    const u32* col;
    const double* val;
};

struct DevAmgLevel {
    u32 n;
    DevCsr A;
    const double* dinv;
    DevCsr P, Pt;  // null at the coarsest level
};

template <class T>
__global__ void k_amg_resid(DevAmgLevel L, const T* __restrict__ r, int R, T* __restrict__ t) {
    const size_t tot = size_t(L.n) * R;
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < tot; idx += size_t(gridDim.x) * blockDim.x) {
        const u32 i = u32(idx / R);
        const int j = int(idx % R);
        double v = double(r[idx]);
        for (u32 e = L.A.ptr[i]; e < L.A.ptr[i + 1]; e++) {
            const u32 c = L.A.col[e];
            v -= L.A.val[e] * L.dinv[c] * double(r[size_t(c) * R + j]);
        }
        t[idx] = T(v);
    }
}

template <class T>
__global__ void k_amg_restrict(DevCsr Pt, u32 nc, const T* __restrict__ t, int R, T* __restrict__ rc) {
    const size_t tot = size_t(nc) * R;
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < tot; idx += size_t(gridDim.x) * blockDim.x) {
        const u32 I = u32(idx / R);
        const int j = int(idx % R);
        double v = 0.0;
        for (u32 e = Pt.ptr[I]; e < Pt.ptr[I + 1]; e++) v += Pt.val[e] * double(t[size_t(Pt.col[e]) * R + j]);
        rc[idx] = T(v);
    }
}

template <class T>
__global__ void k_amg_up1(DevAmgLevel L, const T* __restrict__ r, const T* __restrict__ zc, int R, T* __restrict__ z1) {
    const size_t tot = size_t(L.n) * R;
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < tot; idx += size_t(gridDim.x) * blockDim.x) {
        const u32 i = u32(idx / R);
        const int j = int(idx % R);
        double v = L.dinv[i] * double(r[idx]);
        for (u32 e = L.P.ptr[i]; e < L.P.ptr[i + 1]; e++) v += L.P.val[e] * double(zc[size_t(L.P.col[e]) * R + j]);
        z1[idx] = T(v);
    }
}

template <class T>
__global__ void k_amg_up2(DevAmgLevel L, const T* __restrict__ r, const T* __restrict__ z1, int R, T* __restrict__ z) {
    const size_t tot = size_t(L.n) * R;
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < tot; idx += size_t(gridDim.x) * blockDim.x) {
        const u32 i = u32(idx / R);
        const int j = int(idx % R);
        const double di = L.dinv[i];
        if (di == 0.0) {
            z[idx] = T(0);
            continue;
        }
        double v = double(r[idx]);
        for (u32 e = L.A.ptr[i]; e < L.A.ptr[i + 1]; e++) v -= L.A.val[e] * double(z1[size_t(L.A.col[e]) * R + j]);
        z[idx] = T(double(z1[idx]) + di * v);
    }
}

// z = Minv r at the coarsest level (n x n generalized inverse).
template <class T>
__global__ void k_amg_dense(const double* __restrict__ minv, u32 n, const T* __restrict__ r, int R, T* __restrict__ z) {
    const size_t tot = size_t(n) * R;
    for (size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < tot; idx += size_t(gridDim.x) * blockDim.x) {
        const u32 i = u32(idx / R);
        const int j = int(idx % R);
        double v = 0.0;
        const double* row = minv + size_t(i) * n;
        for (u32 k = 0; k < n; k++) v += row[k] * double(r[size_t(k) * R + j]);
        z[idx] = T(v);
    }
}

}  // namespace fereg
