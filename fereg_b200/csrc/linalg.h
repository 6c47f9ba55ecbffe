// Small dense symmetric algebra of the OLS variance (K x K, K = regressors + 1), on the host:
// the reghdfe sweep inverse (vcov.rs:17-64 invsym in column order, :70 invsym_greedy in largest-
// pivot order), the constant's bordered inverse (vcov.rs:220 inv_ext), the sandwich
// (vcov.rs:254), and the eigenvalue clip of a multiway variance (vcov.rs:602-720 fix_psd, cyclic
// Jacobi rotations). Matrices are row-major std::vector<double>.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

namespace fereg {
namespace la {

using Mat = std::vector<double>;

inline void symmetrize(Mat& m, size_t k) {
    for (size_t i = 0; i < k; i++)
        for (size_t j = i + 1; j < k; j++) m[i * k + j] = m[j * k + i] = 0.5 * (m[i * k + j] + m[j * k + i]);
}

// One sweep step on pivot p with value d.
inline void sweep(Mat& m, size_t k, size_t p, double d) {
    double* rp = m.data() + p * k;
    for (size_t j = 0; j < k; j++) rp[j] /= d;
    for (size_t i = 0; i < k; i++) {
        if (i == p) continue;
        const double f = m[i * k + p];
        if (f == 0.0) continue;
        double* ri = m.data() + i * k;
        for (size_t j = 0; j < k; j++) ri[j] -= f * rp[j];
        ri[p] = -f / d;
    }
    rp[p] = 1.0 / d;
}

// Generalized inverse by sweeps. A pivot is dropped (its row and column zeroed) when it is NaN,
// non-positive or at most tol times its original diagonal. greedy: pivots in decreasing order
// of their current value, else in column order.
inline Mat sweep_inverse(const Mat& a, size_t k, double tol, bool greedy, std::vector<bool>& dropped) {
    Mat m = a;
    dropped.assign(k, false);
    std::vector<bool> done(k, false);
    for (size_t step = 0; step < k; step++) {
        size_t p = step;
        if (greedy) {
            p = k;
            for (size_t i = 0; i < k; i++)
                if (!done[i] && (p == k || m[i * k + i] > m[p * k + p])) p = i;
        }
        done[p] = true;
        const double d = m[p * k + p];
        if (std::isnan(d) || d <= 0.0 || d <= tol * a[p * k + p]) {
            dropped[p] = true;
            for (size_t j = 0; j < k; j++) m[p * k + j] = m[j * k + p] = 0.0;
            continue;
        }
        sweep(m, k, p, d);
    }
    symmetrize(m, k);
    return m;
}

// Inverse of the Gram bordered by the constant: inv is the k x k inverse of the centered Gram,
// means the column means, nc the constant's weight total.
inline Mat bordered(const Mat& inv, size_t k, const std::vector<double>& means, double nc) {
    const size_t k1 = k + 1;
    Mat out(k1 * k1, 0.0);
    std::vector<double> side(k, 0.0);
    for (size_t j = 0; j < k; j++) {
        double s = 0.0;
        for (size_t i = 0; i < k; i++) s += means[i] * inv[i * k + j];
        side[j] = -s;
    }
    double corner = 1.0 / nc;
    for (size_t j = 0; j < k; j++) corner -= side[j] * means[j];
    for (size_t i = 0; i < k; i++) {
        for (size_t j = 0; j < k; j++) out[i * k1 + j] = inv[i * k + j];
        out[i * k1 + k] = out[k * k1 + i] = side[i];
    }
    out[k * k1 + k] = corner;
    return out;
}

inline Mat mul(const Mat& a, const Mat& b, size_t k) {
    Mat out(k * k, 0.0);
    for (size_t i = 0; i < k; i++)
        for (size_t l = 0; l < k; l++) {
            const double x = a[i * k + l];
            if (x == 0.0) continue;
            for (size_t j = 0; j < k; j++) out[i * k + j] += x * b[l * k + j];
        }
    return out;
}

// Inverse of a symmetric positive definite matrix by its Cholesky factor L L^T (the 2SLS cross
// products, iv.rs dense::spd_inv); false when a pivot is not positive.
inline bool spd_inv(const Mat& a, size_t k, Mat& out) {
    Mat l(k * k, 0.0);
    for (size_t j = 0; j < k; j++) {
        double d = a[j * k + j];
        for (size_t p = 0; p < j; p++) d -= l[j * k + p] * l[j * k + p];
        if (!(d > 0.0)) return false;
        const double ljj = std::sqrt(d);
        l[j * k + j] = ljj;
        for (size_t i = j + 1; i < k; i++) {
            double s = a[i * k + j];
            for (size_t p = 0; p < j; p++) s -= l[i * k + p] * l[j * k + p];
            l[i * k + j] = s / ljj;
        }
    }
    // L^-1 by forward substitution, then (L^-1)^T L^-1
    Mat li(k * k, 0.0);
    for (size_t c = 0; c < k; c++) {
        li[c * k + c] = 1.0 / l[c * k + c];
        for (size_t i = c + 1; i < k; i++) {
            double s = 0.0;
            for (size_t p = c; p < i; p++) s -= l[i * k + p] * li[p * k + c];
            li[i * k + c] = s / l[i * k + i];
        }
    }
    out.assign(k * k, 0.0);
    for (size_t i = 0; i < k; i++)
        for (size_t j = 0; j <= i; j++) {
            double s = 0.0;
            for (size_t p = i; p < k; p++) s += li[p * k + i] * li[p * k + j];
            out[i * k + j] = out[j * k + i] = s;
        }
    return true;
}

// Row-major product of an m x p and a p x q matrix.
inline Mat mul_rect(const Mat& a, const Mat& b, size_t m, size_t p, size_t q) {
    Mat out(m * q, 0.0);
    for (size_t i = 0; i < m; i++)
        for (size_t l = 0; l < p; l++) {
            const double x = a[i * p + l];
            for (size_t j = 0; j < q; j++) out[i * q + j] += x * b[l * q + j];
        }
    return out;
}

// scale * bread * meat * bread, symmetrized.
inline Mat sandwich(const Mat& bread, const Mat& meat, size_t k, double scale) {
    Mat v = mul(mul(bread, meat, k), bread, k);
    symmetrize(v, k);
    for (double& x : v) x *= scale;
    return v;
}

// Eigen-decomposition of a symmetric matrix by cyclic Jacobi rotations: lam (k), vec columns.
inline void jacobi_eigen(const Mat& a, size_t k, std::vector<double>& lam, Mat& vec) {
    Mat m = a;
    vec.assign(k * k, 0.0);
    for (size_t i = 0; i < k; i++) vec[i * k + i] = 1.0;
    const double eps = 2.220446049250313e-16;
    for (int sweep_no = 0; sweep_no < 100; sweep_no++) {
        double off = 0.0, all = 0.0;
        for (size_t i = 0; i < k; i++)
            for (size_t j = 0; j < k; j++) {
                const double x = m[i * k + j] * m[i * k + j];
                all += x;
                if (i != j) off += x;
            }
        if (off == 0.0 || off <= eps * eps * all * 1e-4) break;
        for (size_t p = 0; p < k; p++)
            for (size_t q = p + 1; q < k; q++) {
                const double apq = m[p * k + q];
                if (apq == 0.0) continue;
                const double theta = (m[q * k + q] - m[p * k + p]) / (2.0 * apq);
                double t = theta == 0.0 ? 1.0
                                        : (theta > 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (size_t r = 0; r < k; r++) {
                    const double x = m[r * k + p], y = m[r * k + q];
                    m[r * k + p] = c * x - s * y;
                    m[r * k + q] = s * x + c * y;
                }
                for (size_t r = 0; r < k; r++) {
                    const double x = m[p * k + r], y = m[q * k + r];
                    m[p * k + r] = c * x - s * y;
                    m[q * k + r] = s * x + c * y;
                }
                for (size_t r = 0; r < k; r++) {
                    const double x = vec[r * k + p], y = vec[r * k + q];
                    vec[r * k + p] = c * x - s * y;
                    vec[r * k + q] = s * x + c * y;
                }
            }
    }
    lam.resize(k);
    for (size_t i = 0; i < k; i++) lam[i] = m[i * k + i];
}

// The matrix rebuilt from its positive eigenvalues; false (out untouched) when none is negative.
inline bool clip_negative(const Mat& v, size_t k, Mat& out) {
    std::vector<double> lam;
    Mat u;
    jacobi_eigen(v, k, lam, u);
    if (std::none_of(lam.begin(), lam.end(), [](double l) { return l < 0.0; })) return false;
    out.assign(k * k, 0.0);
    for (size_t e = 0; e < k; e++) {
        if (lam[e] <= 0.0) continue;
        for (size_t i = 0; i < k; i++) {
            const double ui = u[i * k + e] * lam[e];
            for (size_t j = 0; j <= i; j++) out[i * k + j] += ui * u[j * k + e];
        }
    }
    for (size_t i = 0; i < k; i++)
        for (size_t j = 0; j < i; j++) out[j * k + i] = out[i * k + j];
    return true;
}

// Multiway variance made positive semi-definite; with a reported constant the slope block is
// clipped on its own and written back over the clipped whole.
inline bool fix_psd(Mat& v, size_t k, bool constant) {
    symmetrize(v, k);
    const size_t kb = constant ? k - 1 : k;
    Mat slopes(kb * kb);
    for (size_t i = 0; i < kb; i++)
        for (size_t j = 0; j < kb; j++) slopes[i * kb + j] = v[i * k + j];
    Mat whole;
    if (!clip_negative(v, k, whole)) return false;
    v = whole;
    if (constant) {
        Mat sub;
        if (!clip_negative(slopes, kb, sub)) sub = slopes;
        for (size_t i = 0; i < kb; i++)
            for (size_t j = 0; j < kb; j++) v[i * k + j] = sub[i * kb + j];
    }
    return true;
}

// fixest's collinearity rule by Cholesky with exclusions (vcov.rs:124-200 chol_collin): column j
// is excluded when its pivot a_jj - sum over the kept earlier columns of r_ij^2 is below tol
// (or NaN); returns the inverse of the kept columns' block (kept x kept, in column order).
inline Mat chol_collin(const Mat& a, size_t k, double tol, std::vector<bool>& excluded) {
    Mat r(k * k, 0.0);
    excluded.assign(k, false);
    for (size_t j = 0; j < k; j++) {
        double rjj = a[j * k + j];
        for (size_t i = 0; i < j; i++)
            if (!excluded[i]) rjj -= r[i * k + j] * r[i * k + j];
        if (!(rjj >= tol)) {
            excluded[j] = true;
            continue;
        }
        const double d = std::sqrt(rjj);
        r[j * k + j] = d;
        for (size_t c = j + 1; c < k; c++) {
            double v = a[c * k + j];
            for (size_t i = 0; i < j; i++)
                if (!excluded[i]) v -= r[i * k + c] * r[i * k + j];
            r[j * k + c] = v / d;
        }
    }
    std::vector<size_t> kept;
    for (size_t j = 0; j < k; j++)
        if (!excluded[j]) kept.push_back(j);
    const size_t m = kept.size();
    Mat ri(m * m, 0.0);
    for (size_t c = 0; c < m; c++) {
        ri[c * m + c] = 1.0 / r[kept[c] * k + kept[c]];
        for (size_t row = c; row-- > 0;) {
            double s = 0.0;
            for (size_t l = row + 1; l <= c; l++) s += r[kept[row] * k + kept[l]] * ri[l * m + c];
            ri[row * m + c] = -s / r[kept[row] * k + kept[row]];
        }
    }
    Mat inv(m * m, 0.0);
    for (size_t i = 0; i < m; i++)
        for (size_t j = i; j < m; j++) {
            double s = 0.0;
            for (size_t l = j; l < m; l++) s += ri[i * m + l] * ri[j * m + l];
            inv[i * m + j] = inv[j * m + i] = s;
        }
    return inv;
}

}  // namespace la
}  // namespace fereg
