// Sigma-point (unscented) covariance propagation: generation of the sigma
// points of each object on the device, and the recombination of the
// propagated points into a mean and covariance.  The propagation in between
// is the ordinary batch propagation of n * S rows.
//
// Two sigma sets:
//   Julier 7-point simplex at W0 = 0 (dust_ukf_rs/src/lib.rs:22-37, 69-78,
//     247-275): x_i = mean + L xi_i, L = chol(P), weights 1/7 in both moments,
//     offsets xi from Julier's n + 2 recursion with the centre point dropped.
//   Van der Merwe scaled 13-point set (Wan & van der Merwe 2000, "The
//     unscented Kalman filter for nonlinear estimation"): lambda =
//     alpha^2 (n + kappa) - n, L = chol((n + lambda) P), x_0 = mean,
//     x_{1+i} = mean + L e_i, x_{7+i} = mean - L e_i; Wm_0 = lambda / (n +
//     lambda), Wc_0 = Wm_0 + 1 - alpha^2 + beta, W_i = 1 / (2 (n + lambda)).
// A covariance whose Cholesky factorisation fails is repaired as the
// reference does (lib.rs:202-240): eigenvalues below 1e-12 are raised to
// 1e-12 and the matrix rebuilt; if none was below, the object fails.
// Recombination (lib.rs:277-312): mean = sum Wm_i x_i, covariance = sum Wc_i
// (x_i - mean)(x_i - mean)^T, then symmetrised; the scaled set evaluates the
// same sums on deviations from its centre point.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "kernels.cuh"
#include "launch.h"

namespace bqp {

namespace {

constexpr int D = 6;

// Lower Cholesky factor of a symmetric 6x6 (row-major); false when a pivot
// is not positive and finite (nalgebra's Cholesky::new declines the same).
__device__ bool chol6(const double* a, double* l) {
    for (int i = 0; i < D * D; ++i) l[i] = 0.0;
    for (int j = 0; j < D; ++j) {
        double s = a[j * D + j];
        for (int k = 0; k < j; ++k) s -= l[j * D + k] * l[j * D + k];
        if (!(s > 0.0) || !isfinite(s)) return false;
        const double d = sqrt(s);
        l[j * D + j] = d;
        for (int i = j + 1; i < D; ++i) {
            double t = a[i * D + j];
            for (int k = 0; k < j; ++k) t -= l[i * D + k] * l[j * D + k];
            l[i * D + j] = t / d;
        }
    }
    return true;
}

// Cyclic Jacobi eigen-decomposition of a symmetric 6x6: a -> diagonal
// (eigenvalues), v = eigenvectors (columns).  At most 50 sweeps.
__device__ void jacobi6(double* a, double* v) {
    for (int i = 0; i < D * D; ++i) v[i] = (i % (D + 1)) == 0 ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < D; ++p)
            for (int q = p + 1; q < D; ++q) off += a[p * D + q] * a[p * D + q];
        if (!(off > 1e-300)) break;
        for (int p = 0; p < D; ++p) {
            for (int q = p + 1; q < D; ++q) {
                const double apq = a[p * D + q];
                if (apq == 0.0) continue;
                const double theta = (a[q * D + q] - a[p * D + p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < D; ++k) {  // columns p, q
                    const double akp = a[k * D + p], akq = a[k * D + q];
                    a[k * D + p] = c * akp - s * akq;
                    a[k * D + q] = s * akp + c * akq;
                }
                for (int k = 0; k < D; ++k) {  // rows p, q
                    const double apk = a[p * D + k], aqk = a[q * D + k];
                    a[p * D + k] = c * apk - s * aqk;
                    a[q * D + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < D; ++k) {
                    const double vkp = v[k * D + p], vkq = v[k * D + q];
                    v[k * D + p] = c * vkp - s * vkq;
                    v[k * D + q] = s * vkp + c * vkq;
                }
            }
        }
    }
}

// Repair toward positive definite (eigenvalues floored at 1e-12); false if
// no eigenvalue was below the floor.
__device__ bool repair6(const double* a, double* out) {
    double w[D * D], v[D * D];
    for (int i = 0; i < D * D; ++i) w[i] = a[i];
    jacobi6(w, v);
    bool floored = false;
    double ev[D];
    for (int i = 0; i < D; ++i) {
        ev[i] = w[i * D + i];
        if (ev[i] < 1e-12) {  // a NaN eigenvalue is not floored (the reference's comparison)
            ev[i] = 1e-12;
            floored = true;
        }
    }
    if (!floored) return false;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            double s = 0.0;
            for (int k = 0; k < D; ++k) s += v[i * D + k] * ev[k] * v[j * D + k];
            out[i * D + j] = s;
        }
    return true;
}

}  // namespace

// One thread per object: S sigma states per object, row-major [n][S][6];
// per-row epoch / end time / ballistics replicated.  status[n]: 0 or
// kInvalidInput (covariance not factorisable even after the repair).
__global__ void k_sigma_gen(int64_t n, int set, double scale, const double* __restrict__ offsets,
                            const double* __restrict__ mean, const double* __restrict__ cov,
                            const double* __restrict__ epoch, const double* __restrict__ tf,
                            const double* __restrict__ ballistic, double* __restrict__ rows,
                            double* __restrict__ row_epoch, double* __restrict__ row_tf,
                            double* __restrict__ row_bal, int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int S = set == 0 ? 7 : 13;
    double a[D * D], l[D * D], m[D];
    for (int k = 0; k < D; ++k) m[k] = mean[D * i + k];
    for (int k = 0; k < D * D; ++k) a[k] = cov[D * D * i + k] * scale;
    bool ok = chol6(a, l);
    if (!ok) {
        double r[D * D];
        ok = repair6(a, r) && chol6(r, l);
    }
    status[i] = ok ? kOk : kInvalidInput;
    for (int s = 0; s < S; ++s) {
        const int64_t row = i * S + s;
        double x[D];
        for (int k = 0; k < D; ++k) x[k] = m[k];
        if (set == 0) {  // x = mean + L xi_s
            for (int r = 0; r < D; ++r) {
                double t = 0.0;
                for (int c = 0; c <= r; ++c) t += l[r * D + c] * offsets[s * D + c];
                x[r] += t;
            }
        } else if (s > 0) {  // x = mean +/- column of L
            const int c = (s - 1) % D;
            const double sg = s <= D ? 1.0 : -1.0;
            for (int r = 0; r < D; ++r) x[r] += sg * l[r * D + c];
        }
        for (int k = 0; k < D; ++k) rows[D * row + k] = ok ? x[k] : NAN;
        row_epoch[row] = epoch[i];
        row_tf[row] = tf[i];
        if (row_bal) {
            row_bal[2 * row] = ballistic[2 * i];
            row_bal[2 * row + 1] = ballistic[2 * i + 1];
        }
    }
}

// One thread per object: weighted mean and covariance of its S propagated
// rows; any failed row fails the object with that row's status.
__global__ void k_sigma_recombine(int64_t n, int S, const double* __restrict__ wm, const double* __restrict__ wc,
                                  const double* __restrict__ rows, const int32_t* __restrict__ row_status,
                                  const int64_t* __restrict__ row_evals, double* __restrict__ mean_out,
                                  double* __restrict__ cov_out, int32_t* __restrict__ status,
                                  int64_t* __restrict__ evals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t st = status[i];
    int64_t ev = 0;
    for (int s = 0; s < S; ++s) {
        const int32_t rs = row_status[i * S + s];
        if (st == kOk && rs != kOk) st = rs;
        if (row_evals) ev += row_evals[i * S + s];
    }
    if (evals) evals[i] = ev;
    status[i] = st;
    if (st != kOk) {
        for (int k = 0; k < D; ++k) mean_out[D * i + k] = NAN;
        for (int k = 0; k < D * D; ++k) cov_out[D * D * i + k] = NAN;
        return;
    }
    double m[D] = {0, 0, 0, 0, 0, 0};
    double c[D * D];
    for (int k = 0; k < D * D; ++k) c[k] = 0.0;
    const double* x0 = rows + D * (i * S);
    if (S == 7) {
        // the reference's plain weighted sums (lib.rs:284-296)
        for (int s = 0; s < S; ++s)
            for (int k = 0; k < D; ++k) m[k] += wm[s] * rows[D * (i * S + s) + k];
        for (int s = 0; s < S; ++s) {
            double d[D];
            for (int k = 0; k < D; ++k) d[k] = rows[D * (i * S + s) + k] - m[k];
            for (int r = 0; r < D; ++r)
                for (int q = 0; q < D; ++q) c[r * D + q] += wc[s] * (d[r] * d[q]);
        }
    } else {
        // scaled set: sums of deviations from the centre point x_0 (the same
        // moments; with Wm_0 ~ -1/alpha^2 the plain sum would multiply the
        // rows' independent rounding by ~1e6, here only their differences
        // from x_0 enter)
        double dm[D] = {0, 0, 0, 0, 0, 0};
        for (int s = 1; s < S; ++s)
            for (int k = 0; k < D; ++k) dm[k] += wm[s] * (rows[D * (i * S + s) + k] - x0[k]);
        for (int k = 0; k < D; ++k) m[k] = x0[k] + dm[k];
        for (int s = 0; s < S; ++s) {
            double d[D];
            for (int k = 0; k < D; ++k) d[k] = (rows[D * (i * S + s) + k] - x0[k]) - dm[k];
            for (int r = 0; r < D; ++r)
                for (int q = 0; q < D; ++q) c[r * D + q] += wc[s] * (d[r] * d[q]);
        }
    }
    for (int r = 0; r < D; ++r)
        for (int q = 0; q < r; ++q) {
            const double v = 0.5 * (c[r * D + q] + c[q * D + r]);
            c[r * D + q] = v;
            c[q * D + r] = v;
        }
    for (int k = 0; k < D; ++k) mean_out[D * i + k] = m[k];
    for (int k = 0; k < D * D; ++k) cov_out[D * D * i + k] = c[k];
}

cudaError_t launch_sigma_gen(int64_t n, int set, double scale, const double* offsets, const double* mean,
                             const double* cov, const double* epoch, const double* tf, const double* ballistic,
                             double* rows, double* row_epoch, double* row_tf, double* row_bal, int32_t* status,
                             cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    k_sigma_gen<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(
        n, set, scale, offsets, mean, cov, epoch, tf, ballistic, rows, row_epoch, row_tf, row_bal, status);
    return cudaGetLastError();
}

cudaError_t launch_sigma_recombine(int64_t n, int S, const double* wm, const double* wc, const double* rows,
                                   const int32_t* row_status, const int64_t* row_evals, double* mean_out,
                                   double* cov_out, int32_t* status, int64_t* evals, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    k_sigma_recombine<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(
        n, S, wm, wc, rows, row_status, row_evals, mean_out, cov_out, status, evals);
    return cudaGetLastError();
}

}  // namespace bqp
