// Spherical-harmonic gravity by the normalised column recursion.
//
// The reference evaluates the field with the unnormalised Cunningham /
// Montenbruck-Gill V/W recursion and then a separate summation over (n, m)
// terms that reads V/W at orders m-1, m, m+1 of row n+1
// (satpy_core/src/gravity.rs:291-377 and 2075-2223).  Here the same
// acceleration is computed with 4-pi normalised V/W (no overflow to degree
// 128+, and usable in FP32), and the summation is folded into the recursion:
// every term that reads cell (l, j) of V/W is gathered, on the host, into six
// per-cell weights (Ax, Bx, Ay, By, Az, Bz) so that
//
//     a_x += Ax V(l,j) + Bx W(l,j),   a_y += Ay V + By W,   a_z += Az V + Bz W
//
// as soon as V(l,j), W(l,j) are produced.  A trajectory then streams the
// field column by column (j = 0..N+1, rows l = j..N+1) keeping only two rows
// of V/W in registers.  Per cell the thread reads 8 doubles (recursion
// coefficients a, b plus the six weights) -- the same address for every lane
// of the warp, i.e. a shared-memory broadcast -- and issues 12 FP64 ops.
//
// Table layout (built by the host, bqp_api.cu: build_gravity_table):
//   cell = 8 doubles {a, b, Ax, Bx, Ay, By, Az, Bz}, columns j ascending,
//   rows l ascending inside a column; (N+2)(N+3)/2 cells.
//   diagonal cell (j, j):     a = sqrt((2j+1)/(2j)) (j >= 2), sqrt(3) (j = 1)
//   sub-diagonal (j+1, j):    a = sqrt(2j+3)
//   interior (l >= j+2):      a = sqrt((2l-1)(2l+1)/((l-j)(l+j)))
//                             b = sqrt((2l+1)(l+j-1)(l-j-1)/((2l-3)(l+j)(l-j)))
// The weights already carry GM/R^2, so the result is in km/s^2.
#pragma once
#include "physics.cuh"

namespace bqp {

constexpr int kCellDoubles = 8;

BQP_HD int gravity_cells(int order) { return (order + 2) * (order + 3) / 2; }

// Acceleration (km/s^2, Earth-fixed) of the field encoded in `tab` at an
// Earth-fixed position (km).  `tab` may point to shared or global memory.
BQP_HD void gravity_field(const double* __restrict__ tab, int order, double px, double py,
                          double pz, double* acc) {
    const double r2 = fma(px, px, fma(py, py, pz * pz));
    const double c2 = kReGravity / r2;  // R/r^2
    const double xc = px * c2, yc = py * c2, zc = pz * c2;
    const double c2re = c2 * kReGravity;  // (R/r)^2
    double vd = sqrt(c2re);              // V(0,0) = R/r
    double wd = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    const int last = order + 1;
    const double* cell = tab;
    for (int j = 0; j <= last; ++j) {
        // diagonal (j, j)
        {
            const double a = cell[0];
            if (j > 0) {
                const double nv = a * fma(xc, vd, -yc * wd);
                const double nw = a * fma(xc, wd, yc * vd);
                vd = nv;
                wd = nw;
            }
            ax = fma(cell[2], vd, fma(cell[3], wd, ax));
            ay = fma(cell[4], vd, fma(cell[5], wd, ay));
            az = fma(cell[6], vd, fma(cell[7], wd, az));
            cell += kCellDoubles;
        }
        if (j == last) break;
        // sub-diagonal (j+1, j)
        double v0 = vd, w0 = wd;
        double v1, w1;
        {
            const double a = cell[0] * zc;
            v1 = a * vd;
            w1 = a * wd;
            ax = fma(cell[2], v1, fma(cell[3], w1, ax));
            ay = fma(cell[4], v1, fma(cell[5], w1, ay));
            az = fma(cell[6], v1, fma(cell[7], w1, az));
            cell += kCellDoubles;
        }
        // interior rows
        for (int l = j + 2; l <= last; ++l) {
            const double ta = cell[0] * zc;
            const double tb = cell[1] * c2re;
            const double v2 = fma(ta, v1, -tb * v0);
            const double w2 = fma(ta, w1, -tb * w0);
            ax = fma(cell[2], v2, fma(cell[3], w2, ax));
            ay = fma(cell[4], v2, fma(cell[5], w2, ay));
            az = fma(cell[6], v2, fma(cell[7], w2, az));
            v0 = v1; v1 = v2;
            w0 = w1; w1 = w2;
            cell += kCellDoubles;
        }
    }
    acc[0] = ax;
    acc[1] = ay;
    acc[2] = az;
}

// Index of the first cell of column j (columns hold rows j..order+1).
BQP_HD int gravity_col_offset(int order, int j) {
    const int rows0 = order + 2;  // cells in column 0
    return j * rows0 - j * (j - 1) / 2;
}

// First column of part p when the columns are cut into `parts` runs of about
// equal cell count (p = parts gives order + 2, one past the last column).
BQP_HD int gravity_part_column(int order, int p, int parts) {
    const int ncol = order + 2;
    if (p <= 0) return 0;
    if (p >= parts) return ncol;
    const long long target = (long long)gravity_cells(order) * p / parts;
    int j = 0;
    long long cells = 0;
    while (j < ncol && cells + (ncol - j) <= target) cells += ncol - j++;
    return j;
}

// Partial field of columns [j0, j1) for NT trajectories per thread.  Every
// table read (four 16-byte loads per cell, the same address in every lane)
// feeds NT independent recursions: the loads move 64 bytes per cell into
// every lane's registers, so sharing them over NT trajectories is what keeps
// the FP64 pipe, not the shared-memory data path, the limit.  The diagonal
// V/W recursion is first carried (without accumulation) through columns
// 1..j0-1, so a part that starts at j0 > 0 needs nothing from another part.
// Interior cells are read two at a time and the next pair is loaded before
// the current one is used.
template <int NT>
BQP_HD void gravity_columns(const double* __restrict__ tab, int order, int j0, int j1, const double* px,
                            const double* py, const double* pz, double (*acc)[3]) {
    double xc[NT], yc[NT], zc[NT], c2re[NT], vd[NT], wd[NT], ax[NT], ay[NT], az[NT];
#pragma unroll
    for (int q = 0; q < NT; ++q) {
        const double r2 = fma(px[q], px[q], fma(py[q], py[q], pz[q] * pz[q]));
        const double c2 = kReGravity / r2;
        xc[q] = px[q] * c2;
        yc[q] = py[q] * c2;
        zc[q] = pz[q] * c2;
        c2re[q] = c2 * kReGravity;
        vd[q] = sqrt(c2re[q]);
        wd[q] = 0.0;
        ax[q] = ay[q] = az[q] = 0.0;
    }
    const int last = order + 1;
    const double2* tab2 = reinterpret_cast<const double2*>(tab);
    for (int j = 1; j < j0; ++j) {
        const double a = tab2[(size_t)gravity_col_offset(order, j) * 4].x;
#pragma unroll
        for (int q = 0; q < NT; ++q) {
            const double nv = a * fma(xc[q], vd[q], -yc[q] * wd[q]);
            const double nw = a * fma(xc[q], wd[q], yc[q] * vd[q]);
            vd[q] = nv;
            wd[q] = nw;
        }
    }
    const double2* cell = tab2 + (size_t)gravity_col_offset(order, j0) * 4;
    for (int j = j0; j < j1; ++j) {
        {
            const double2 ab = cell[0], wx = cell[1], wy = cell[2], wz = cell[3];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                if (j > 0) {
                    const double nv = ab.x * fma(xc[q], vd[q], -yc[q] * wd[q]);
                    const double nw = ab.x * fma(xc[q], wd[q], yc[q] * vd[q]);
                    vd[q] = nv;
                    wd[q] = nw;
                }
                ax[q] = fma(wx.x, vd[q], fma(wx.y, wd[q], ax[q]));
                ay[q] = fma(wy.x, vd[q], fma(wy.y, wd[q], ay[q]));
                az[q] = fma(wz.x, vd[q], fma(wz.y, wd[q], az[q]));
            }
            cell += 4;
        }
        if (j == last) break;
        double v0[NT], w0[NT], v1[NT], w1[NT];
        {
            const double2 ab = cell[0], wx = cell[1], wy = cell[2], wz = cell[3];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const double a = ab.x * zc[q];
                v0[q] = vd[q];
                w0[q] = wd[q];
                v1[q] = a * vd[q];
                w1[q] = a * wd[q];
                ax[q] = fma(wx.x, v1[q], fma(wx.y, w1[q], ax[q]));
                ay[q] = fma(wy.x, v1[q], fma(wy.y, w1[q], ay[q]));
                az[q] = fma(wz.x, v1[q], fma(wz.y, w1[q], az[q]));
            }
            cell += 4;
        }
        // interior rows j+2..last, two per iteration (the row registers
        // rotate without moves); the next pair is in flight meanwhile
        const int pairs = (last - j - 1) >> 1;
        double2 nx[8];
        if (pairs > 0) {
#pragma unroll
            for (int i = 0; i < 8; ++i) nx[i] = cell[i];
        }
#pragma unroll 2
        for (int p = 0; p < pairs; ++p) {
            double2 cb[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) cb[i] = nx[i];
            if (p + 1 < pairs) {
#pragma unroll
                for (int i = 0; i < 8; ++i) nx[i] = cell[8 + i];
            }
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const double ta = cb[0].x * zc[q], tb = cb[0].y * c2re[q];
                v0[q] = fma(ta, v1[q], -tb * v0[q]);
                w0[q] = fma(ta, w1[q], -tb * w0[q]);
                ax[q] = fma(cb[1].x, v0[q], fma(cb[1].y, w0[q], ax[q]));
                ay[q] = fma(cb[2].x, v0[q], fma(cb[2].y, w0[q], ay[q]));
                az[q] = fma(cb[3].x, v0[q], fma(cb[3].y, w0[q], az[q]));
                const double ta2 = cb[4].x * zc[q], tb2 = cb[4].y * c2re[q];
                v1[q] = fma(ta2, v0[q], -tb2 * v1[q]);
                w1[q] = fma(ta2, w0[q], -tb2 * w1[q]);
                ax[q] = fma(cb[5].x, v1[q], fma(cb[5].y, w1[q], ax[q]));
                ay[q] = fma(cb[6].x, v1[q], fma(cb[6].y, w1[q], ay[q]));
                az[q] = fma(cb[7].x, v1[q], fma(cb[7].y, w1[q], az[q]));
            }
            cell += 8;
        }
        if ((last - j - 1) & 1) {
            const double2 ab = cell[0], wx = cell[1], wy = cell[2], wz = cell[3];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const double ta = ab.x * zc[q], tb = ab.y * c2re[q];
                const double v2 = fma(ta, v1[q], -tb * v0[q]);
                const double w2 = fma(ta, w1[q], -tb * w0[q]);
                ax[q] = fma(wx.x, v2, fma(wx.y, w2, ax[q]));
                ay[q] = fma(wy.x, v2, fma(wy.y, w2, ay[q]));
                az[q] = fma(wz.x, v2, fma(wz.y, w2, az[q]));
            }
            cell += 4;
        }
    }
#pragma unroll
    for (int q = 0; q < NT; ++q) {
        acc[q][0] = ax[q];
        acc[q][1] = ay[q];
        acc[q][2] = az[q];
    }
}

// ---------------------------------------------------------------------------
// Split-precision form.  Cell (l, j) carries only degree n = l - 1, so rows
// l <= ls hold degrees n <= ls - 1 (the central-field corrections J2...,
// kept in FP64) and every other cell the higher degrees, evaluated in FP32:
//   lo: FP64 cells of columns 0..ls, rows j..ls (column-major)
//   hi: FP32 cells {a, b, Ax, Bx | Ay, By, Az, Bz} of columns 0..ls, rows
//       ls+1..order+1, then columns ls+1..order+1, rows j..order+1
// The V/W values of the last FP64 rows seed the FP32 rows below them; the
// two parts are accumulated separately and added in FP64.  Needs
// 1 <= ls <= order.
BQP_HD int split_lo_offset(int ls, int j) { return j * (ls + 1) - j * (j - 1) / 2; }
BQP_HD int split_lo_cells(int ls) { return (ls + 1) * (ls + 2) / 2; }
BQP_HD int split_hi_offset(int order, int ls, int j) {
    const int h = order + 1 - ls;  // FP32 rows under an FP64 column
    if (j <= ls + 1) return j * h;
    const int k = j - (ls + 1);
    return (ls + 1) * h + k * h - k * (k - 1) / 2;
}
BQP_HD int split_hi_cells(int order, int ls) { return split_hi_offset(order, ls, order + 2); }

template <int NT>
BQP_HD void gravity_columns_split(const double* __restrict__ lo, const float* __restrict__ hi, int order, int ls,
                                  int j0, int j1, const double* px, const double* py, const double* pz,
                                  double (*acc)[3]) {
    double xc[NT], yc[NT], zc[NT], c2re[NT], vd[NT], wd[NT], ax[NT], ay[NT], az[NT];
    float xf[NT], yf[NT], zf[NT], cf[NT], vdf[NT], wdf[NT], fx[NT], fy[NT], fz[NT];
#pragma unroll
    for (int q = 0; q < NT; ++q) {
        const double r2 = fma(px[q], px[q], fma(py[q], py[q], pz[q] * pz[q]));
        const double c2 = kReGravity / r2;
        xc[q] = px[q] * c2;
        yc[q] = py[q] * c2;
        zc[q] = pz[q] * c2;
        c2re[q] = c2 * kReGravity;
        vd[q] = sqrt(c2re[q]);
        wd[q] = 0.0;
        ax[q] = ay[q] = az[q] = 0.0;
        xf[q] = (float)xc[q];
        yf[q] = (float)yc[q];
        zf[q] = (float)zc[q];
        cf[q] = (float)c2re[q];
        vdf[q] = wdf[q] = 0.0f;
        fx[q] = fy[q] = fz[q] = 0.0f;
    }
    const int last = order + 1;
    const double2* lo2 = reinterpret_cast<const double2*>(lo);
    const float4* hi4 = reinterpret_cast<const float4*>(hi);
    // diagonal V(j,j), W(j,j) from column j-1's
    auto advance_diag = [&](int j) {
        if (j <= ls) {
            const double a = lo2[(size_t)split_lo_offset(ls, j) * 4].x;
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const double nv = a * fma(xc[q], vd[q], -yc[q] * wd[q]);
                const double nw = a * fma(xc[q], wd[q], yc[q] * vd[q]);
                vd[q] = nv;
                wd[q] = nw;
            }
        } else {
            const float a = hi4[(size_t)split_hi_offset(order, ls, j) * 2].x;
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                if (j == ls + 1) {
                    vdf[q] = (float)vd[q];
                    wdf[q] = (float)wd[q];
                }
                const float nv = a * fmaf(xf[q], vdf[q], -yf[q] * wdf[q]);
                const float nw = a * fmaf(xf[q], wdf[q], yf[q] * vdf[q]);
                vdf[q] = nv;
                wdf[q] = nw;
            }
        }
    };
    // FP32 interior rows: n cells from hc, recursion seeded by rows l-2, l-1
    auto fp32_interior = [&](const float4* hc, int n, float* v0, float* w0, float* v1, float* w1) {
        const int pairs = n >> 1;
        float4 nx[4];
        if (pairs > 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i) nx[i] = hc[i];
        }
#pragma unroll 2
        for (int p = 0; p < pairs; ++p) {
            float4 cb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) cb[i] = nx[i];
            if (p + 1 < pairs) {
#pragma unroll
                for (int i = 0; i < 4; ++i) nx[i] = hc[4 + i];
            }
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const float ta = cb[0].x * zf[q], tb = cb[0].y * cf[q];
                v0[q] = fmaf(ta, v1[q], -tb * v0[q]);
                w0[q] = fmaf(ta, w1[q], -tb * w0[q]);
                fx[q] = fmaf(cb[0].z, v0[q], fmaf(cb[0].w, w0[q], fx[q]));
                fy[q] = fmaf(cb[1].x, v0[q], fmaf(cb[1].y, w0[q], fy[q]));
                fz[q] = fmaf(cb[1].z, v0[q], fmaf(cb[1].w, w0[q], fz[q]));
                const float ta2 = cb[2].x * zf[q], tb2 = cb[2].y * cf[q];
                v1[q] = fmaf(ta2, v0[q], -tb2 * v1[q]);
                w1[q] = fmaf(ta2, w0[q], -tb2 * w1[q]);
                fx[q] = fmaf(cb[2].z, v1[q], fmaf(cb[2].w, w1[q], fx[q]));
                fy[q] = fmaf(cb[3].x, v1[q], fmaf(cb[3].y, w1[q], fy[q]));
                fz[q] = fmaf(cb[3].z, v1[q], fmaf(cb[3].w, w1[q], fz[q]));
            }
            hc += 4;
        }
        if (n & 1) {
            const float4 c0 = hc[0], c1 = hc[1];
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                const float ta = c0.x * zf[q], tb = c0.y * cf[q];
                const float v2 = fmaf(ta, v1[q], -tb * v0[q]);
                const float w2 = fmaf(ta, w1[q], -tb * w0[q]);
                fx[q] = fmaf(c0.z, v2, fmaf(c0.w, w2, fx[q]));
                fy[q] = fmaf(c1.x, v2, fmaf(c1.y, w2, fy[q]));
                fz[q] = fmaf(c1.z, v2, fmaf(c1.w, w2, fz[q]));
            }
        }
    };
    for (int j = 1; j < j0; ++j) advance_diag(j);
    for (int j = j0; j < j1; ++j) {
        if (j > 0) advance_diag(j);
        float v0f[NT], w0f[NT], v1f[NT], w1f[NT];
        if (j <= ls) {
            // FP64 rows j..ls
            const double2* cell = lo2 + (size_t)split_lo_offset(ls, j) * 4;
            double v0[NT], w0[NT], v1[NT], w1[NT];
            {
                const double2 wxx = cell[1], wyy = cell[2], wzz = cell[3];
#pragma unroll
                for (int q = 0; q < NT; ++q) {
                    ax[q] = fma(wxx.x, vd[q], fma(wxx.y, wd[q], ax[q]));
                    ay[q] = fma(wyy.x, vd[q], fma(wyy.y, wd[q], ay[q]));
                    az[q] = fma(wzz.x, vd[q], fma(wzz.y, wd[q], az[q]));
                    v0[q] = 0.0;
                    w0[q] = 0.0;
                    v1[q] = vd[q];
                    w1[q] = wd[q];
                }
                cell += 4;
            }
            for (int l = j + 1; l <= ls; ++l) {
                const double2 ab = cell[0], wxx = cell[1], wyy = cell[2], wzz = cell[3];
#pragma unroll
                for (int q = 0; q < NT; ++q) {
                    const double ta = ab.x * zc[q];
                    const double v2 = l == j + 1 ? ta * v1[q] : fma(ta, v1[q], -(ab.y * c2re[q]) * v0[q]);
                    const double w2 = l == j + 1 ? ta * w1[q] : fma(ta, w1[q], -(ab.y * c2re[q]) * w0[q]);
                    ax[q] = fma(wxx.x, v2, fma(wxx.y, w2, ax[q]));
                    ay[q] = fma(wyy.x, v2, fma(wyy.y, w2, ay[q]));
                    az[q] = fma(wzz.x, v2, fma(wzz.y, w2, az[q]));
                    v0[q] = v1[q];
                    w0[q] = w1[q];
                    v1[q] = v2;
                    w1[q] = w2;
                }
                cell += 4;
            }
#pragma unroll
            for (int q = 0; q < NT; ++q) {
                v0f[q] = (float)v0[q];
                w0f[q] = (float)w0[q];
                v1f[q] = (float)v1[q];
                w1f[q] = (float)w1[q];
            }
            // FP32 rows ls+1..last
            const float4* hc = hi4 + (size_t)split_hi_offset(order, ls, j) * 2;
            int n = last - ls;
            if (j == ls) {  // row ls+1 is this column's sub-diagonal
                const float4 c0 = hc[0], c1 = hc[1];
#pragma unroll
                for (int q = 0; q < NT; ++q) {
                    const float a = c0.x * zf[q];
                    v0f[q] = v1f[q];
                    w0f[q] = w1f[q];
                    v1f[q] = a * v0f[q];
                    w1f[q] = a * w0f[q];
                    fx[q] = fmaf(c0.z, v1f[q], fmaf(c0.w, w1f[q], fx[q]));
                    fy[q] = fmaf(c1.x, v1f[q], fmaf(c1.y, w1f[q], fy[q]));
                    fz[q] = fmaf(c1.z, v1f[q], fmaf(c1.w, w1f[q], fz[q]));
                }
                hc += 2;
                --n;
            }
            fp32_interior(hc, n, v0f, w0f, v1f, w1f);
        } else {
            // all FP32: diagonal, sub-diagonal, interior
            const float4* hc = hi4 + (size_t)split_hi_offset(order, ls, j) * 2;
            {
                const float4 c0 = hc[0], c1 = hc[1];
#pragma unroll
                for (int q = 0; q < NT; ++q) {
                    fx[q] = fmaf(c0.z, vdf[q], fmaf(c0.w, wdf[q], fx[q]));
                    fy[q] = fmaf(c1.x, vdf[q], fmaf(c1.y, wdf[q], fy[q]));
                    fz[q] = fmaf(c1.z, vdf[q], fmaf(c1.w, wdf[q], fz[q]));
                }
                hc += 2;
            }
            if (j == last) continue;
            {
                const float4 c0 = hc[0], c1 = hc[1];
#pragma unroll
                for (int q = 0; q < NT; ++q) {
                    const float a = c0.x * zf[q];
                    v0f[q] = vdf[q];
                    w0f[q] = wdf[q];
                    v1f[q] = a * vdf[q];
                    w1f[q] = a * wdf[q];
                    fx[q] = fmaf(c0.z, v1f[q], fmaf(c0.w, w1f[q], fx[q]));
                    fy[q] = fmaf(c1.x, v1f[q], fmaf(c1.y, w1f[q], fy[q]));
                    fz[q] = fmaf(c1.z, v1f[q], fmaf(c1.w, w1f[q], fz[q]));
                }
                hc += 2;
            }
            fp32_interior(hc, last - j - 1, v0f, w0f, v1f, w1f);
        }
    }
#pragma unroll
    for (int q = 0; q < NT; ++q) {
        acc[q][0] = ax[q] + (double)fx[q];
        acc[q][1] = ay[q] + (double)fy[q];
        acc[q][2] = az[q] + (double)fz[q];
    }
}

// The whole field for NT trajectories per thread.
template <int NT>
BQP_HD void gravity_field_multi(const double* __restrict__ tab, int order, const double* px, const double* py,
                                const double* pz, double (*acc)[3]) {
    gravity_columns<NT>(tab, order, 0, order + 2, px, py, pz, acc);
}

}  // namespace bqp
