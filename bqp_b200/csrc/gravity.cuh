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

// The whole field for NT trajectories per thread.
template <int NT>
BQP_HD void gravity_field_multi(const double* __restrict__ tab, int order, const double* px, const double* py,
                                const double* pz, double (*acc)[3]) {
    gravity_columns<NT>(tab, order, 0, order + 2, px, py, pz, acc);
}

}  // namespace bqp
