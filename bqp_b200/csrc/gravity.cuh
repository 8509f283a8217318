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

}  // namespace bqp
