// Device side of the batched propagator: the Encke force call and the
// one-trajectory-per-thread adaptive RK driver (DOPRI5(4), DOP853 and the
// DOPRI5 compatibility loop), as a persistent kernel that pulls trajectories
// from a device work queue.
#pragma once
#include <cstdint>

#include "gravity.cuh"
#include "jb2008.cuh"
#include "physics.cuh"
#include "frame_time.h"

namespace bqp {

// Per-trajectory status words (mirroring the reference's IntegrationStatus,
// GravityError and FinalPropagationFailure; values are part of the C ABI).
enum Status : int32_t {
    kOk = 0,
    kMaxSteps = 1,
    kStepUnderflow = 2,
    kInvalidInput = 3,
    kNonFinite = 4,
    kMaxRejects = 5,
    kGravityRadius = 6,
    kRebaseFailed = 7,
    kRestartBudget = 8,
    kGround = 9,
    kWatchdog = 10,
    // binary-eclipse coordinator failures (EclipseError, eclipse.rs)
    kEclEnvelope = 11,
    kEclChatter = 12,
    kEclBracket = 13,
    kEclNonProgress = 14,
    kEclGeometry = 15,
    kEclSplitLimit = 16,
    // the Earth-fixed frame has no segment at an evaluation's instant (the
    // reference's GravityError::InvalidTime from its frame authority)
    kFrameTime = 17,
};

enum Method : int32_t { kDopri5 = 0, kDop853 = 1, kDopri5Compat = 2, kVern7 = 3, kVern9 = 4 };

// Force switches and constants (ForceConfig, types.rs:332-411).
struct ForceParams {
    int32_t order;
    int32_t gravity_on;
    int32_t drag, sun, moon;
    int32_t ground_check;  // terminal ground event (final-state path)
    int32_t atm_model;     // JB2008 profile: 4 exact; 5, 6, 7 the coarse quadrature profiles
    int32_t drag_fp32;     // split precision: the coarse profile's density in FP32
    int32_t srp;           // solar radiation pressure through the eclipse coordinator
    double cr, p_sun;      // SRP reflectivity coefficient, pressure at 1 AU (N/m^2)
    double sun_rate;       // bound of the Sun direction's angular rate, rad/day
    double earth_radius;
    double omega;
    double mu_sun, mu_moon;
    jb::Drivers drivers;
    jb::DriverTable dtab;  // space-weather tables (n_solar 0: the fixed drivers above)
    EphemTable eph_sun, eph_moon;  // precomputed catalogues (n 0: the analytic series)
    const jb::JbFit* fit;  // device copy of the fixed-node sweep fits, or null
    const jb::JbFit2* fit2;  // altitude-dependent sweep fits (stage-synchronous drag), or null
    ft::FrameTab frame;      // IAU 2006/2000A segments (frame.mode 1) or the GMST rotation (0)
};

// The Earth-fixed rotation of an instant under `frame.mode` 1: the segment
// holding continuous-TAI `tai`; false (a frame-time failure) when the table
// has none.
__device__ __forceinline__ bool frame_rot(const ft::FrameTab& F, double tai, ft::FrameRot& R) {
    const int32_t slot = ft::segment_slot(F, tai);
    if (slot < 0) return false;
    ft::rotation_at(F.seg[slot], tai, R);
    return true;
}

// Solver controls (IntegratorConfig, solver.rs:35-60 and integrator.rs:404-558).
struct CtrlParams {
    int32_t scaled;  // 0: absolute eps, max-norm; 1: rtol/atol, WRMS
    int32_t max_rejects;
    double eps, rtol, atol;
    double h_min, h_max;
    int64_t max_steps;        // per segment
    int64_t max_attempts;     // per trajectory, device watchdog
    int64_t max_kernel_ns;    // wall-clock watchdog of one launch (0: none)
};

// Nanosecond global timer (PTX %globaltimer).
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Copy the field table into dynamic shared memory with 16-byte vector loads.
__device__ __forceinline__ const double* stage_table(const double* __restrict__ g, int ncells,
                                                     bool to_smem) {
    extern __shared__ __align__(16) double smem_tab[];
    if (!to_smem) return g;
    const int nvec = ncells * (kCellDoubles / 2);
    const double2* src = reinterpret_cast<const double2*>(g);
    double2* dst = reinterpret_cast<double2*>(smem_tab);
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    return smem_tab;
}

// One Encke force evaluation: derivative of the deviation `d` from the
// baseline orbit (rhs.rs:3885-4118).  Gravity uses the field table without
// its C00 term, which equals the reference's full field followed by the
// analytic removal of mu r/r^3.
struct Encke {
    const double* tab;
    const ForceParams* fp;
    Baseline base;
    double seg_t0;
    double jd0;
    double tai0;  // continuous TAI seconds of t = 0 (IAU frame)
    double am, cd;
    int side;  // SRP eclipse side of the row's leg (1 shadow, 0 lit), -1 without SRP
    int bad;   // latched error: 1 invalid-radius gravity, 3 no frame segment

    __device__ __noinline__ void eval(double t, const double* d, double* out) {
        double rs[6];
        baseline_state(base, t - seg_t0, rs);
        double sp[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) sp[i] = rs[i] + d[i];
        const double r2 = fma(sp[0], sp[0], fma(sp[1], sp[1], sp[2] * sp[2]));
        const double r = sqrt(r2);
        double acc[3] = {0.0, 0.0, 0.0};
        const double jd = utc_jd_at(jd0, t);
        // Earth-fixed position: the GMST z-rotation, or the IAU 2006/2000A
        // rotation with its angular velocity (rhs.rs:3924-3935)
        const bool iau = fp->frame.mode == 1;
        double s = 0.0, c = 1.0;
        ft::FrameRot F;
        double pi[3];
        if (iau) {
            if (fp->gravity_on || fp->drag) {
                if (!frame_rot(fp->frame, tai0 + t, F)) {
                    bad = 3;
                    for (int i = 0; i < 6; ++i) out[i] = NAN;
                    return;
                }
                ft::to_itrs(F.r, sp, pi);
            }
        } else {
            if (fp->gravity_on || fp->drag) sincos(gmst_rad(jd), &s, &c);
            pi[0] = fma(c, sp[0], s * sp[1]);
            pi[1] = fma(-s, sp[0], c * sp[1]);
            pi[2] = sp[2];
        }
        if (fp->gravity_on) {
            if (!(isfinite(r2) && r2 > 0.0)) bad = 1;
            double ai[3];
            gravity_field(tab, fp->order, pi[0], pi[1], pi[2], ai);
            if (iau) {
                ft::to_gcrs(F.r, ai, acc);
            } else {
                acc[0] = fma(c, ai[0], -s * ai[1]);
                acc[1] = fma(s, ai[0], c * ai[1]);
                acc[2] = ai[2];
            }
        }
        double sun[3];
        bool have_sun = false;
        if (fp->drag && cd != 0.0 && am != 0.0) {
            sun_at(fp->eph_sun, jd, sun);
            have_sun = true;
            double si[3];
            if (iau) {
                ft::to_itrs(F.r, sun, si);
            } else {
                si[0] = fma(c, sun[0], s * sun[1]);
                si[1] = fma(-s, sun[0], c * sun[1]);
                si[2] = sun[2];
            }
            double rho = density_at(pi, si, jd);
            if (isnan(rho)) {
                acc[0] = acc[1] = acc[2] = NAN;
            } else if (rho > 0.0) {
                // co-rotating atmosphere, m/s inside, km/s^2 out (rhs.rs:1119-1163)
                double vr0, vr1, vr2;
                if (iau) {
                    const double* w = F.w;
                    vr0 = (sp[3] - (w[1] * sp[2] - w[2] * sp[1])) * 1000.0;
                    vr1 = (sp[4] - (w[2] * sp[0] - w[0] * sp[2])) * 1000.0;
                    vr2 = (sp[5] - (w[0] * sp[1] - w[1] * sp[0])) * 1000.0;
                } else {
                    const double w = fp->omega;
                    vr0 = (sp[3] + w * sp[1]) * 1000.0;
                    vr1 = (sp[4] - w * sp[0]) * 1000.0;
                    vr2 = sp[5] * 1000.0;
                }
                const double v2 = fma(vr0, vr0, fma(vr1, vr1, vr2 * vr2));
                if (v2 != 0.0) {
                    const double k = -0.5 * cd * am * rho * sqrt(v2) * 1e-3;
                    acc[0] += k * vr0;
                    acc[1] += k * vr1;
                    acc[2] += k * vr2;
                }
            }
        }
        if (side >= 0) {
            // after drag, before the third bodies (rhs.rs:4033-4063)
            if (!have_sun) sun_at(fp->eph_sun, jd, sun);
            have_sun = true;
            srp_accel(sp, sun, fp->p_sun, fp->cr, am, side, acc);
        }
        if (fp->sun) {
            if (!have_sun) sun_at(fp->eph_sun, jd, sun);
            third_body(sp, sun, fp->mu_sun, acc);
        }
        if (fp->moon) {
            double moon[3];
            moon_at(fp->eph_moon, jd, moon);
            third_body(sp, moon, fp->mu_moon, acc);
        }
        battin(rs, d, r2, r, acc);
        out[0] = d[3];
        out[1] = d[4];
        out[2] = d[5];
        out[3] = acc[0];
        out[4] = acc[1];
        out[5] = acc[2];
    }

    // JB2008 adapter (rhs.rs:3551-3776): Earth-fixed satellite and Sun,
    // geocentric latitude, WGS84 altitude, exospheric ceiling above 2500 km.
    __device__ __forceinline__ double density_at(const double* pi, const double* si, double jd) const {
        const double sun_r = sqrt(fma(si[0], si[0], fma(si[1], si[1], si[2] * si[2])));
        const double sat_r = sqrt(fma(pi[0], pi[0], fma(pi[1], pi[1], pi[2] * pi[2])));
        if ((sat_r - fp->earth_radius) * 1000.0 > 2500.0e3) return 1.0e-19;
        const double alt_m = geodetic_altitude_km(pi[0], pi[1], pi[2], fp->earth_radius) * 1000.0;
        const double dec = asin(fmin(1.0, fmax(-1.0, si[2] / sun_r)));
        const double ha = atan2(fma(pi[1], si[0], -(pi[0] * si[1])), fma(pi[0], si[0], pi[1] * si[1]));
        const double lat = asin(fmin(1.0, fmax(-1.0, pi[2] / sat_r)));
        jb::Drivers dr = fp->drivers;
        // rhs.rs:3560-3571: no drivers at this instant -> NaN density
        if (fp->dtab.n_solar > 0 && !jb::lookup_drivers(fp->dtab, jd, &dr)) return NAN;
        double rho = (fp->drag_fp32 && fp->atm_model != 4)
                         ? jb::density_coarse_r<float>(jd - 2400000.5, dec, ha, lat, alt_m, dr, fp->atm_model)
                         : jb::density_model(jd - 2400000.5, dec, ha, lat, alt_m, dr, fp->atm_model, fp->fit);
        if (!(rho > 0.0) || !isfinite(rho)) return NAN;
        if (alt_m > 2500.0e3) rho = fmin(rho, 1.0e-19);
        return rho;
    }
};

}  // namespace bqp
