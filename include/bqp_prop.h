/*
 * bqp_prop.h -- C ABI of the B200 batched orbit propagator (libbqp_b200.so).
 *
 * Drop-in boundary for the Lightyear propagator of tdude78/bqp
 * (dust_transfer).  Each entry point names the reference interface it
 * replaces (paths inside dust_transfer/).  Plain pointers and sizes only.
 *
 * Units and frames (reference dust_transfer/src/lib.rs:1-24): km, km/s, s,
 * Julian Date (UTC).  States are row-major [x, y, z, vx, vy, vz] in the
 * propagator's inertial frame; the gravity field is Earth-fixed, related to
 * the inertial frame by the GMST rotation about +z
 * (satpy_core/src/lib.rs:905-978).  Equinoctial elements are
 * [a, h, k, p, q, L] (satpy_core/src/lib.rs:1738-1870).
 *
 * Return codes: 0 on success, a negative BQP_E_* code on a call-level error
 * (bqp_last_error() has the message).  Per-trajectory outcomes are reported
 * in `status` arrays with the BQP_ST_* codes; failed rows are NaN-filled
 * (lightyear_odeint_rs/src/batch.rs:297).
 *
 * Entry points without `_device` take HOST buffers and copy to and from the
 * GPU inside the call.  `_device` variants take device pointers and enqueue
 * on the context's stream without synchronising.
 */
#ifndef BQP_PROP_H
#define BQP_PROP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BQP_API_VERSION 1

/* call-level return codes */
#define BQP_E_ARG (-1)         /* invalid argument */
#define BQP_E_CUDA (-2)        /* CUDA runtime error or no device */
#define BQP_E_COEFF (-3)       /* gravity coefficient text rejected */
#define BQP_E_UNSUPPORTED (-4) /* option outside this build */
#define BQP_E_NOMEM (-5)

/* per-trajectory status (IntegrationStatus, odesolve/solver.rs:64-95;
 * GravityError, satpy_core/src/gravity.rs:21-37; FinalPropagationFailure,
 * lightyear_odeint_rs/src/integrator.rs:2588-2612) */
#define BQP_ST_OK 0
#define BQP_ST_MAX_STEPS 1
#define BQP_ST_STEP_UNDERFLOW 2
#define BQP_ST_INVALID_INPUT 3
#define BQP_ST_NON_FINITE 4
#define BQP_ST_MAX_REJECTS 5
#define BQP_ST_GRAVITY_RADIUS 6
#define BQP_ST_REBASE_FAILED 7
#define BQP_ST_RESTART_BUDGET 8
#define BQP_ST_GROUND 9
#define BQP_ST_WATCHDOG 10
/* binary-eclipse SRP coordinator failures (EclipseError, lightyear_odeint_rs/src/eclipse.rs) */
#define BQP_ST_ECLIPSE_ENVELOPE 11     /* state outside radius 6000-50000 km, speed <= 20 km/s */
#define BQP_ST_ECLIPSE_CHATTER 12      /* side changed where a leg held it, or a root out of order */
#define BQP_ST_ECLIPSE_BRACKET 13      /* a replay or proof leg failed to confirm the crossing */
#define BQP_ST_ECLIPSE_NON_PROGRESS 14 /* a bracket or window that cannot shrink */
#define BQP_ST_ECLIPSE_GEOMETRY 15     /* non-finite geometry or a Sun outside the catalogue */
#define BQP_ST_ECLIPSE_SPLIT_LIMIT 16  /* more than 4096 roots, bisections or iterations */
/* the IAU frame has no segment at an evaluation's instant: a UTC epoch
 * before 1972 or an instant past the EOP table (GravityError::InvalidTime
 * from frame_rotation_at_checked, lightyear_odeint_rs/src/rhs.rs:3124-3174) */
#define BQP_ST_FRAME_TIME 17

/* force flags (ForceFlags, lightyear_odeint_rs/src/types.rs:266-286) */
#define BQP_FORCE_DRAG 1
#define BQP_FORCE_SRP 2 /* solar radiation pressure with binary eclipse (cr, p_sun below) */
#define BQP_FORCE_SUN 4
#define BQP_FORCE_MOON 8

/* steppers (StepperMethod, types.rs:148-157) */
#define BQP_METHOD_DOPRI5 0        /* solver.rs Dopri5 tableau, IntegratorConfig control */
#define BQP_METHOD_DOP853 1        /* StepperMethod::Dop853 */
#define BQP_METHOD_DOPRI5_COMPAT 2 /* StepperMethod::Dopri5Compat, Python method="dopri5" */
#define BQP_METHOD_VERN7 3         /* StepperMethod::Vern7 (tableau/vern7.rs), the Python default */
#define BQP_METHOD_VERN9 4         /* StepperMethod::Vern9 (tableau/vern9.rs) */

/* Force model and solver settings; replaces ForceConfig
 * (lightyear_odeint_rs/src/types.rs:332-411) as built by force_config()
 * (dust_transfer/src/lib.rs:128-190). */
typedef struct bqp_force_config {
    int32_t order;          /* spherical-harmonic degree/order, 0..120 */
    int32_t force_flags;    /* BQP_FORCE_* */
    int32_t atm_model;      /* JB2008 profile (AtmModel, lightyear_odeint_rs/src/rhs.rs:1607-1698;
                               jb_rs/src/jb2008.rs:339-838): 4 exact; 5, 6 the coarse log-quadrature
                               profiles; 7 the fitted kernel (the Python default) */
    int32_t method;         /* BQP_METHOD_* */
    int32_t error_control;  /* 0: absolute eps, max-norm; 1: scaled rtol/atol, RMS */
    int32_t ground_check;   /* 1: stop with BQP_ST_GROUND below 100 km altitude */
    double eps;             /* absolute tolerance (error_control 0) */
    double rtol, atol;      /* scaled tolerances (error_control 1) */
    double dt_max;          /* maximum step, s */
    double am_ratio, cd;    /* default ballistics: A/m (m^2/kg), drag coefficient */
    double earth_radius;    /* km, altitude geometry (WGS84 6378.137) */
    double omega_earth;     /* rad/s, co-rotating atmosphere */
    double mu_sun, mu_moon; /* km^3/s^2 */
    double jb_drivers[9];   /* F10.7, F10.7bar, S10, S10bar, M10, M10bar, Y10, Y10bar, dTc (K) */
    int64_t max_steps;      /* per rectification segment (MAX_STEPS = 500000) */
    int64_t max_attempts;   /* device watchdog: step attempts per trajectory */
    double max_kernel_seconds; /* watchdog: wall-clock limit of one propagation call (> 0);
                                  rows not finished by then end with BQP_ST_WATCHDOG */
    int32_t engine;            /* BQP_ENGINE_* */
    int32_t gravity_threads;   /* threads per CTA of the gravity kernels, 32..256 (0: 256) */
    int32_t gravity_slots;     /* trajectories per thread in the gravity kernels: 1, 2 or 4 (0: 4) */
    int32_t drag_quadrature;   /* 1: always walk the JB2008 Boole quadrature; 0: use the
                                  Chebyshev fits of its fixed-node sweeps where they apply */
    int32_t split_degree;      /* split precision: 0 plain FP64; d >= 4: spherical-harmonic
                                  degrees above d in FP32, the rest in FP64 (stage-synchronous
                                  engine and gravity evaluation) */
    int32_t drag_fp32;         /* split precision: 1 evaluates the JB2008 density in FP32 (the coarse
                                  profiles, atm_model 5-7; stage-synchronous engine and force calls) */
    int32_t surrogate;         /* 1: gravity = exact degrees <= BQP_SURROGATE_DEGREE + the trained
                                  surrogate (stage-synchronous engine; bqp_surrogate_train first) */
    double surrogate_check;    /* surrogate only: at each step's first stage the whole exact field
                                  is evaluated too; a row whose surrogate field misses it by more
                                  than this fraction of the whole field's magnitude (central term
                                  included; e.g. 1e-3) takes the exact field for the whole step.
                                  0: no check (no counterpart in the reference) */
    double cr;                 /* SRP reflectivity coefficient (Python cr, default 1.3) */
    double p_sun;              /* solar radiation pressure at 1 AU, N/m^2 (ForceConfig p_sun 4.56e-6).
                                  SRP acts on rows with BQP_FORCE_SRP and cr, p_sun, A/m all > 0; such
                                  rows run the reference's binary-eclipse coordinator
                                  (eclipse_coordinator.rs, events off): legs that hold the shadow side
                                  fixed, a crossing scan of every accepted step, a replay of the step
                                  that crossed and a committed root where the side flips.  Absolute
                                  error control and the dopri5 / dop853 / vern7 / vern9 steppers only. */
} bqp_force_config;

/* propagation engines */
#define BQP_ENGINE_PIPELINE 0   /* stage-synchronous: prep / gravity / drag / control kernels,
                                   CUDA-graph replay, active-list compaction */
#define BQP_ENGINE_PERSISTENT 1 /* one persistent kernel, one trajectory per thread, device
                                   work queue */

typedef struct bqp_ctx bqp_ctx;

/* Defaults of the reference's ForceConfig::default + Python kwargs. */
void bqp_force_config_default(bqp_force_config* cfg);

/* Last error message of the calling thread ("" if none). */
const char* bqp_last_error(void);

/* Parse a normalised "deg ord C S" coefficient text (D exponents and '#'
 * comments accepted), build the device field table and bind the force
 * configuration.  Replaces packed_constants_from_bytes
 * (lightyear_odeint_rs/src/config.rs:80-85,128-225) plus the per-context
 * state of ScalarPropagationContext (integrator.rs).  The context lives on
 * the CUDA device current at creation. */
int bqp_ctx_create(const char* coeff_text, int64_t text_len, const bqp_force_config* cfg,
                   bqp_ctx** out);
int bqp_ctx_destroy(bqp_ctx* ctx);
/* cudaStream_t to enqueue on (NULL: the legacy default stream). */
int bqp_ctx_set_stream(bqp_ctx* ctx, void* cuda_stream);
/* info[0]=order, [1]=table cells, [2]=table bytes, [3]=table staged in shared memory */
int bqp_ctx_info(const bqp_ctx* ctx, int64_t* info4);
/* Worst relative error of the JB2008 sweep fits against the quadrature at
 * the check points (-1: no fit, the quadrature always runs). */
int bqp_ctx_info_fit(const bqp_ctx* ctx, double* worst_rel);
/* Kernel timing, for measurement; no counterpart in the reference.  With
 * on != 0 the propagation calls of this context record a CUDA event on each
 * side of every kernel launch and add up the durations by kernel class
 * (BQP_KCLASS_*); the totals restart at zero.  While it is on, the
 * stage-synchronous engine waits for each graph replay before queueing the
 * next.  on == 0 stops recording and keeps the totals. */
#define BQP_KCLASS_PREP 0       /* stage preparation (baseline, frame, third body) */
#define BQP_KCLASS_GRAVITY 1    /* spherical-harmonic gravity */
#define BQP_KCLASS_DRAG 2       /* JB2008 density and drag (both altitude lists) */
#define BQP_KCLASS_CONTROL 3    /* step combination, error control, compaction */
#define BQP_KCLASS_PERSISTENT 4 /* the persistent engine's single kernel */
#define BQP_KCLASSES 5
int bqp_ctx_profile(bqp_ctx* ctx, int32_t on);
/* Totals since profiling was last switched on: ms[BQP_KCLASSES] kernel
 * milliseconds, launches[BQP_KCLASSES] kernel launches. */
int bqp_ctx_profile_read(const bqp_ctx* ctx, double* ms, int64_t* launches);

/* Builds, on the host only, the JB2008 sweep fits for a driver set
 * (drivers[9] as in bqp_force_config) and reports their self-check:
 * worst[0] the fixed-node 1-D fits, worst[1..3] the altitude-dependent 2-D
 * families (middle, up to 500 km, above 500 km; -1 when not built), worst[4],
 * worst[5] the T_inf range of the 2-D fits.  No counterpart in the
 * reference, whose quadrature these fits replace. */
int bqp_jb_fit_check(const double* drivers, double* worst6);

/* Eclipse crossing scan on given cubic Hermite paths, for tests (no
 * counterpart in the reference; eclipse.rs:341-491 is the scan itself).
 * paths [n][16]: p0[3], v0[3], p1[3], v1[3] (km, km/s), t0, t1 (s after the
 * epoch), the scan start (s) and the epoch (JD UTC); the context's Sun
 * (catalogue or analytic series) and Earth radius.  warp 0 runs the
 * per-thread walk of the persistent engine, 1 the warp-cooperative walk of
 * the stage-synchronous engine.  out [n][7]: status (BQP_ST_OK or an
 * eclipse code), found, old side, new side, t_old, t_new, motion bound. */
int bqp_ecl_scan_check(bqp_ctx* ctx, int64_t n, const double* paths, int32_t warp, double* out);

/* JB2008 density on the host, by the same function the force kernels run:
 * in[14 i] = UTC MJD, solar declination (rad), hour angle of the satellite
 * from the Sun (rad), geocentric latitude (rad), altitude (m), F10, F10bar,
 * S10, S10bar, M10, M10bar, Y10, Y10bar, dTc (K); out[i] kg/m^3, or a
 * negative code (-1 non-finite input, -2 altitude below 90 km, -3 angle out
 * of range, -4 non-positive index, -5 numerical domain).  model 4: the exact
 * quadrature (jb_rs/src/jb2008.rs:880); 5, 6, 7: the coarse profiles
 * (jb2008.rs:890-920, 7 = jb2008_density_fitted_v7).  fp32 != 0: a coarse
 * profile in FP32 arithmetic, as the split form's drag evaluates it (no
 * counterpart in the reference). */
int bqp_jb_density(int32_t model, int32_t fp32, int64_t n, const double* in14, double* out);

/* JB2008 space-weather tables: the SET SOLFSMY (daily F10, S10, M10, Y10 and
 * their 81-day centred means) and DTCFILE (hourly dTc, K) texts.  Replaces
 * Jb2008Drivers::from_set_bytes (jb_rs/src/drivers.rs:374-390, same checks,
 * 1025-1240) together with the per-evaluation lookup of the JB2008 adapter
 * (lightyear_odeint_rs/src/rhs.rs:3548-3571 calling drivers.rs:559-580):
 * after this call the context's propagations take the drivers at each force
 * evaluation's UTC instant from these tables (F10/S10 1 day lagged, M10 2,
 * Y10 5; dTc interpolated hourly and rounded) instead of cfg.jb_drivers, and
 * an instant the tables do not cover gives a NaN density, so the row ends
 * with BQP_ST_NON_FINITE.  [jd_lo, jd_hi] is the UTC span the propagations
 * will cover, which bounds the exospheric temperatures the drag sweep fits
 * are built for (0, 0: the whole table).  NULL texts: back to
 * cfg.jb_drivers.  BQP_E_ARG names the first rejected line. */
int bqp_ctx_set_jb_drivers(bqp_ctx* ctx, const char* solfsmy, int64_t solfsmy_len, const char* dtcfile,
                           int64_t dtcfile_len, double jd_lo, double jd_hi);
/* The drivers the force kernels would use at n UTC Julian days, evaluated by
 * the device lookup (Jb2008Drivers::lookup_utc_jd, drivers.rs:559-780):
 * out[9 i] = F10, F81c, S10, S81c, M10, M81c, Y10, Y81c, dTc; ok[i] = 1, or 0
 * with a NaN row where the tables do not cover the instant.  Host buffers. */
int bqp_ctx_jb_lookup(bqp_ctx* ctx, const double* utc_jd, int64_t n, double* out, int32_t* ok);
/* Precomputed Sun / Moon catalogues ("DUST" binary: 48-byte header, then
 * samples x 3 f64 Earth-centred ICRS km on a uniform UTC Julian-day grid).
 * Replaces PrecomputedEphemeris (lightyear_odeint_rs/src/precomputed_ephem.rs:
 * loader 680-830, linear interpolation 1066-1131) as the force model reads it
 * (rhs.rs:2964-3018): after this call the context's propagations take that
 * body's position by linear interpolation at each evaluation's UTC instant,
 * JD roundoff at an end clamped and any other instant outside the grid NaN
 * (the row then fails, BQP_ST_GRAVITY_RADIUS).  Without a catalogue the
 * analytic series apply.  bytes NULL: back to the series. */
#define BQP_BODY_SUN 0
#define BQP_BODY_MOON 1
int bqp_ctx_set_ephemeris(bqp_ctx* ctx, int32_t body, const uint8_t* bytes, int64_t len);

/* ---- IAU 2006/2000A Earth-fixed frame (satpy_core/src/frame_time/) ----
 * The Earth-fixed frame of gravity and drag.  BQP_FRAME_GMST (the default)
 * is the z-rotation by GMST of greenwichsrt_impl (satpy_core/src/lib.rs:
 * 905-936) with the atmosphere turning at cfg.omega_earth.  BQP_FRAME_IAU2006
 * replaces frame_rotation_at_checked (lightyear_odeint_rs/src/rhs.rs:
 * 3113-3174) over the reference's frame authority (frame_time/authority.rs):
 * per stage, R = GCRS->ITRS from 1800 s segments of the CIO-based IAU
 * 2006/2000A chain, gravity evaluated at R r and rotated back by R^T, the JB2008
 * inputs from R r and R r_sun, and the atmosphere turning with the frame's
 * own angular velocity (rhs.rs:1119-1163).  Time is continuous TAI from the
 * row's UTC epoch (rhs.rs:2754).  eop: n_records x 5 doubles per UTC day
 * from first_mjd (x_p arcsec, y_p arcsec, UT1-UTC s, dX mas, dY mas: the
 * layout of the reference's sealed eop_table.bin, which can be passed as
 * is with first_mjd 41684), interpolated by four-node Lagrange
 * (authority.rs:925-1022); NULL: zero EOP, over 1973 .. 2049.  Segments are
 * built on the host for each batch's time span and kept for the next
 * call.  Not with bqp_propagate_final_noalloc. */
#define BQP_FRAME_GMST 0
#define BQP_FRAME_IAU2006 1
int bqp_ctx_set_frame(bqp_ctx* ctx, int32_t mode, const double* eop, int32_t first_mjd, int32_t n_records);
/* Build and upload, once, the IAU frame's segments for the UTC Julian days
 * [jd_lo, jd_hi]; later calls then launch without reading their epochs back
 * to the host (the `_device` entry points stay asynchronous), and an
 * evaluation outside the span fails with BQP_ST_FRAME_TIME.  (0, 0): back to
 * segments per call. */
int bqp_ctx_set_frame_span(bqp_ctx* ctx, double utc_jd_lo, double utc_jd_hi);

/* The host functions below return -5 (NULL for _new) when host memory
 * cannot be had.
 * The chain's pieces on the host (no GPU), ERFA-restated (frame_time/
 * iau2006.rs, cio.rs, era.rs): dates are two-part TT Julian days (UT1 for
 * era).  nut: out[2] = dpsi, deps of IAU 2000A (iau2006 0) or 2006/2000A (1);
 * pfw06: out[4] = gamb, phib, psib, epsa; xys06a: out[3] = X, Y, s; c2ixys
 * and pom00: row-major r[9]. */
void bqp_frame_nut(double d1, double d2, int32_t iau2006, double* out);
double bqp_frame_obl06(double d1, double d2);
void bqp_frame_pfw06(double d1, double d2, double* out);
void bqp_frame_xys06a(double d1, double d2, double* out);
void bqp_frame_c2ixys(double x, double y, double s, double* r);
double bqp_frame_sp00(double d1, double d2);
void bqp_frame_pom00(double xp, double yp, double sp, double* r);
double bqp_frame_era(double ut1_1, double ut1_2);
/* UTC calendar instant -> two-part quasi-JD (ERFA dtf2d "UTC", timescale.rs:
 * 321-380; 23:59:60.x on a leap-second day).  0, or -1 on a bad instant. */
int bqp_frame_utc_calendar(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, double* out);
/* Continuous TAI seconds (from 0h TAI of MJD 41684) of UTC Julian days: one
 * part (utc_jd2 NULL; split as rhs.rs:3090-3093) or two.  Returns 1 and NaN
 * rows for instants before 1972. (authority.rs:1162-1190) */
int bqp_frame_tai_seconds(int64_t n, const double* utc_jd, const double* utc_jd2, double* tai_s);
/* GCRS->ITRS R[9] of the exact chain at a UTC calendar instant plus
 * `offset` s (frame_time/chain.rs frame_matrix: policy 0 zero EOP, 1 the
 * records' four-node Lagrange); and R, Rdot, Rddot from its centred
 * five-point stencil of step h (chain.rs derivatives). */
int bqp_frame_matrix(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, int32_t policy,
                     double offset, const double* eop, int32_t first_mjd, int32_t n_eop, double* r);
int bqp_frame_derivatives(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, int32_t policy,
                          double h, const double* eop, int32_t first_mjd, int32_t n_eop, double* r, double* rdot,
                          double* rddot);
/* A standalone segment authority (FrameAuthority, authority.rs:355-650) on
 * the host: intervals out[98] = n, 48 starts, 48 TAI - UTC, span end;
 * rotation: R [n][9] and ITRS angular velocity in GCRS [n][3] at TAI
 * instants (1 and NaN rows outside the span); segments: the keys and
 * [count][60] segments (M0..M2, K0..K2, theta cubic, centre, TAI - UTC)
 * holding [lo, hi], or -1 when more than cap. */
/* A GCRS position (km), velocity and acceleration in ITRS through the
 * stencil's R, Rdot, Rddot, summed in double-double (chain.rs
 * transform_state): r' = R r, v' = R v + Rdot r, a' = R a + 2 Rdot v + Rddot r. */
int bqp_frame_transform_state(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, int32_t policy,
                              double h, const double* eop, int32_t first_mjd, int32_t n_eop, const double* r,
                              const double* v, const double* a, double* r_out, double* v_out, double* a_out);
/* EOP records from IERS finals2000A text, by the reference's column rules
 * (frame_time/eop.rs load_eop): rows of >= 125 characters with I/P flags at
 * 16, 57, 95; x_p, y_p, UT1-UTC, dX, dY read from their fixed columns;
 * incomplete rows skipped.  Returns the length of the contiguous run of days
 * from the first complete one (*first_mjd its MJD), writing records [count][5]
 * when cap >= count (records NULL: size query); -3 for a day given twice. */
int64_t bqp_frame_eop_from_finals(const char* text, int64_t len, int64_t cap, int32_t* first_mjd,
                                  double* records);
typedef struct bqp_frame_authority bqp_frame_authority;
bqp_frame_authority* bqp_frame_authority_new(const double* eop, int32_t first_mjd, int32_t n_eop);
void bqp_frame_authority_free(bqp_frame_authority* h);
int bqp_frame_authority_intervals(const bqp_frame_authority* h, double* out);
int bqp_frame_authority_rotation(bqp_frame_authority* h, int64_t n, const double* tai, double* r, double* w);
int64_t bqp_frame_authority_segments(bqp_frame_authority* h, double lo, double hi, int64_t cap, int64_t* keys,
                                     double* segs);
/* Positions (km) of a body at n UTC Julian days as the force kernels take
 * them (catalogue or series), evaluated on the device.  Host buffers. */
int bqp_ctx_body_positions(bqp_ctx* ctx, int32_t body, const double* utc_jd, int64_t n, double* out);
/* Catalogue parsing and interpolation on the host, without a context:
 * n_samples[0] = the catalogue's sample count; out as above (n may be 0). */
int bqp_ephemeris_check(int32_t body, const uint8_t* bytes, int64_t len, const double* utc_jd, int64_t n,
                        double* out, int64_t* n_samples);

/* The same parsing and lookup on the host, without a context or a device:
 * counts2[0], counts2[1] = parsed SOLFSMY and DTCFILE rows, then n lookups as
 * in bqp_ctx_jb_lookup (n may be 0).  BQP_E_ARG names a rejected line. */
int bqp_jb_drivers_check(const char* solfsmy, int64_t solfsmy_len, const char* dtcfile, int64_t dtcfile_len,
                         const double* utc_jd, int64_t n, double* out, int32_t* ok, int64_t* counts2);

/* Replace the force/solver settings of a context (the field is kept; the
 * order may only shrink up to the parsed order). */
int bqp_ctx_set_config(bqp_ctx* ctx, const bqp_force_config* cfg);

/* Full-field gravity (C00 included) at Earth-fixed positions.
 * Replaces spherical_gravity_impl_frame_packed
 * (satpy_core/src/gravity.rs:2638-2675). pos [n][3] km -> acc [n][3] km/s^2.
 * status[n] (nullable): BQP_ST_OK, BQP_ST_GRAVITY_RADIUS, or BQP_ST_WATCHDOG when
 * the field table's copy into shared memory did not land within 1 s. */
int bqp_gravity_eval(bqp_ctx* ctx, int64_t n, const double* pos_km, double* acc_km_s2,
                     int32_t* status);
int bqp_gravity_eval_device(bqp_ctx* ctx, int64_t n, const double* d_pos_km, double* d_acc,
                            int32_t* d_status);

/* One Encke force evaluation per row: d(delta)/dt = [dv, a] of the deviation
 * from the baseline orbit of elements equ (valid at seg_t0), at time t (s
 * after epoch_jd).  Replaces LightyearRHS::compute_internal
 * (lightyear_odeint_rs/src/rhs.rs:3872-4118).  ballistic [n][2] nullable. */
int bqp_rhs_eval(bqp_ctx* ctx, int64_t n, const double* equ, const double* seg_t0,
                 const double* epoch_jd, const double* t, const double* delta,
                 const double* ballistic, double* out);
int bqp_rhs_eval_device(bqp_ctx* ctx, int64_t n, const double* equ, const double* seg_t0,
                        const double* epoch_jd, const double* t, const double* delta,
                        const double* ballistic, double* out);

/* Final-state propagation of a batch with per-row epoch, end time and
 * ballistics, Encke rectification every 5400 s / 10 km.  Replaces
 * integrate_final_checked (integrator.rs:3197) per row and
 * LightyearSession::integrate_variable_final_into (session.rs:2325-2430).
 * in [n][6]: ECI (input_equinoctial = 0) or equinoctial elements at t0.
 * epoch_jd[n], tf[n] (s after epoch, >= t0), ballistic [n][2] nullable.
 * out [n][6]: ECI at tf.  status/steps/evals per row (steps/evals nullable). */
int bqp_propagate_final(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equinoctial,
                        const double* epoch_jd, double t0, const double* tf,
                        const double* ballistic, double* out, int32_t* status, int64_t* steps,
                        int64_t* evals);
int bqp_propagate_final_device(bqp_ctx* ctx, int64_t n, const double* in,
                               int32_t input_equinoctial, const double* epoch_jd, double t0,
                               const double* tf, const double* ballistic, double* out,
                               int32_t* status, int64_t* steps, int64_t* evals);

/* Final-state propagation that allocates no memory.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they propagate -- a host application whose device memory is all reserved in
 * its own pool at start-up, or a loop that must not let a cudaFree stall the
 * whole device -- and who still want host buffers in and out.
 *
 * Same arguments, results and per-row status as bqp_propagate_final, always
 * on the persistent kernel (whatever cfg.engine says) with the plain FP64
 * field: a context configured for split precision, the learned surrogate or
 * the FP32 density (forms only the stage-synchronous engine runs), or for
 * binary-eclipse SRP (whose per-row coordinator state the fixed array has
 * no room for), or for the IAU frame (whose segment table is built per call),
 * is refused with BQP_E_UNSUPPORTED.  The JB2008 sweep fits it uses are the ones the
 * context built when it was created or last reconfigured (bqp_ctx_set_config,
 * bqp_ctx_set_jb_drivers), so identical calls give identical bits whatever
 * was called in between.  With bqp_ctx_profile on, its kernel time counts
 * under BQP_KCLASS_PERSISTENT.  The inputs and
 * outputs are staged through one fixed device array inside the library, of
 * room for BQP_NOALLOC_MAX_TRAJ rows (about 2.3 MiB), which every GPU that
 * loads the library holds until the process exits; n above that limit is
 * rejected with BQP_E_ARG before any device work.  The call makes no
 * cudaMalloc, cudaFree or host-pinning call; the context (created earlier)
 * holds the gravity table.
 *
 * The first call on a device looks up that array's device address (and loads
 * the kernel), so make it during set-up, before any stream capture.  Every
 * call on a device shares the array and the next call overwrites it.  Calls
 * made through this library are serialised by a lock and each returns only
 * after its stream has finished, so two such calls never overlap on the GPU;
 * calls that did overlap (for example from two copies of the library in one
 * process) would race on the array. */
#define BQP_NOALLOC_MAX_TRAJ 16384
int bqp_propagate_final_noalloc(bqp_ctx* ctx, int64_t n, const double* in,
                                int32_t input_equinoctial, const double* epoch_jd, double t0,
                                const double* tf, const double* ballistic, double* out,
                                int32_t* status, int64_t* steps, int64_t* evals);

/* Sampled propagation on a common grid t_eval[n_t] (sorted, within
 * [t0, tf_i], containing t0 and tf_i as the reference's binding arranges,
 * lib.rs:277-290).  Replaces integrate_adaptive's rectified sampled path
 * (integrator.rs:2313-2416, 2426) and integrate_batch_native_into
 * (batch.rs:247-391).  out [n][n_t][6]: ECI states (out_deltas = 0) or Encke
 * deviations against the initial baseline (out_deltas = 1, the batch API). */
int bqp_propagate_sampled(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equinoctial,
                          const double* epoch_jd, double t0, const double* tf, int32_t n_t,
                          const double* t_eval, int32_t out_deltas, double* out,
                          int32_t* status, int64_t* steps, int64_t* evals);
int bqp_propagate_sampled_device(bqp_ctx* ctx, int64_t n, const double* in,
                                 int32_t input_equinoctial, const double* epoch_jd, double t0,
                                 const double* tf, int32_t n_t, const double* t_eval,
                                 int32_t out_deltas, double* out, int32_t* status,
                                 int64_t* steps, int64_t* evals);

/* Sigma-point (unscented) covariance propagation: per object, the sigma
 * points of (mean[6], cov[6][6] row-major) are generated on the device,
 * propagated as ordinary rows from t0 to tf[i] (epoch, ballistics as for
 * bqp_propagate_final, ECI in and out), and recombined on the device into
 * mean_out[6] and the symmetrised cov_out[6][6].  Replaces get_sigmas_ukf
 * and rebuild_mean_covar_ukf (dust_ukf_rs/src/lib.rs:247-275, 277-312)
 * around the batch propagation.  sigma_set BQP_SIGMA_JULIER7: the
 * reference's 7-point simplex at W0 = 0 (lib.rs:22-37, 69-78; alpha, beta,
 * kappa unused); BQP_SIGMA_MERWE13: the scaled 13-point set of Wan & van der
 * Merwe (alpha, beta, kappa).  A covariance that does not factorise is
 * repaired as the reference does (eigenvalues floored at 1e-12,
 * lib.rs:202-240); status[i] is BQP_ST_INVALID_INPUT when even that fails,
 * else the first failing sigma row's status.  evals[i] (nullable): force
 * evaluations over the object's sigma rows. */
#define BQP_SIGMA_JULIER7 0
#define BQP_SIGMA_MERWE13 1
int bqp_sigma_propagate(bqp_ctx* ctx, int64_t n, const double* mean, const double* cov,
                        int32_t sigma_set, double alpha, double beta, double kappa,
                        const double* epoch_jd, double t0, const double* tf,
                        const double* ballistic, double* mean_out, double* cov_out,
                        int32_t* status, int64_t* evals);
int bqp_sigma_propagate_device(bqp_ctx* ctx, int64_t n, const double* mean, const double* cov,
                               int32_t sigma_set, double alpha, double beta, double kappa,
                               const double* epoch_jd, double t0, const double* tf,
                               const double* ballistic, double* mean_out, double* cov_out,
                               int32_t* status, int64_t* evals);
/* The weights and offsets of a sigma set (host only): points (7 or 13),
 * wm/wc[points], offsets[7][6] (Julier; zero for Merwe).  Any output may be
 * NULL. */
int bqp_sigma_weights(int32_t sigma_set, double alpha, double beta, double kappa, int32_t* points,
                      double* wm, double* wc, double* offsets);

/* BF16 tensor-core GEMM of the gravity surrogate, exported for its tests (no
 * counterpart in the reference): c[m][n] (FP32) = a[m][k] b[n][k]^T with
 * BF16 row-major device operands, m % 128 == 0, n % 256 == 0, k % 64 == 0;
 * enqueued on `stream` and synchronised. */
int bqp_gemm_bf16_device(int64_t m, int64_t n, int64_t k, const void* a, const void* b, float* c,
                         void* stream);

/* Learned gravity surrogate.  An MLP (input: body-fixed unit vector and
 * scaled radius; 4 hidden layers of 256, SiLU; output: the acceleration of the
 * degrees above BQP_SURROGATE_DEGREE times (r/R)^2, normalised) trained on the
 * GPU with BF16 tensor-core forward and backward GEMMs (FP32 accumulation) and
 * Adam on FP32 masters.  No counterpart in the reference (its learned parts
 * are elsewhere); the samples come from the context's own exact field.
 *
 * train: `samples` positions uniform in radius 6578-7578 km and on the sphere,
 * targets from the exact harmonic kernel (context order) minus degrees <= 8;
 * `epochs` passes of minibatches of `batch` (multiple of 128); Adam, cosine
 * decay from lr; loss_per_epoch[epochs] (nullable): mean squared error of the
 * normalised targets.
 * infer: pos[n][3] Earth-fixed km -> acc[n][3] km/s^2: the predicted residual
 * (add_low bit 0 clear) or the exact degree <= 8 field (C00 included) plus it
 * (bit 0 set).  The network runs as one fused kernel (weights staged per layer
 * by bulk copy, activations in shared and tensor memory); bit 1 selects the
 * layer-by-layer kernels used in training instead, for checking.
 * params / set_params: the BQP_SURROGATE_PARAMS FP32 parameters and the
 * output scale sigma.  grad: loss and gradient of given parameters on one
 * batch (x[batch][4], normalised targets t[batch][3]), for checking. */
#define BQP_SURROGATE_DEGREE 8
#define BQP_SURROGATE_PARAMS 199427
int bqp_surrogate_train(bqp_ctx* ctx, int64_t samples, int32_t epochs, int32_t batch, double lr,
                        uint64_t seed, double* loss_per_epoch);
int bqp_surrogate_infer(bqp_ctx* ctx, int64_t n, const double* pos_km, double* acc, int32_t add_low);
int bqp_surrogate_infer_device(bqp_ctx* ctx, int64_t n, const double* d_pos_km, double* d_acc,
                               int32_t add_low);
int bqp_surrogate_params(bqp_ctx* ctx, float* params, double* sigma);
int bqp_surrogate_set_params(bqp_ctx* ctx, const float* params, double sigma);
int bqp_surrogate_grad(bqp_ctx* ctx, int32_t batch, const float* params, const float* x, const float* t,
                       float* grad, double* loss, float* y);

/* UTC Julian day of each force evaluation as the kernels form it, on the
 * host: out[i] = the instant t[i] elapsed (SI/TAI) seconds after the UTC
 * epoch jd0[i], with UTC days that end in a leap second running over 86,401 s
 * (the reference's TAI integration time and its taiutc lookup seam,
 * lightyear_odeint_rs/src/rhs.rs:3090-3110, 3264-3300).  Without a
 * leap-second day within a day of the arc it is jd0 + t/86400. */
int bqp_utc_jd(int64_t n, const double* jd0, const double* t, double* out);

/* Element conversions on the host (no GPU).  eci_to_equinoctial replaces
 * eci2equinoc_impl (satpy_core/src/lib.rs:1738-1870; ok[i] = 0 on an
 * unbound or degenerate orbit); equinoctial_to_eci replaces equinoc2eci_impl
 * (lib.rs:2580-2591) at tof[i] seconds; kep_to_eci / eci_to_kep replace the
 * Python kep_to_eci / eci_to_kep (dust_transfer/src/lib.rs:200-221):
 * [a_km, e, i_deg, raan_deg, argp_deg, true_anomaly_deg]. */
int bqp_eci_to_equinoctial(int64_t n, const double* eci, double* equ, int32_t* ok);
int bqp_equinoctial_to_eci(int64_t n, const double* equ, const double* tof, double* eci);
int bqp_kep_to_eci(int64_t n, const double* kep, double* eci);
int bqp_eci_to_kep(int64_t n, const double* eci, double* kep);

#ifdef __cplusplus
}
#endif
#endif /* BQP_PROP_H */
