// Launch interface between the C ABI (bqp_api.cu) and the kernels (propagate.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "gravity_cta.cuh"
#include "kernels.cuh"

namespace bqp {

// A trained gravity surrogate, as the propagation's gravity stage uses it.
struct SurrogateRef {
    const float* P;                    // FP32 parameters (null: no surrogate)
    const __nv_bfloat16* Wtile;        // hidden matrices in the tensor cores' layout
    double R, r_mid, r_half, sigma;    // output and input scaling
    int* err;                          // set when a tensor-core wait timed out
    GravTable low;                     // exact table of the degrees the network leaves out
    GravTable full;                    // the whole exact field (the per-step check's fallback)
    double check;                      // residual check threshold (0: none)
};

// Arguments of k_propagate (all device pointers).
struct PropArgs {
    int64_t n;                     // trajectories
    const double* in;              // [n][6] ECI or equinoctial at t0
    int32_t input_equinoctial;
    const double* epoch;           // [n] JD (UTC) of t = 0
    double t0;                     // common start, seconds after epoch
    const double* tf;              // [n] end time, seconds after epoch
    const double* ballistic;       // [n][2] (A/m m^2/kg, Cd) or null
    double am0, cd0;               // defaults when ballistic is null
    const double* t_eval;          // [n_t] common sample grid (sampled modes)
    int32_t n_t;
    int32_t out_mode;              // 0 final ECI [n][6]; 1 sampled ECI; 2 sampled deltas [n][n_t][6]
    double* out;
    int32_t* status;               // [n]
    int64_t* steps;                // [n] or null
    int64_t* evals;                // [n] or null
    unsigned long long* queue;     // work-queue head, zeroed before launch
    const double* gtab;            // gravity table (global), FP64 cells (the Encke force call)
    int32_t ncells;
    int32_t use_smem;
    GravTable grav;                // the gravity stage's table (plain or split precision)
    SurrogateRef sur;              // gravity stage through the surrogate (sur.P != null)
    ForceParams force;
    CtrlParams ctrl;
    const jb::JbFit* fit_host;     // host copy of *force.fit (null with it): the stage-synchronous
                                   // drag kernel takes it by value, in kernel parameter space
    struct EclState* ecl;          // [n] eclipse coordinator state of SRP rows (null without SRP)
};

struct TrajState;

// Device buffers of the stage-synchronous engine.  Per-trajectory controller
// state is an array of TrajState; everything per stage is indexed by the
// trajectory's slot in the active list of the current attempt (so the force
// kernels read contiguous, coalesced arrays).
struct PipeBufs {
    int64_t cap;          // slots (= trajectories)
    TrajState* st;        // [cap]
    int32_t* idx[2];      // active lists (slot -> trajectory), double-buffered
    int32_t* count;       // [2] active counts
    double* k;            // [(S+1)][6][cap] stage derivatives
    double* sp;           // [6][cap] perturbed state of the stage (ECI)
    double* sc;           // [2][cap] sin, cos of the GMST angle
    double* fr;           // [12][cap] IAU frame: R (row-major) and ITRS angular velocity (GCRS)
    int32_t iau;          // 1: the Earth-fixed frame is fr (IAU 2006/2000A), 0: sc (GMST)
    double* sun;          // [3][cap] Sun position (ECI), drag only
    double* part;         // [3][cap] third-body + Battin acceleration (ECI)
    double* agrav;        // [3][cap] gravity (Earth-fixed)
    double* adrag;        // [3][cap] drag (ECI)
    double* jd;           // [cap]
    double* amcd;         // [2][cap]
    int32_t* skip;        // [cap] 1: stage derivative reused, no force call
    int32_t* bad;         // [cap] latched invalid-radius gravity error
    int32_t* dlist[2];    // drag work lists of the stage: 0 above ~510 km (sweep fits), 1 below
    int32_t* dcount;      // [2]
    double* ef;           // [cap][3] Earth-fixed positions of the stage (surrogate gravity)
    // surrogate residual check (surrogate with a check only)
    double* agx;          // [3][cap] the exact field of the step's first stage
    int32_t* fall;        // [cap] by trajectory: 1 while the row's step takes the exact field
    int32_t* flist;       // [cap] slots of this step's rows on the exact field
    int32_t* fcount;      // [1]
};

// Kernel durations by class, summed from CUDA events recorded around each
// launch (instrumentation; null when off).
enum KernelClass { kKcPrep = 0, kKcGravity = 1, kKcDrag = 2, kKcControl = 3, kKcPersistent = 4, kKcCount = 5 };
struct KernelTimes {
    double ms[kKcCount];
    int64_t launches[kKcCount];
};

size_t pipeline_bytes(int64_t cap);
void pipeline_carve(PipeBufs& P, void* base, int64_t cap);
cudaError_t launch_pipeline(const PropArgs& A, const PipeBufs& P, int method, cudaStream_t st,
                            double max_seconds, int gravity_threads, int gravity_slots,
                            KernelTimes* times = nullptr);

cudaError_t launch_gravity(const GravTable& T, int64_t n, const double* pos, double* acc, int32_t* status,
                           cudaStream_t st, int threads = 256, int slots = 4);
cudaError_t launch_rhs(const double* gtab, int ncells, int use_smem, const ForceParams& fp, int64_t n,
                       const double* equ, const double* seg_t0, const double* jd0, const double* t,
                       const double* delta, const double* ballistic, double am0, double cd0,
                       double* out, cudaStream_t st);
cudaError_t launch_propagate(const PropArgs& A, int method, int threads, int blocks, cudaStream_t st);
cudaError_t launch_ecl_scan(const ForceParams& fp, int64_t n, const double* paths, double* out, int warp,
                            cudaStream_t st);
cudaError_t launch_jb_lookup(const jb::DriverTable& T, const double* jd, int64_t n, double* out, int32_t* ok,
                             cudaStream_t st);
cudaError_t launch_body_positions(const EphemTable& E, int body, const double* jd, int64_t n, double* out,
                                  cudaStream_t st);
cudaError_t launch_sigma_gen(int64_t n, int set, double scale, const double* offsets, const double* mean,
                             const double* cov, const double* epoch, const double* tf, const double* ballistic,
                             double* rows, double* row_epoch, double* row_tf, double* row_bal, int32_t* status,
                             cudaStream_t st);
cudaError_t launch_sigma_recombine(int64_t n, int S, const double* wm, const double* wc, const double* rows,
                                   const int32_t* row_status, const int64_t* row_evals, double* mean_out,
                                   double* cov_out, int32_t* status, int64_t* evals, cudaStream_t st);
int device_sm_count();
// C[M x N] (FP32) = A[M x K] B[N x K]^T, BF16 row-major operands (mlp.cu);
// M % 128, N % 256, K % 64 == 0.  *err is set if a wait timed out.
// The surrogate's residual at the first *n_dev positions pos[i][3], added to
// out[i * si + k * sk] (surrogate.cu).  Grid sized for up to cap rows.
cudaError_t launch_surrogate_stage(const SurrogateRef& S, const int32_t* n_dev, int64_t cap, const double* pos,
                                   double* out, int64_t si, int64_t sk, cudaStream_t st);
cudaError_t launch_gemm_bf16(int64_t M, int64_t N, int64_t K, const void* A, const void* B, float* C, int* err,
                             cudaStream_t st);

}  // namespace bqp
