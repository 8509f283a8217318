// Test infrastructure, not product code: a launcher for the reference's own
// CUDA gravity kernel, spherical_gravity_batch_dense
// (satpy_core/kernels/cuda/gravity.cu:117-317), which the reference ships but
// never launches.  The kernel source is compiled where it lies in the
// reference tree (oracle/Makefile's `ref` target passes its path in
// REF_GRAVITY_CU); nothing of it is copied here.  The library's tests use the
// launcher to check that kernel against the oracle and to time it beside the
// library's own gravity kernel on the same positions.
//
// Its layout (from the reference's comments): one block of 32 threads per
// state, V/W in a per-state global scratch of 2 x 131 x 131 doubles,
// unnormalised dense C/S with a given stride, GCRS positions and a 3x3
// GCRS->ITRS rotation in, GCRS accelerations (central term included) out.
#include <cuda_runtime.h>

#include <cstdint>

#ifndef REF_GRAVITY_CU
#error "REF_GRAVITY_CU must name the reference's gravity.cu"
#endif
#include REF_GRAVITY_CU

extern "C" {

// doubles of scratch one state needs (2 x MAX_REC x MAX_REC)
int64_t refgrav_scratch_doubles_per_state(void) { return 2LL * MAX_REC * MAX_REC; }

// Launch on `stream` (no synchronisation); returns the cudaError_t value.
int refgrav_launch(int64_t n, const double* d_states6, const double* d_rot9, int order, int stride,
                   const double* d_c, const double* d_s, double* d_acc3, double* d_scratch, void* stream) {
    if (n <= 0) return 0;
    if (order + 2 > MAX_REC || stride > MAX_REC) return (int)cudaErrorInvalidValue;
    spherical_gravity_batch_dense<<<(unsigned)n, 32, 0, (cudaStream_t)stream>>>(
        d_states6, d_rot9, order, stride, d_c, d_s, d_acc3, d_scratch);
    return (int)cudaGetLastError();
}

}  // extern "C"
