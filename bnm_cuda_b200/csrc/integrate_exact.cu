// Reference-order integrators, compiled with -fmad=false (no FMA contraction)
// so their arithmetic is the reference CPU build's: FP64 (default u_real) and
// FP32 in the reference's USE_FLOATS operand types.  These are the parity
// kernels of the oracle-noise mode; see integrate_generic.cuh.
#include "kernels.h"
#define BNM_GENERIC_NS exact
#include "integrate_generic.cuh"

cudaError_t bnm_launch_integrate_exact(const bnm::SimArgs& a, int fp64, int num_sms, cudaStream_t st) {
    using namespace bnm;
    const int threads = ((a.N + 31) / 32) * 32;
    if (threads > 1024) return cudaErrorInvalidValue;
    const size_t elt = fp64 ? sizeof(double) : sizeof(float);
    size_t smem = 2 * (size_t)threads * elt;
    const size_t sc_bytes = (size_t)a.N * (fp64 ? a.N : a.sc_ld) * elt;
    const int sc_in_smem = (smem + sc_bytes) <= 200 * 1024;
    if (sc_in_smem) smem += sc_bytes;
    const int grid = a.n_sims < 2 * num_sms ? a.n_sims : 2 * num_sms;
    cudaError_t e;
    if (fp64) {
        e = cudaFuncSetAttribute(exact::integrate_generic_kernel<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        exact::integrate_generic_kernel<double><<<grid, threads, smem, st>>>(a, sc_in_smem);
    } else {
        e = cudaFuncSetAttribute(exact::integrate_generic_kernel<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        exact::integrate_generic_kernel<float><<<grid, threads, smem, st>>>(a, sc_in_smem);
    }
    return cudaGetLastError();
}
