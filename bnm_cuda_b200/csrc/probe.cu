// FP32 FMA-pipe throughput probe.  The measured peak tables in the repo hold
// HBM copy bandwidth and tensor-core GEMM rates only; the integrator is bound
// by the FP32 pipe, so its roofline denominator is measured here: eight
// independent chains of packed FP32 FMA (fma.rn.f32x2) per thread, enough
// CTAs for every SM, timed with CUDA events.
#include <cuda_runtime.h>
#include "../../include/bnm_b200.h"
#include "kernels.h"
#include "fp32_model.cuh"

int bnm_fail_cuda(cudaError_t e, const char* expr, const char* file, int line);
int bnm_fail_msg(int code, const char* msg);

__global__ void __launch_bounds__(256) ffma2_probe_kernel(float* out, int iters) {
    float2 a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = make_float2(1.0f + 1e-3f * threadIdx.x + i, 0.5f + 1e-3f * i);
    const float2 m = make_float2(0.99999f, 1.00001f), c = make_float2(1e-6f, -1e-6f);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = __ffma2_rn(a[i], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; i++) s += a[i].x + a[i].y;
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

extern "C" int bnm_measure_fp32_peak(int32_t device, double* tflops) {
    BNM_CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    BNM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = sms * 8, block = 256, iters = 1 << 15;
    float* out = nullptr;
    BNM_CUDA_TRY(cudaMalloc(&out, (size_t)grid * block * sizeof(float)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        ffma2_probe_kernel<<<grid, block>>>(out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    BNM_CUDA_TRY(err);
    const double flops = (double)grid * block * iters * 8 * 2 * 2;
    *tflops = flops / (best * 1e-3) / 1e12;
    return BNM_OK;
}

// expm1_bw / log1p_bw (the Balloon-Windkessel step's e^y - 1 and ln(1 + x))
// next to CUDA's expm1f / log1pf on the same inputs.
__global__ void bw_math_probe_kernel(const float* x, int n, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = x[i];
    out[4 * i + 0] = bnm::expm1_bw(v);
    out[4 * i + 1] = expm1f(v);
    out[4 * i + 2] = bnm::log1p_bw(v);
    out[4 * i + 3] = log1pf(v);
}

extern "C" int bnm_bw_math_probe(int32_t device, const float* x, int32_t n, float* out4) {
    if (!x || !out4 || n < 1) return BNM_EINVAL;
    BNM_CUDA_TRY(cudaSetDevice(device));
    float *dx = nullptr, *dout = nullptr;
    BNM_CUDA_TRY(cudaMalloc(&dx, (size_t)n * sizeof(float)));
    cudaError_t e = cudaMalloc(&dout, (size_t)n * 4 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        bw_math_probe_kernel<<<(n + 255) / 256, 256>>>(dx, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out4, dout, (size_t)n * 4 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dx);
    if (dout) cudaFree(dout);
    BNM_CUDA_TRY(e);
    return BNM_OK;
}

// Failure detection of the bounded device waits, exercised without a fault:
// one CTA initialises an mbarrier that nothing ever arrives on (no bulk copy,
// no MMA and no other thread is involved) and waits on its first phase with
// the integrators' own mbar_wait and the given wall-clock limit.  The wait
// must give up, the kernel records the timeout status and the elapsed time,
// and returns normally, so the context stays usable.
__global__ void wait_probe_kernel(long long limit_ns, int* status, unsigned long long* elapsed_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bnm::smem_addr(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const unsigned long long t0 = bnm::global_ns();
    const bool ok = bnm::mbar_wait(bnm::smem_addr(&bar), 0, limit_ns);
    const unsigned long long t1 = bnm::global_ns();
    if (__syncthreads_or(!ok) && threadIdx.x == 0) {
        atomicOr(status, bnm::kStatusTimeout);
        *elapsed_ns = t1 - t0;
    }
}

extern "C" int bnm_wait_probe(int32_t device, int64_t limit_ns, int32_t* status_out, double* elapsed_ms) {
    if (limit_ns < 0 || limit_ns > bnm::kWaitNs) return bnm_fail_msg(BNM_EINVAL, "wait probe: limit out of range");
    BNM_CUDA_TRY(cudaSetDevice(device));
    int* d_status = nullptr;
    unsigned long long* d_ns = nullptr;
    BNM_CUDA_TRY(cudaMalloc(&d_status, 2 * sizeof(int) + sizeof(unsigned long long)));  // status, pad, elapsed
    d_ns = reinterpret_cast<unsigned long long*>(d_status + 2);
    cudaError_t e = cudaMemset(d_status, 0, sizeof(int) * 2 + sizeof(unsigned long long));
    if (e == cudaSuccess) {
        wait_probe_kernel<<<1, 64>>>((long long)limit_ns, d_status, d_ns);
        e = cudaGetLastError();
    }
    int status = 0;
    unsigned long long ns = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&ns, d_ns, sizeof(ns), cudaMemcpyDeviceToHost);
    cudaFree(d_status);
    BNM_CUDA_TRY(e);
    if (status_out) *status_out = status;
    if (elapsed_ms) *elapsed_ms = ns * 1e-6;
    if (status & bnm::kStatusTimeout) return bnm_fail_msg(BNM_ETIMEOUT, "wait probe: the bounded wait gave up");
    return BNM_OK;
}
