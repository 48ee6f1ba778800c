// FP32 integrator for N <= 128: structural connectivity held in registers.
//
// Same model and time loop as the reference's bnm kernel (bnm.cu:72-315) and
// CPU path (bnm.cpp:167-290), re-laid out for Blackwell:
//   * one thread per node, one CTA per particle (persistent over particles,
//     two CTAs per SM); the CTA's SC block is staged once into shared memory
//     with a TMA bulk copy (cp.async.bulk + mbarrier, no multicast), then each
//     thread keeps its SC row in registers for the whole run, so the coupling
//     sum G*J*(SC.S_E) reads only the broadcast S_E vector from shared memory;
//   * the coupling row-dot uses packed FP32 FMA (fma.rn.f32x2, __ffma2_rn)
//     over column pairs with four independent accumulators;
//   * S_E is double buffered in shared memory so a substep needs one barrier;
//   * the next millisecond's noise (10 substeps x (E, I)) is prefetched into
//     registers while the current one is integrated;
//   * firing rates use ex2.approx / rcp.approx with an exact-limit series for
//     |d(aI-b)| < 0.1, where 1-exp(-u) cancels (the reference FP32 build
//     clamps |aI-b| to 1e-4 instead, bnm.cu:195-199);
//   * FIC sampling and the extended-output sums accumulate in FP64.
#include "kernels.h"
#define BNM_GENERIC_NS fastgen
#include "integrate_generic.cuh"

namespace bnm {

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// r = x / (1 - exp(-d x)); for |d x| < 0.1 the quotient is evaluated as
// (1/d) / P(u) with P(u) = (1 - e^-u)/u truncated after u^4 (rel. err < 2e-8).
__device__ __forceinline__ float rate(float x, float d, float inv_d, float neg_d_log2e) {
    const float u = d * x;
    const float e = ex2_approx(x * neg_d_log2e);
    float p = fmaf(u, 1.0f / 120.0f, -1.0f / 24.0f);
    p = fmaf(p, u, 1.0f / 6.0f);
    p = fmaf(p, u, -0.5f);
    p = fmaf(p, u, 1.0f);
    const bool small = fabsf(u) < 0.1f;
    const float num = small ? inv_d : x;
    const float den = small ? p : (1.0f - e);
    return num * rcp_approx(den);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded wait on an mbarrier phase; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long max_iter) {
    for (long long i = 0; i < max_iter; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

template <int KMAX>
__global__ void __launch_bounds__(128, 2) integrate_fast_kernel(SimArgs a) {
    static_assert(KMAX % 8 == 0 && KMAX <= 128, "KMAX");
    typedef Model<float> C;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // layout: [SC stage: N*KMAX floats][S: 2*KMAX floats][mbarrier]
    const int N = a.N;
    float* sc_stage = reinterpret_cast<float*>(smem_raw);
    float* S_buf = sc_stage + (size_t)N * KMAX;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(S_buf + 2 * KMAX);
    __shared__ int s_sim;

    const int j = threadIdx.x;
    const bool act = j < N;

    // ---- stage SC into shared memory with one TMA bulk copy --------------
    const uint32_t bar = smem_addr(mbar);
    const uint32_t bytes = (uint32_t)(N * KMAX * sizeof(float));
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(sc_stage)),
            "l"(a.sc_f32), "r"(bytes), "r"(bar)
            : "memory");
    }
    if (!mbar_wait(bar, 0, 1ll << 26)) {
        if (threadIdx.x == 0) atomicOr(a.status, kStatusTimeout);
        // the copy may still land in shared memory; wait (bounded) before exiting
        mbar_wait(bar, 0, 1ll << 26);
        return;
    }
    float2 sc[KMAX / 2];
#pragma unroll
    for (int m = 0; m < KMAX / 2; m++) {
        sc[m] = act ? reinterpret_cast<const float2*>(sc_stage + (size_t)j * KMAX)[m] : make_float2(0.f, 0.f);
    }

    const float2* noise2 = reinterpret_cast<const float2*>(a.noise);
    const size_t sub_stride = (size_t)N;  // float2 entries per substep
    const double duration = (double)(a.samp_end - a.samp_start + 1);
    const float SQ = C::sigma_model * C::sqrt_dt;
    const float LOG2E = 1.4426950408889634f;
    const float log2_1mrho = -0.59946207279f;  // log2(1 - 0.34)

    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_sim = atomicAdd(a.work_counter, 1);
        __syncthreads();
        const int sim = s_sim;
        if (sim >= a.n_sims) break;

        const float GJ = (float)a.G[sim] * C::J_NMDA;
        const float wEE = act ? (float)a.wEE[(size_t)sim * N + j] : 0.f;
        const float wEI = act ? (float)a.wEI[(size_t)sim * N + j] : 0.f;
        float wIE = act ? (float)a.wIE[(size_t)sim * N + j] : 0.f;
        float delta = (float)a.init_delta;
        float S_E = 0.001f, S_I = 0.001f, x = 0.f, f = 1.f, nu = 1.f, q = 1.f;
        float IE = 0.f, II = 0.f, rE = 0.f, rI = 0.f;
        double mean_IE = 0.0;
        double ext[6] = {0, 0, 0, 0, 0, 0};
        for (int k = threadIdx.x; k < 2 * KMAX; k += blockDim.x) S_buf[k] = (k < N) ? S_E : 0.f;
        int cur = 0, trial = 0, ts = 0, frame = 0;
        bool failed = false, adjusting = a.adjust_fic != 0;

        float2 nz[10], nz_next[10];
#pragma unroll
        for (int s = 0; s < 10; s++) nz[s] = act ? __ldg(noise2 + (size_t)s * sub_stride + j) : make_float2(0.f, 0.f);
        __syncthreads();

        while (ts <= a.T) {
            // prefetch the next millisecond's noise
            if (act && ts < a.T) {
                const float2* src = noise2 + ((size_t)(ts + 1) * 10) * sub_stride + j;
#pragma unroll
                for (int s = 0; s < 10; s++) nz_next[s] = __ldg(src + (size_t)s * sub_stride);
            }
#pragma unroll
            for (int sub = 0; sub < 10; sub++) {
                const float4* S4 = reinterpret_cast<const float4*>(S_buf + cur * KMAX);
                float2 acc0 = make_float2(0.f, 0.f), acc1 = acc0, acc2 = acc0, acc3 = acc0;
#pragma unroll
                for (int qd = 0; qd < KMAX / 8; qd++) {
                    const float4 s0 = S4[2 * qd], s1 = S4[2 * qd + 1];
                    acc0 = __ffma2_rn(sc[4 * qd + 0], make_float2(s0.x, s0.y), acc0);
                    acc1 = __ffma2_rn(sc[4 * qd + 1], make_float2(s0.z, s0.w), acc1);
                    acc2 = __ffma2_rn(sc[4 * qd + 2], make_float2(s1.x, s1.y), acc2);
                    acc3 = __ffma2_rn(sc[4 * qd + 3], make_float2(s1.z, s1.w), acc3);
                }
                const float coupling = ((acc0.x + acc0.y) + (acc1.x + acc1.y)) + ((acc2.x + acc2.y) + (acc3.x + acc3.y));
                IE = fmaf(GJ, coupling, fmaf(wEE, S_E, C::w_E__I_0)) - wIE * S_I;
                II = fmaf(wEI, S_E, C::w_I__I_0) - S_I;
                rE = rate(fmaf(C::a_E, IE, -C::b_E), C::d_E, 1.0f / C::d_E, -C::d_E * LOG2E);
                rI = rate(fmaf(C::a_I, II, -C::b_I), C::d_I, 1.0f / C::d_I, -C::d_I * LOG2E);
                const float2 n = nz[sub];
                const float dSE = fmaf(n.x, SQ, C::dt * fmaf((1.f - S_E) * C::gamma_E, rE, -S_E * (1.f / C::tau_E)));
                const float dSI = fmaf(n.y, SQ, C::dt * fmaf(C::gamma_I, rI, -S_I * (1.f / C::tau_I)));
                S_E = fminf(fmaxf(S_E + dSE, 0.f), 1.f);
                S_I = fminf(fmaxf(S_I + dSI, 0.f), 1.f);
                if (act) S_buf[(cur ^ 1) * KMAX + j] = S_E;
                __syncthreads();
                cur ^= 1;
            }
            // Balloon-Windkessel once per ms (nu is updated before q uses it,
            // as in bnm.cpp:208-209)
            x = x + C::model_dt * (S_E - C::kappa * x - C::y * (f - 1.f));
            const float tmp_f = f + C::model_dt * x;
            nu = nu + C::model_dt * C::itau * (f - ex2_approx(C::ialpha * lg2_approx(nu)));
            const float inv_nu = rcp_approx(nu);
            const float flow = f * (1.f - ex2_approx(log2_1mrho * rcp_approx(f))) * (1.f / C::rho);
            q = q + C::model_dt * C::itau * (flow - ex2_approx(C::ialpha * lg2_approx(nu)) * q * inv_nu);
            f = tmp_f;
            if (ts % a.TR == 0) {
                if (act) {
                    const float b = C::V_0 * (C::k1 * (1.f - q) + C::k2 * (1.f - q * inv_nu) + C::k3 * (1.f - nu));
                    a.bold[((size_t)sim * a.frames + frame) * N + j] = b;
                    if (frame >= a.n_vols_remove) {
                        ext[0] += S_E;
                        ext[1] += IE;
                        ext[2] += rE;
                        ext[3] += S_I;
                        ext[4] += II;
                        ext[5] += rI;
                    }
                }
                frame++;
            }
            ts++;
            if (adjusting) {
                if (ts >= a.samp_start && ts <= a.samp_end) mean_IE += (double)IE;
                if (ts == a.samp_end) {
                    bool needs = false;
                    if (act) {
                        const double diff = mean_IE / duration - (double)C::b_a_ratio_E;
                        if (fabs(diff + 0.026) > 0.005) {
                            needs = true;
                            if (trial < a.max_trials) {
                                if (diff < -0.026) {
                                    wIE -= delta;
                                    delta = fmaxf(delta - 0.001f, 0.001f);
                                } else {
                                    wIE += delta;
                                }
                            }
                        }
                    }
                    if (__syncthreads_or(needs)) {
                        if (trial < a.max_trials) {
                            S_E = 0.001f;
                            S_I = 0.001f;
                            x = 0.f;
                            f = 1.f;
                            nu = 1.f;
                            q = 1.f;
                            mean_IE = 0.0;
#pragma unroll
                            for (int v = 0; v < 6; v++) ext[v] = 0.0;
                            if (act) S_buf[cur * KMAX + j] = S_E;
                            ts = 0;
                            frame = 0;
                            trial++;
#pragma unroll
                            for (int s = 0; s < 10; s++)
                                nz_next[s] = act ? __ldg(noise2 + (size_t)s * sub_stride + j) : make_float2(0.f, 0.f);
                        } else {
                            failed = true;
                            adjusting = false;
                        }
                    } else {
                        adjusting = false;
                    }
                    __syncthreads();
                }
            }
#pragma unroll
            for (int s = 0; s < 10; s++) nz[s] = nz_next[s];
        }
        if (act) {
            a.wIE_out[(size_t)sim * N + j] = (double)wIE;
            const double kept = (double)(frame - a.n_vols_remove);
#pragma unroll
            for (int v = 0; v < 6; v++) a.ext[((size_t)sim * 6 + v) * N + j] = ext[v] / kept;
        }
        if (threadIdx.x == 0) {
            a.trials[sim] = trial;
            a.failed[sim] = failed ? 1 : 0;
        }
    }
}


template <int KMAX>
static cudaError_t launch_fast(const SimArgs& a, int grid, cudaStream_t st) {
    const int threads = ((a.N + 31) / 32) * 32;
    const size_t smem = (size_t)a.N * KMAX * sizeof(float) + 2 * KMAX * sizeof(float) + 16;
    cudaError_t e = cudaFuncSetAttribute(integrate_fast_kernel<KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    integrate_fast_kernel<KMAX><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace bnm

// Padded row length of the register-resident SC for a node count (0 = the
// fast kernel does not cover it).
extern "C" int bnm_fast_kmax(int N) {
    if (N <= 0 || N > 128) return 0;
    return ((N + 7) / 8) * 8;
}

// FP32 launch: the register-SC kernel when N <= 128, else the reference-order
// kernel in float (SC from shared memory when it fits, else from L2).
cudaError_t bnm_launch_integrate_f32(const bnm::SimArgs& a, int num_sms, cudaStream_t st) {
    using namespace bnm;
    const int kmax = bnm_fast_kmax(a.N);
    if (kmax) {
        const int grid = a.n_sims < 2 * num_sms ? a.n_sims : 2 * num_sms;
        switch (kmax) {
#define BNM_K(K) \
    case K: return launch_fast<K>(a, grid, st);
            BNM_K(8) BNM_K(16) BNM_K(24) BNM_K(32) BNM_K(40) BNM_K(48) BNM_K(56) BNM_K(64) BNM_K(72) BNM_K(80)
            BNM_K(88) BNM_K(96) BNM_K(104) BNM_K(112) BNM_K(120) BNM_K(128)
#undef BNM_K
            default: return cudaErrorInvalidValue;
        }
    }
    const int threads = ((a.N + 31) / 32) * 32;
    if (threads > 1024) return cudaErrorInvalidValue;
    size_t smem = 2 * (size_t)threads * sizeof(float);
    const size_t sc_bytes = (size_t)a.N * a.sc_ld * sizeof(float);
    int sc_in_smem = (smem + sc_bytes) <= 200 * 1024;
    if (sc_in_smem) smem += sc_bytes;
    cudaError_t e = cudaFuncSetAttribute(fastgen::integrate_generic_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = a.n_sims < 2 * num_sms ? a.n_sims : 2 * num_sms;
    fastgen::integrate_generic_kernel<float><<<grid, threads, smem, st>>>(a, sc_in_smem);
    return cudaGetLastError();
}
