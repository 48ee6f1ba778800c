// FP32 integrator for N <= 128: structural connectivity held in registers.
//
// Same model and time loop as the reference's bnm kernel (bnm.cu:72-315) and
// CPU path (bnm.cpp:167-290), re-laid out for Blackwell:
//   * one CTA per particle (persistent over particles, two CTAs per SM); warp
//     w owns nodes 32w..32w+31.  The coupling G*J*(SC.S_E) is a register-
//     blocked mat-vec: lane l = 4u+v of warp w keeps the 4 x K block
//     SC[32w+4u .. 32w+4u+3][Kv .. Kv+K-1] in registers for the whole run,
//     reads only its K entries of S_E (broadcast LDS.128), and the four lanes
//     of a row group finish with a 3-shuffle reduce-scatter after which lane l
//     holds the full sum of node 32w+l.  Shared-memory traffic per substep is
//     K floats per lane instead of N;
//   * SC is staged once into shared memory by a TMA bulk copy (cp.async.bulk
//     + mbarrier, no multicast, bounded wait) before being read into registers;
//   * the row dot products use packed FP32 FMA (fma.rn.f32x2) over column
//     pairs, two accumulators per row;
//   * S_E is double buffered in shared memory: one barrier per substep;
//   * the next millisecond's noise is prefetched into registers;
//   * firing rates use ex2.approx / rcp.approx with an exact-limit series for
//     |d(aI-b)| < 0.1, where 1-exp(-u) cancels (the reference FP32 build
//     clamps |aI-b| to 1e-4 instead, bnm.cu:195-199);
//   * the Balloon-Windkessel state is integrated as deviations from rest
//     (f-1, nu-1, q-1, with log1p / expm1), so FP32 keeps full relative
//     precision in the small BOLD fluctuations; the update order is the
//     reference's (x, then f from the new x, nu from the old f, q from the old
//     f and the new nu, bnm.cpp:204-211);
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

// Balloon-Windkessel in deviation variables ft = f-1, nt = nu-1, qt = q-1.
struct BW {
    float x = 0.f, ft = 0.f, nt = 0.f, qt = 0.f;
    __device__ __forceinline__ void step(float S_E) {
        typedef Model<float> C;
        const float L1mr = -0.41551544396166582f;  // ln(1 - rho)
        const float a1 = C::ialpha - 1.0f;         // exponent of nu in nu^(1/alpha) q / nu
        x = x + C::model_dt * (S_E - C::kappa * x - C::y * ft);
        const float ft_new = ft + C::model_dt * x;
        const float pw = expm1f(C::ialpha * log1pf(nt));  // nu^(1/alpha) - 1, old nu
        const float f_old = 1.0f + ft;
        const float nt_new = nt + C::model_dt * C::itau * (ft - pw);
        // f (1 - (1-rho)^(1/f)) / rho - 1, without cancellation:
        // 1 - (1-rho)^(1/f) - rho = -(1-rho) expm1(ln(1-rho) (1/f - 1))
        const float h = -(1.0f - C::rho) * expm1f(-L1mr * ft / f_old);
        const float inflow = (h + ft * (C::rho + h)) * (1.0f / C::rho);
        // nu^(1/alpha - 1) q - 1 with the updated nu
        const float e = expm1f(a1 * log1pf(nt_new));
        const float outflow = e + qt * (1.0f + e);
        qt = qt + C::model_dt * C::itau * (inflow - outflow);
        nt = nt_new;
        ft = ft_new;
    }
    __device__ __forceinline__ float bold() const {
        typedef Model<float> C;
        // V0 (k1 (1-q) + k2 (1 - q/nu) + k3 (1-nu))
        return C::V_0 * (-C::k1 * qt + C::k2 * (nt - qt) / (1.0f + nt) - C::k3 * nt);
    }
};

template <int K>
__global__ void __launch_bounds__(128, 2) integrate_fast_kernel(SimArgs a) {
    static_assert(K % 4 == 0 && K <= 32, "K");
    constexpr int LD = 4 * K;  // padded SC row length and S_E buffer length
    typedef Model<float> C;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // layout: [SC stage: N*LD floats][S: 2*LD floats][mbarrier]
    const int N = a.N;
    float* sc_stage = reinterpret_cast<float*>(smem_raw);
    float* S_buf = sc_stage + (size_t)N * LD;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(S_buf + 2 * LD);
    __shared__ int s_sim;

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int u = lane >> 2, v = lane & 3;
    const int j = threadIdx.x;  // node owned after the reduce-scatter (32w + lane)
    const bool act = j < N;

    // ---- stage SC into shared memory with one TMA bulk copy --------------
    const uint32_t bar = smem_addr(mbar);
    const uint32_t bytes = (uint32_t)(N * LD * sizeof(float));
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
        mbar_wait(bar, 0, 1ll << 26);  // let a late copy land before the CTA exits
        return;
    }
    // this lane's 4 x K block of SC, as column pairs
    float2 sc[4][K / 2];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int row = 32 * w + 4 * u + r;
#pragma unroll
        for (int c = 0; c < K / 2; c++)
            sc[r][c] = row < N ? reinterpret_cast<const float2*>(sc_stage + (size_t)row * LD + v * K)[c]
                               : make_float2(0.f, 0.f);
    }

    const float2* noise2 = reinterpret_cast<const float2*>(a.noise);
    const size_t sub_stride = (size_t)N;  // float2 entries per substep
    const double duration = (double)(a.samp_end - a.samp_start + 1);
    const float SQ = C::sigma_model * C::sqrt_dt;
    const float LOG2E = 1.4426950408889634f;

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
        float S_E = 0.001f, S_I = 0.001f;
        BW bw;
        float IE = 0.f, II = 0.f, rE = 0.f, rI = 0.f;
        double mean_IE = 0.0;
        double ext[6] = {0, 0, 0, 0, 0, 0};
        for (int k = threadIdx.x; k < 2 * LD; k += blockDim.x) S_buf[k] = ((k % LD) < N) ? S_E : 0.f;
        int cur = 0, trial = 0, ts = 0, frame = 0;
        bool failed = false, adjusting = a.adjust_fic != 0;

        float2 nz[10], nz_next[10];
#pragma unroll
        for (int s = 0; s < 10; s++) nz[s] = act ? __ldg(noise2 + (size_t)s * sub_stride + j) : make_float2(0.f, 0.f);
        __syncthreads();

        while (ts <= a.T) {
            if (act && ts < a.T) {  // prefetch the next millisecond's noise
                const float2* src = noise2 + ((size_t)(ts + 1) * 10) * sub_stride + j;
#pragma unroll
                for (int s = 0; s < 10; s++) nz_next[s] = __ldg(src + (size_t)s * sub_stride);
            }
#pragma unroll
            for (int sub = 0; sub < 10; sub++) {
                const float4* S4 = reinterpret_cast<const float4*>(S_buf + cur * LD + v * K);
                float2 acc[4][2];
#pragma unroll
                for (int r = 0; r < 4; r++) acc[r][0] = acc[r][1] = make_float2(0.f, 0.f);
#pragma unroll
                for (int c4 = 0; c4 < K / 4; c4++) {
                    const float4 s = S4[c4];
                    const float2 s01 = make_float2(s.x, s.y), s23 = make_float2(s.z, s.w);
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        acc[r][0] = __ffma2_rn(sc[r][2 * c4], s01, acc[r][0]);
                        acc[r][1] = __ffma2_rn(sc[r][2 * c4 + 1], s23, acc[r][1]);
                    }
                }
                float p[4];
#pragma unroll
                for (int r = 0; r < 4; r++) p[r] = (acc[r][0].x + acc[r][0].y) + (acc[r][1].x + acc[r][1].y);
                // reduce-scatter over the 4 lanes of this row group: lane v gets row 4u+v
                const bool hi = (v >> 1) & 1, lo = v & 1;
                const float k0 = hi ? p[2] : p[0], k1 = hi ? p[3] : p[1];
                const float s0 = hi ? p[0] : p[2], s1 = hi ? p[1] : p[3];
                const float q0 = k0 + __shfl_xor_sync(0xffffffffu, s0, 2);
                const float q1 = k1 + __shfl_xor_sync(0xffffffffu, s1, 2);
                const float kk = lo ? q1 : q0, ss = lo ? q0 : q1;
                const float coupling = kk + __shfl_xor_sync(0xffffffffu, ss, 1);

                IE = fmaf(GJ, coupling, fmaf(wEE, S_E, C::w_E__I_0)) - wIE * S_I;
                II = fmaf(wEI, S_E, C::w_I__I_0) - S_I;
                rE = rate(fmaf(C::a_E, IE, -C::b_E), C::d_E, 1.0f / C::d_E, -C::d_E * LOG2E);
                rI = rate(fmaf(C::a_I, II, -C::b_I), C::d_I, 1.0f / C::d_I, -C::d_I * LOG2E);
                const float2 n = nz[sub];
                const float dSE = fmaf(n.x, SQ, C::dt * fmaf((1.f - S_E) * C::gamma_E, rE, -S_E * (1.f / C::tau_E)));
                const float dSI = fmaf(n.y, SQ, C::dt * fmaf(C::gamma_I, rI, -S_I * (1.f / C::tau_I)));
                S_E = fminf(fmaxf(S_E + dSE, 0.f), 1.f);
                S_I = fminf(fmaxf(S_I + dSI, 0.f), 1.f);
                if (act) S_buf[(cur ^ 1) * LD + j] = S_E;
                __syncthreads();
                cur ^= 1;
            }
            bw.step(S_E);
            if (ts % a.TR == 0) {
                if (act) {
                    a.bold[((size_t)sim * a.frames + frame) * N + j] = bw.bold();
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
                            bw = BW();
                            mean_IE = 0.0;
#pragma unroll
                            for (int q = 0; q < 6; q++) ext[q] = 0.0;
                            if (act) S_buf[cur * LD + j] = S_E;
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
            for (int q = 0; q < 6; q++) a.ext[((size_t)sim * 6 + q) * N + j] = ext[q] / kept;
        }
        if (threadIdx.x == 0) {
            a.trials[sim] = trial;
            a.failed[sim] = failed ? 1 : 0;
        }
    }
}

template <int K>
static cudaError_t launch_fast(const SimArgs& a, int grid, cudaStream_t st) {
    const int threads = ((a.N + 31) / 32) * 32;
    const size_t smem = (size_t)a.N * 4 * K * sizeof(float) + 2 * 4 * K * sizeof(float) + 16;
    cudaError_t e =
        cudaFuncSetAttribute(integrate_fast_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    integrate_fast_kernel<K><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace bnm

// Padded SC row length (4K) of the register kernel for a node count (0 = the
// register kernel does not cover it).
extern "C" int bnm_fast_kmax(int N) {
    if (N <= 0 || N > 128) return 0;
    const int K = ((N + 3) / 4 + 3) / 4 * 4;
    return 4 * K;
}

// FP32 launch: the register-SC kernel when N <= 128, else the reference-order
// kernel in float (SC from shared memory when it fits, else from L2).
cudaError_t bnm_launch_integrate_f32(const bnm::SimArgs& a, int num_sms, cudaStream_t st) {
    using namespace bnm;
    const int ld = bnm_fast_kmax(a.N);
    if (ld) {
        if (a.sc_ld != ld) return cudaErrorInvalidValue;
        const int grid = a.n_sims < 2 * num_sms ? a.n_sims : 2 * num_sms;
        switch (ld / 4) {
#define BNM_K(K) \
    case K: return launch_fast<K>(a, grid, st);
            BNM_K(4) BNM_K(8) BNM_K(12) BNM_K(16) BNM_K(20) BNM_K(24) BNM_K(28) BNM_K(32)
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
    cudaError_t e = cudaFuncSetAttribute(fastgen::integrate_generic_kernel<float>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = a.n_sims < 2 * num_sms ? a.n_sims : 2 * num_sms;
    fastgen::integrate_generic_kernel<float><<<grid, threads, smem, st>>>(a, sc_in_smem);
    return cudaGetLastError();
}
