// Reference-order integrator (any N up to 1024, float or double).
//
// One CTA integrates one particle at a time (persistent: CTAs pull particle
// indices from a global counter), one thread per node.  It restates the
// reference's time loop (bnm.cpp:167-290; the same model as bnm.cu:72-315)
// with the reference's operand order and operand types, and it is compiled
// with -fmad=false in integrate_exact.cu, so that in double it reproduces the
// reference's FP64 CPU arithmetic up to the last-ulp differences of the
// device exp/pow, and in float the reference's USE_FLOATS arithmetic.  It is
// the parity path (oracle-noise mode, step-for-step checks) and the fallback
// for node counts the register-resident fast kernel does not cover.
//
// Semantics that follow the reference's CPU path rather than its GPU path
// (bnm.cu differs in these places):
//   * numerical FIC: delta is rounded through fmaxf (bnm.cpp:250) and the
//     per-node extended sums restart with the simulation after an FIC trial
//     (the CPU keeps only the final time series, bnm.cpp:212-226);
//   * no FP32 clamp of |aI-b| < 1e-4 (bnm.cu:195-199 only).
#pragma once
#include "bnm_common.cuh"

// Each translation unit that includes this header instantiates its own copy
// (integrate_exact.cu with -fmad=false, integrate_fast.cu with contraction),
// so the kernels live in a per-TU namespace.
#ifndef BNM_GENERIC_NS
#error "define BNM_GENERIC_NS before including integrate_generic.cuh"
#endif

namespace bnm {
namespace BNM_GENERIC_NS {

__device__ __forceinline__ float dexp(float x) { return expf(x); }
__device__ __forceinline__ double dexp(double x) { return exp(x); }
__device__ __forceinline__ float dpow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double dpow(double a, double b) { return pow(a, b); }

template <typename R>
__device__ __forceinline__ const R* sc_ptr(const SimArgs& a);
template <>
__device__ __forceinline__ const float* sc_ptr<float>(const SimArgs& a) { return a.sc_f32; }
template <>
__device__ __forceinline__ const double* sc_ptr<double>(const SimArgs& a) { return a.sc_f64; }

template <typename R>
__device__ __forceinline__ void store_bold(const SimArgs& a, size_t idx, R v);
template <>
__device__ __forceinline__ void store_bold<float>(const SimArgs& a, size_t idx, float v) { a.bold[idx] = v; }
template <>
__device__ __forceinline__ void store_bold<double>(const SimArgs& a, size_t idx, double v) { a.bold_f64[idx] = v; }

// Dynamic shared memory: S[2][npad] (+ SC[N][ld] when sc_in_smem).
template <typename R>
__global__ void integrate_generic_kernel(SimArgs a, int sc_in_smem) {
    typedef Model<R> C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = a.N, npad = blockDim.x;
    const int ld = (sizeof(R) == 4) ? a.sc_ld : N;
    R* S_buf = reinterpret_cast<R*>(smem_raw);
    const R* SC = sc_ptr<R>(a);
    if (sc_in_smem) {
        R* sc_s = S_buf + 2 * npad;
        for (int i = threadIdx.x; i < N * ld; i += blockDim.x) sc_s[i] = SC[i];
        SC = sc_s;
    }
    __shared__ int s_sim;
    const int j = threadIdx.x;
    const bool act = j < N;
    const R* sc_row = SC + (size_t)(act ? j : 0) * ld;
    const unsigned int duration = a.samp_end - a.samp_start + 1;
    const size_t plane = (size_t)a.noise_ld;  // node stride of the noise table

    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_sim = atomicAdd(a.work_counter, 1);
        __syncthreads();
        const int sim = s_sim;
        if (sim >= a.n_sims) break;

        const R G = (R)a.G[sim];
        const R wEE = act ? (R)a.wEE[(size_t)sim * N + j] : (R)0;
        const R wEI = act ? (R)a.wEI[(size_t)sim * N + j] : (R)0;
        R wIE = act ? (R)a.wIE[(size_t)sim * N + j] : (R)0;
        R S_E = 0.001, S_I = 0.001, x = 0.0, f = 1.0, nu = 1.0, q = 1.0;
        R IE = 0, II = 0, rE = 0, rI = 0, mean_IE = 0, delta = (R)a.init_delta;
        R ext[6] = {0, 0, 0, 0, 0, 0};
        S_buf[j] = act ? S_E : (R)0;
        S_buf[npad + j] = (R)0;
        int cur = 0, trial = 0, ts = 0, frame = 0;
        bool failed = false, adjusting = a.adjust_fic != 0;
        __syncthreads();

        while (ts <= a.T) {
            for (int sub = 0; sub < 10; sub++) {
                const R* Sp = S_buf + cur * npad;
                R coupling = 0;
                for (int k = 0; k < N; k++) coupling += sc_row[k] * Sp[k];
                if (act) {
                    IE = C::w_E__I_0 + wEE * S_E + coupling * G * C::J_NMDA - wIE * S_I;
                    II = C::w_I__I_0 + wEI * S_E - S_I;
                    R eE = dexp(-C::d_E * (C::a_E * IE - C::b_E));
                    R eI = dexp(-C::d_I * (C::a_I * II - C::b_I));
                    rE = (C::a_E * IE - C::b_E) / (1 - eE);
                    rI = (C::a_I * II - C::b_I) / (1 - eI);
                    const size_t nidx = (((size_t)ts * 10 + sub) * plane + j) * 2;
                    R nE = (R)a.noise[nidx];
                    R nI = (R)a.noise[nidx + 1];
                    R dSE = nE * C::sigma_model * C::sqrt_dt +
                            C::dt * ((1 - S_E) * C::gamma_E * rE - (S_E / C::tau_E));
                    R dSI = nI * C::sigma_model * C::sqrt_dt + C::dt * (C::gamma_I * rI - (S_I / C::tau_I));
                    S_E += dSE;
                    S_I += dSI;
                    // std::max(0, std::min(S, 1)) of bnm.cpp:195-199, NaN -> 0 included
                    S_E = ((R)1.0 < S_E) ? (R)1.0 : S_E;
                    S_E = ((R)0.0 < S_E) ? S_E : (R)0.0;
                    S_I = ((R)1.0 < S_I) ? (R)1.0 : S_I;
                    S_I = ((R)0.0 < S_I) ? S_I : (R)0.0;
                    S_buf[(cur ^ 1) * npad + j] = S_E;
                }
                __syncthreads();
                cur ^= 1;
            }
            if (act) {
                // Balloon-Windkessel once per ms (bnm.cpp:204-211); the double
                // literals promote exactly as in the reference.
                x = x + C::model_dt * (S_E - C::kappa * x - C::y * (f - 1.0));
                R tmp_f = f + C::model_dt * x;
                nu = nu + C::model_dt * C::itau * (f - dpow(nu, C::ialpha));
                q = q + C::model_dt * C::itau *
                            (f * (1.0 - dpow(C::oneminrho, (R)(1.0 / f))) / C::rho - dpow(nu, C::ialpha) * q / nu);
                f = tmp_f;
            }
            if (ts % a.TR == 0) {
                if (act) {
                    R b = C::V_0 * (C::k1 * (1 - q) + C::k2 * (1 - q / nu) + C::k3 * (1 - nu));
                    store_bold<R>(a, ((size_t)sim * a.frames + frame) * N + j, b);
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
                if (ts >= a.samp_start && ts <= a.samp_end) mean_IE += IE;
                if (ts == a.samp_end) {
                    bool needs = false;
                    if (act) {
                        mean_IE /= duration;
                        R diff = mean_IE - C::b_a_ratio_E;
                        if (fabs(diff + 0.026) > 0.005) {
                            needs = true;
                            if (trial < a.max_trials) {
                                if (diff < -0.026) {
                                    wIE -= delta;
                                    delta -= 0.001;
                                    delta = fmaxf(delta, 0.001);
                                } else {
                                    wIE += delta;
                                }
                            }
                        }
                    }
                    if (__syncthreads_or(needs)) {
                        if (trial < a.max_trials) {
                            S_E = 0.001;
                            S_I = 0.001;
                            x = 0.0;
                            f = 1.0;
                            nu = 1.0;
                            q = 1.0;
                            mean_IE = 0;
                            for (int v = 0; v < 6; v++) ext[v] = 0;
                            if (act) S_buf[cur * npad + j] = S_E;
                            ts = 0;
                            frame = 0;
                            trial++;
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
        }
        if (act) {
            a.wIE_out[(size_t)sim * N + j] = (double)wIE;
            const int kept = frame - a.n_vols_remove;
            for (int v = 0; v < 6; v++) {
                R m = ext[v];
                m /= kept;
                a.ext[((size_t)sim * 6 + v) * N + j] = (double)m;
            }
        }
        if (threadIdx.x == 0) {
            a.trials[sim] = trial;
            a.failed[sim] = failed ? 1 : 0;
        }
    }
}

}  // namespace BNM_GENERIC_NS
}  // namespace bnm
