// FP32 model pieces shared by the register integrator (N <= 128) and the
// cluster integrator (N > 128): firing rate, Balloon-Windkessel in deviation
// variables, shared-memory addressing and a bounded mbarrier wait.
#pragma once
#include "kernels.h"

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

// r = x / (1 - exp(-d x)) from x and e = exp(-d x) (the caller forms e, so
// that the exponent's argument need not wait for x); for |d x| < 0.1 the
// quotient is evaluated as (1/d) / P(u) with P(u) = (1 - e^-u)/u truncated
// after u^4 (rel. err < 2e-8).
__device__ __forceinline__ float rate_from(float x, float e, float d, float inv_d) {
    const float u = d * x;
    float p = fmaf(u, 1.0f / 120.0f, -1.0f / 24.0f);
    p = fmaf(p, u, 1.0f / 6.0f);
    p = fmaf(p, u, -0.5f);
    p = fmaf(p, u, 1.0f);
    const bool small = fabsf(u) < 0.1f;
    const float num = small ? inv_d : x;
    const float den = small ? p : (1.0f - e);
    return num * rcp_approx(den);
}

__device__ __forceinline__ float rate(float x, float d, float inv_d, float neg_d_log2e) {
    return rate_from(x, ex2_approx(x * neg_d_log2e), d, inv_d);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Wall-clock limit of every bounded wait in the integrators: a copy or an
// exchange normally lands within microseconds.
constexpr long long kWaitNs = 1000000000ll;  // 1 s

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait on an mbarrier phase for at most limit_ns nanoseconds of wall time
// (%globaltimer, read every 16 unsuccessful polls; try_wait itself may suspend
// the thread for a hardware-defined interval, so the bound is on time, not on
// polls).  Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit_ns) {
    unsigned long long t0 = 0;
    for (uint32_t i = 0;; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 15) == 0) {
            const unsigned long long t = global_ns();
            if (i == 0)
                t0 = t;
            else if ((long long)(t - t0) > limit_ns)
                return false;
        }
    }
}

// e^y - 1 for the Balloon-Windkessel step.  Near zero, where e^y - 1 cancels,
// the Taylor series y (1 + y/2 + y^2/6 + y^3/24 + y^4/120) (|y| < 1/16:
// truncation below 2e-9 relative); elsewhere the identity e^y = 2^(y log2 e)
// with the hardware base-2 exponential (ex2.approx), whose relative error the
// subtraction of 1 magnifies at most e^y / (e^y - 1) < 17 times.  Both are
// evaluated and one selected (no branch).  Measured against expm1f over the
// step's argument range by tests/test_bw_math.py.
__device__ __forceinline__ float expm1_bw(float y) {
    float t = fmaf(y, 1.0f / 120.0f, 1.0f / 24.0f);
    t = fmaf(t, y, 1.0f / 6.0f);
    t = fmaf(t, y, 0.5f);
    t = fmaf(t, y, 1.0f);
    const float near0 = t * y;
    const float far = ex2_approx(y * 1.4426950408889634f) - 1.0f;
    return fabsf(y) < 0.0625f ? near0 : far;
}
// ln(1 + x) for the Balloon-Windkessel step: the Mercator series
// x - x^2/2 + ... + x^7/7 for |x| < 1/16 (truncation below 1e-9 relative),
// else ln(1 + x) = log2(1 + x) ln 2 with the hardware base-2 logarithm
// (lg2.approx); selected without a branch.  Measured against log1pf by
// tests/test_bw_math.py.
__device__ __forceinline__ float log1p_bw(float x) {
    float t = fmaf(x, 1.0f / 7.0f, -1.0f / 6.0f);
    t = fmaf(t, x, 1.0f / 5.0f);
    t = fmaf(t, x, -0.25f);
    t = fmaf(t, x, 1.0f / 3.0f);
    t = fmaf(t, x, -0.5f);
    t = fmaf(t, x, 1.0f);
    const float near0 = t * x;
    float l2;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"(1.0f + x));
    const float far = l2 * 0.6931471805599453f;
    return fabsf(x) < 0.0625f ? near0 : far;
}

// Balloon-Windkessel in deviation variables ft = f-1, nt = nu-1, qt = q-1
// (log1p / expm1 through log1p_bw / expm1_bw).
struct BW {
    float x = 0.f, ft = 0.f, nt = 0.f, qt = 0.f, lnu = 0.f;  // lnu = log(nu) = log1p(nt)
    __device__ __forceinline__ void step(float S_E) {
        typedef Model<float> C;
        const float L1mr = -0.41551544396166582f;  // ln(1 - rho)
        const float a1 = C::ialpha - 1.0f;         // exponent of nu in nu^(1/alpha) q / nu
        x = x + C::model_dt * (S_E - C::kappa * x - C::y * ft);
        const float ft_new = ft + C::model_dt * x;
        const float pw = expm1_bw(C::ialpha * lnu);  // nu^(1/alpha) - 1, old nu
        const float nt_new = nt + C::model_dt * C::itau * (ft - pw);
        // f (1 - (1-rho)^(1/f)) / rho - 1, without cancellation:
        // 1 - (1-rho)^(1/f) - rho = -(1-rho) expm1(ln(1-rho) (1/f - 1))
        const float h = -(1.0f - C::rho) * expm1_bw(-L1mr * __fdividef(ft, 1.0f + ft));
        const float inflow = (h + ft * (C::rho + h)) * (1.0f / C::rho);
        // nu^(1/alpha - 1) q - 1 with the updated nu
        const float lnu_new = log1p_bw(nt_new);
        const float e = expm1_bw(a1 * lnu_new);
        const float outflow = e + qt * (1.0f + e);
        qt = qt + C::model_dt * C::itau * (inflow - outflow);
        nt = nt_new;
        lnu = lnu_new;
        ft = ft_new;
    }
    __device__ __forceinline__ float bold() const {
        typedef Model<float> C;
        // V0 (k1 (1-q) + k2 (1 - q/nu) + k3 (1-nu))
        return C::V_0 * (-C::k1 * qt + C::k2 * (nt - qt) / (1.0f + nt) - C::k3 * nt);
    }
};

}  // namespace bnm
