// Counter-based noise source (BNM_NOISE_PHILOX): Philox4x32-10 (Salmon,
// Moraes, Dror, Shaw, SC'11) with a Box-Muller transform.
//
// The reference draws one stream of standard normals per run, in the order
// (millisecond, substep, node, E then I), and every particle and every FIC
// trial reads the same stream from its start (run_CMAES.cpp:640-657,
// bnm.cu:202-205).  Here the element for (ms, substep, node, E|I) is a pure
// function of the seed and those indices, so a kernel can draw it where it is
// consumed instead of reading a table: one Philox call with counter
// (ms * 5 + substep / 2) * N + node and key = seed yields the E and I values
// of that node for the substep pair (2k, 2k + 1).  The table filled by
// philox_fill_kernel holds exactly these values in the reference's array
// order, for the kernels that read a table.
#pragma once
#include <cstdint>

namespace bnm {

__device__ __forceinline__ void philox_round(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0;
    c[1] = n1;
    c[2] = n2;
    c[3] = n3;
}

__device__ __forceinline__ void philox4x32_10(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        philox_round(c, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Box-Muller on two 32-bit words: radius sqrt(-2 ln u0) with u0 in (0, 1]
// from the base-2 logarithm, angle 2 pi (u1 - 1/2) in [-pi, pi) where the
// hardware sine and cosine are accurate to about 1e-6 absolute.
__device__ __forceinline__ float2 box_muller(uint32_t a, uint32_t b) {
    const float s = 2.3283064365386963e-10f;  // 2^-32
    const float u0 = fmaf((float)a, s, s);     // (a + 1) 2^-32, in (0, 1]
    const float v = fmaf((float)b, s, -0.5f);  // in [-1/2, 1/2)
    float l2, r, sn, cs;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"(fminf(u0, 1.0f)));
    const float t = -1.3862943611198906f * l2;  // -2 ln 2 log2(u0) = -2 ln u0 >= 0
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(t));
    const float th = 6.283185307179586f * v;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(sn) : "f"(th));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(cs) : "f"(th));
    return make_float2(r * cs, r * sn);
}

// Noise of `node` for the substep pair (2 pair, 2 pair + 1) of millisecond
// `ms`: (E, I) of the first substep in .x, .y and of the second in .z, .w.
__device__ __forceinline__ float4 philox_noise_pair(uint32_t key0, uint32_t key1, int ms, int pair, int node, int N) {
    const uint64_t ctr = ((uint64_t)ms * 5 + (uint64_t)pair) * (uint64_t)N + (uint64_t)node;
    uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u};
    philox4x32_10(c, key0, key1);
    const float2 g0 = box_muller(c[0], c[1]), g1 = box_muller(c[2], c[3]);
    return make_float4(g0.x, g0.y, g1.x, g1.y);
}

// One millisecond of noise for the nodes [r0, r0 + n_own) of a CTA, drawn by
// the whole block into a ring stage laid out [substep][R] (float2 E, I); the
// nodes at or above n_real (a padding node) get zeros.  The caller orders
// the writes before the reads with a block barrier.
__device__ __forceinline__ void philox_fill_stage(float2* stage, int R, int r0, int n_own, int n_real, int ms,
                                                  uint32_t key0, uint32_t key1) {
    for (int k = threadIdx.x; k < 5 * n_own; k += blockDim.x) {
        const int pair = k / n_own, i = k - pair * n_own, node = r0 + i;
        const float4 v = node < n_real ? philox_noise_pair(key0, key1, ms, pair, node, n_real)
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
        stage[(2 * pair) * R + i] = make_float2(v.x, v.y);
        stage[(2 * pair + 1) * R + i] = make_float2(v.z, v.w);
    }
}

}  // namespace bnm
