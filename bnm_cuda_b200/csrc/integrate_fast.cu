// FP32 integrator for N <= 128: structural connectivity held in registers.
//
// Same model and time loop as the reference's bnm kernel (bnm.cu:72-315) and
// CPU path (bnm.cpp:167-290), re-laid out for Blackwell:
//   * one CTA per particle (persistent over particles, two CTAs per SM); warp
//     w owns nodes 32w..32w+31.  The coupling G*J*(SC.S_E) is a register-
//     blocked mat-vec: lane l = 4u+v of warp w keeps the 4 x KC block
//     SC[32w+4u .. 32w+4u+3][KC v .. KC v+KC-1] in registers for the whole
//     run (KC = ceil(N/4) rounded up to even: 26 at N = 100), reads only its
//     KC entries of S_E (broadcast LDS.128 from a buffer that keeps each
//     quarter at a stride of K = KC rounded up to 4 floats), and the four lanes
//     of a row group finish with a select-free reduce-scatter of three
//     independent shuffles (rows stored in xor-permuted slots) after which
//     lane l holds the full sum of node 32w+l.  Shared-memory traffic per substep is
//     KC floats per lane instead of N;
//   * SC is staged once into shared memory by a TMA bulk copy (cp.async.bulk
//     + mbarrier, no multicast, bounded wait) before being read into registers;
//   * the row dot products use packed FP32 FMA (fma.rn.f32x2) over column
//     pairs, two accumulators per row;
//   * S_E is double buffered in shared memory: one barrier per substep;
//   * noise arrives one simulated millisecond at a time (10 substeps x N x
//     (E, I), contiguous in the table) by TMA bulk copies into a 4-stage
//     shared-memory ring, issued three milliseconds ahead by one thread and
//     tracked with mbarriers; an FIC restart drains the copies in flight and
//     refetches from millisecond 0;
//   * firing rates use ex2.approx / rcp.approx with an exact-limit series for
//     |d(aI-b)| < 0.1, where 1-exp(-u) cancels (the reference FP32 build
//     clamps |aI-b| to 1e-4 instead, bnm.cu:195-199);
//   * the Balloon-Windkessel state is integrated as deviations from rest
//     (f-1, nu-1, q-1, with log1p / expm1), so FP32 keeps full relative
//     precision in the small BOLD fluctuations; the update order is the
//     reference's (x, then f from the new x, nu from the old f, q from the old
//     f and the new nu, bnm.cpp:204-211);
//   * FIC sampling and the extended-output sums accumulate in FP64.
#include <cstdlib>
#include "kernels.h"
#include "fp32_model.cuh"
#include "noise.cuh"
#ifndef BNM_FAST_CHAIN
#define BNM_FAST_CHAIN 1  // the folded substep chain below (0: the plain form, kept for comparison)
#endif
#define BNM_GENERIC_NS fastgen
#include "integrate_generic.cuh"

namespace bnm {

// Noise ring: the 10 substeps x N nodes x (E, I) floats of one simulated
// millisecond are contiguous in the table (80 N bytes), so one thread brings a
// whole millisecond into shared memory with one TMA bulk copy.  kStages
// copies are in flight ahead of the consumer; copy c lives in stage c % kStages
// and completes phase (c / kStages) & 1 of that stage's mbarrier.
constexpr int kStages = 4;

// Per-particle ("slot") state that every thread keeps for its node.
struct Slot {
    float GJ, GJa, GJe, wEE, wEI, wIE, delta, S_E, S_I, IE, II, rE, rI;
    double mean_IE;
    BW bw;
};

// One CTA integrates P particles at a time (P slots) with the same warps:
// the SC block in registers serves every slot, so the slots' independent
// dependency chains interleave inside each warp (instruction-level
// parallelism instead of a second CTA on the SM).  Slots advance one
// simulated millisecond per iteration in lockstep but keep their own time,
// FIC trial and noise stream; a slot whose particle ends takes the next one
// from the batch's work counter.
//
// NZI: the noise is drawn in the kernel (Philox, noise.cuh: one call per node
// and substep pair gives the E and I values of both substeps) instead of
// being streamed from the table through the TMA ring; the values are the
// table's, so both give the same results.
template <int K, int KC, int P, bool NZI, bool PL = false>
__global__ void __launch_bounds__(128, 1) integrate_fast_kernel(SimArgs a) {
    static_assert(K % 4 == 0 && K <= 32, "K");
    static_assert(!PL || (P == 1 && !NZI), "placement: one particle per CTA, table noise");
    static_assert(KC % 2 == 0 && KC <= K && KC + 2 >= K, "KC");
    static_assert(P >= 1 && P <= 2, "P");
    constexpr int LD = 4 * K;  // padded SC row length and S_E buffer length (quarter v at K v)
    typedef Model<float> C;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // layout: [noise rings: P * kStages * 10*N float2][SC stage: N*LD floats]
    //         [S: P * 2*LD floats][extended sums: P*6*blockDim doubles][mbarriers: 1 + P*kStages]
    const int N = a.N;
    const uint32_t ms_bytes = (uint32_t)(10 * N * sizeof(float2));
    float2* ring = reinterpret_cast<float2*>(smem_raw);
    float* sc_stage = reinterpret_cast<float*>(smem_raw + (NZI ? 0 : (size_t)P * kStages * ms_bytes));
    float* S_buf = sc_stage + (size_t)N * LD;
    double* ext = reinterpret_cast<double*>(S_buf + P * 2 * LD);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(ext + (size_t)P * 6 * blockDim.x);
    __shared__ int s_sim[P], s_flag;

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int u = lane >> 2, v = lane & 3;
    const int j = threadIdx.x;  // node owned after the reduce-scatter (32w + lane)
    const bool act = j < N;
    const int pos_j = K * (j / KC) + j % KC;  // S_E buffer slot of node j
    const long long kSpin = kWaitNs;  // wall-clock limit of each bounded wait

    // ---- barriers; stage SC into shared memory with one TMA bulk copy ----
    if (threadIdx.x == 0) {
        for (int b = 0; b <= P * kStages; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar + b)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t sc_bytes = (uint32_t)(N * LD * sizeof(float));
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(sc_bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(sc_stage)),
            "l"(a.sc_f32), "r"(sc_bytes), "r"(smem_addr(mbar))
            : "memory");
    }
    if (__syncthreads_or(!mbar_wait(smem_addr(mbar), 0, kSpin))) {
        if (threadIdx.x == 0) atomicOr(a.status, kStatusTimeout);
        mbar_wait(smem_addr(mbar), 0, kSpin);  // let a late copy land before the CTA exits
        return;
    }
    // This lane's 4 x KC block of SC as column pairs.  Slot r of a lane holds
    // row 4u + (v ^ r), so the reduce-scatter below needs no selects: lane v
    // adds its slot 0 and slot m of lane v ^ m (m = 1, 2, 3), all of them row
    // 4u + v.
    float2 sc[4][KC / 2];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int row = 32 * w + 4 * u + (v ^ r);
#pragma unroll
        for (int c = 0; c < KC / 2; c++)
            sc[r][c] = row < N ? reinterpret_cast<const float2*>(sc_stage + (size_t)row * LD + v * KC)[c]
                               : make_float2(0.f, 0.f);
    }

    const char* noise_bytes = reinterpret_cast<const char*>(a.noise);
    const uint32_t key0 = (uint32_t)a.noise_seed, key1 = (uint32_t)(a.noise_seed >> 32);
    const double duration = (double)(a.samp_end - a.samp_start + 1);
    const float SQ = C::sigma_model * C::sqrt_dt;
    const float LOG2E = 1.4426950408889634f;
    const float kDtGammaE = C::dt * C::gamma_E, kDtInvTauE = C::dt / C::tau_E;
    const float kDtGammaI = C::dt * C::gamma_I, kDtInvTauI = C::dt / C::tau_I;

    // per-slot control (uniform over the CTA); thread 0 also owns the copy issue state
    int sim[P], ts[P], frame[P], to_frame[P], trial[P], ms_next[P];
    bool failed[P], adjusting[P], live[P];
    uint32_t c_cons[P], c_issue[P];
    Slot sl[P];
    bool timed_out = false;

    auto wait_copy = [&](int p, uint32_t c) -> bool {
        return mbar_wait(smem_addr(mbar + 1 + p * kStages + c % kStages), (c / kStages) & 1, kSpin);
    };
    auto issue = [&](int p) {  // thread 0: keep up to kStages copies ahead of slot p's consumer
        while (c_issue[p] < c_cons[p] + kStages && ms_next[p] <= a.T) {
            const uint32_t st = c_issue[p] % kStages;
            const uint32_t bar = smem_addr(mbar + 1 + p * kStages + st);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(ms_bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(ring + ((size_t)p * kStages + st) * 10 * N)),
                "l"(noise_bytes + (size_t)ms_next[p] * ms_bytes), "r"(ms_bytes), "r"(bar)
                : "memory");
            c_issue[p]++;
            ms_next[p]++;
        }
    };
    // take the next particle of the batch into slot p (all threads)
    // PL (placement, one particle per CTA, table noise): a.order lists the
    // particles by predicted work, heaviest first.  A CTA that arrives second
    // on its SM takes particles from the light end, every other CTA from the
    // heavy end, so a heavy particle runs alone on an SM or beside a light
    // one, wherever the hardware put the CTAs.  One 64-bit counter holds the
    // heavy claims (high half) and the light claims (low half); a claim is
    // valid while the claims before it number fewer than the particles.  A
    // separate instantiation: claim code in the default kernel changed the
    // code generated for its substep loop and cost 14 %.
    __shared__ int s_light;
    if constexpr (PL) {
        if (threadIdx.x == 0) {
            unsigned smid;
            asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
            s_light = smid < 256 && atomicAdd(a.place_ws + 2 + smid, 1) >= 1;
        }
    }
    auto load = [&](int p) {
        if (threadIdx.x == 0) {
            if constexpr (PL) {
                const unsigned long long c = atomicAdd(reinterpret_cast<unsigned long long*>(a.place_ws),
                                                       s_light ? 1ull : 1ull << 32);
                const int heavy = (int)(c >> 32), light = (int)(unsigned)c;
                s_sim[p] = heavy + light < a.n_sims ? a.order[s_light ? a.n_sims - 1 - light : heavy] : a.n_sims;
            } else {
                s_sim[p] = atomicAdd(a.work_counter, 1);
            }
        }
        __syncthreads();
        sim[p] = s_sim[p];
        live[p] = sim[p] < a.n_sims;
        const int sm = live[p] ? sim[p] : 0;
        Slot& q = sl[p];
        q.GJ = (float)a.G[sm] * C::J_NMDA;
        q.GJa = q.GJ * C::a_E;                 // coupling -> a_E I_E - b_E
        q.GJe = q.GJa * (-C::d_E * LOG2E);     // coupling -> exponent argument of the E rate
        q.wEE = act ? (float)a.wEE[(size_t)sm * N + j] : 0.f;
        q.wEI = act ? (float)a.wEI[(size_t)sm * N + j] : 0.f;
        q.wIE = act ? (float)a.wIE[(size_t)sm * N + j] : 0.f;
        q.delta = (float)a.init_delta;
        q.S_E = q.S_I = 0.001f;
        q.IE = q.II = q.rE = q.rI = 0.f;
        q.mean_IE = 0.0;
        q.bw = BW();
#pragma unroll
        for (int e = 0; e < 6; e++) ext[((size_t)p * 6 + e) * blockDim.x + threadIdx.x] = 0.0;
        for (int k = threadIdx.x; k < 2 * LD; k += blockDim.x) {
            const int o = (k % LD) % K, col = (k % LD) / K * KC + o;  // S_E slot -> column
            S_buf[p * 2 * LD + k] = (o < KC && col < N) ? 0.001f : 0.f;
        }
        ts[p] = 0;
        frame[p] = 0;
        to_frame[p] = 1;
        trial[p] = 0;
        failed[p] = false;
        adjusting[p] = a.adjust_fic != 0;
        ms_next[p] = 0;
        __syncthreads();
    };
#pragma unroll
    for (int p = 0; p < P; p++) {
        c_cons[p] = c_issue[p] = 0;
        load(p);
    }
    int cur = 0;

    for (;;) {
        bool any = false;
#pragma unroll
        for (int p = 0; p < P; p++) any |= live[p];
        if (!any) break;
        const float2* nz[P];
        if (!NZI) {
            if (threadIdx.x == 0) {
#pragma unroll
                for (int p = 0; p < P; p++)
                    if (live[p]) issue(p);
            }
            bool late = false;
#pragma unroll
            for (int p = 0; p < P; p++)
                if (live[p]) late |= !wait_copy(p, c_cons[p]);
            if (__syncthreads_or(late)) {
                timed_out = true;
                break;
            }
#pragma unroll
            for (int p = 0; p < P; p++) nz[p] = ring + ((size_t)p * kStages + c_cons[p] % kStages) * 10 * N + j;
        }
        float4 npair[P];  // NZI: this node's noise for the current substep pair

#pragma unroll
        for (int sub = 0; sub < 10; sub++) {
#if BNM_FAST_CHAIN
            // Rows 1-3 of each lane's slots first: their sums go to the other
            // lanes of the row group by three independent shuffles, whose
            // latency then overlaps the FMAs of slot 0 (this lane's own row,
            // two accumulator chains).
            float2 acc[P][4], acc0b[P];
            float4 sv[P][K / 4];
#pragma unroll
            for (int p = 0; p < P; p++) {
                acc0b[p] = make_float2(0.f, 0.f);
#pragma unroll
                for (int r = 0; r < 4; r++) acc[p][r] = make_float2(0.f, 0.f);
#pragma unroll
                for (int c4 = 0; c4 < K / 4; c4++)
                    sv[p][c4] = reinterpret_cast<const float4*>(S_buf + (p * 2 + cur) * LD + v * K)[c4];
            }
#pragma unroll
            for (int c4 = 0; c4 < K / 4; c4++) {  // pairs 2 c4, 2 c4 + 1 (those below KC / 2)
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const float2 s01 = make_float2(sv[p][c4].x, sv[p][c4].y), s23 = make_float2(sv[p][c4].z, sv[p][c4].w);
#pragma unroll
                    for (int r = 1; r < 4; r++) {
                        acc[p][r] = __ffma2_rn(sc[r][2 * c4], s01, acc[p][r]);
                        if (2 * c4 + 1 < KC / 2) acc[p][r] = __ffma2_rn(sc[r][2 * c4 + 1 < KC / 2 ? 2 * c4 + 1 : 0], s23, acc[p][r]);
                    }
                }
            }
            float rsum[P];
#pragma unroll
            for (int p = 0; p < P; p++) {
                // reduce-scatter over the 4 lanes of this row group: lane v ^ m keeps
                // row v in its slot m, so the three exchanges are independent
                const float r1 = __shfl_xor_sync(0xffffffffu, acc[p][1].x + acc[p][1].y, 1);
                const float r2 = __shfl_xor_sync(0xffffffffu, acc[p][2].x + acc[p][2].y, 2);
                const float r3 = __shfl_xor_sync(0xffffffffu, acc[p][3].x + acc[p][3].y, 3);
                rsum[p] = r1 + (r2 + r3);
            }
#pragma unroll
            for (int c4 = 0; c4 < K / 4; c4++) {
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const float2 s01 = make_float2(sv[p][c4].x, sv[p][c4].y), s23 = make_float2(sv[p][c4].z, sv[p][c4].w);
                    float2& a0 = (c4 & 1) ? acc0b[p] : acc[p][0];
                    a0 = __ffma2_rn(sc[0][2 * c4], s01, a0);
                    if (2 * c4 + 1 < KC / 2) a0 = __ffma2_rn(sc[0][2 * c4 + 1 < KC / 2 ? 2 * c4 + 1 : 0], s23, a0);
                }
            }
#pragma unroll
            for (int p = 0; p < P; p++) {
                Slot& q = sl[p];
                const float coupling = ((acc[p][0].x + acc0b[p].x) + (acc[p][0].y + acc0b[p].y)) + rsum[p];
                float2 n;
                if (NZI) {
                    if (sub % 2 == 0) npair[p] = philox_noise_pair(key0, key1, ts[p], sub / 2, j, N);
                    n = sub % 2 == 0 ? make_float2(npair[p].x, npair[p].y) : make_float2(npair[p].z, npair[p].w);
                } else {
                    n = act ? nz[p][(size_t)sub * N] : make_float2(0.f, 0.f);
                }
                // The dependent chain from the coupling to the new S_E is one FMA to the
                // exponent's argument, the rate, and one FMA to S_E: every term that does
                // not involve the coupling is formed beforehand from the old state.
                const float BE = fmaf(q.wEE, q.S_E, C::w_E__I_0) - q.wIE * q.S_I;  // I_E without coupling
                const float xB = fmaf(C::a_E, BE, -C::b_E);
                q.IE = fmaf(q.GJ, coupling, BE);
                const float xE = fmaf(q.GJa, coupling, xB);  // a_E I_E - b_E
                const float eE = ex2_approx(fmaf(q.GJe, coupling, xB * (-C::d_E * LOG2E)));
                q.rE = rate_from(xE, eE, C::d_E, 1.0f / C::d_E);
                q.II = fmaf(q.wEI, q.S_E, C::w_I__I_0) - q.S_I;
                q.rI = rate(fmaf(C::a_I, q.II, -C::b_I), C::d_I, 1.0f / C::d_I, -C::d_I * LOG2E);
                // S += sigma sqrt(dt) xi + dt ((1-S_E) gamma_E r_E - S_E/tau_E), constants folded;
                // __saturatef clips to [0, 1] and maps NaN to 0 like std::max(0, std::min(S, 1))
                const float aE = fmaf(-kDtGammaE, q.S_E, kDtGammaE);
                const float baseE = q.S_E + fmaf(-kDtInvTauE, q.S_E, SQ * n.x);
                const float dSI = fmaf(kDtGammaI, q.rI, fmaf(-kDtInvTauI, q.S_I, SQ * n.y));
                q.S_E = __saturatef(fmaf(aE, q.rE, baseE));
                q.S_I = __saturatef(q.S_I + dSI);
                if (act) S_buf[(p * 2 + (cur ^ 1)) * LD + pos_j] = q.S_E;
            }
#else
            float2 acc[P][4];
#pragma unroll
            for (int p = 0; p < P; p++)
#pragma unroll
                for (int r = 0; r < 4; r++) acc[p][r] = make_float2(0.f, 0.f);
#pragma unroll
            for (int c4 = 0; c4 < K / 4; c4++) {  // pairs 2 c4, 2 c4 + 1 (those below KC / 2)
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const float4 s = reinterpret_cast<const float4*>(S_buf + (p * 2 + cur) * LD + v * K)[c4];
                    const float2 s01 = make_float2(s.x, s.y), s23 = make_float2(s.z, s.w);
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        acc[p][r] = __ffma2_rn(sc[r][2 * c4], s01, acc[p][r]);
                        if (2 * c4 + 1 < KC / 2) acc[p][r] = __ffma2_rn(sc[r][2 * c4 + 1 < KC / 2 ? 2 * c4 + 1 : 0], s23, acc[p][r]);
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < P; p++) {
                Slot& q = sl[p];
                // reduce-scatter over the 4 lanes of this row group: lane v ^ m keeps
                // row v in its slot m, so the three exchanges are independent (one
                // shuffle latency on the chain instead of two)
                const float r1 = __shfl_xor_sync(0xffffffffu, acc[p][1].x + acc[p][1].y, 1);
                const float r2 = __shfl_xor_sync(0xffffffffu, acc[p][2].x + acc[p][2].y, 2);
                const float r3 = __shfl_xor_sync(0xffffffffu, acc[p][3].x + acc[p][3].y, 3);
                const float coupling = ((acc[p][0].x + acc[p][0].y) + r1) + (r2 + r3);
                float2 n;
                if (NZI) {
                    if (sub % 2 == 0) npair[p] = philox_noise_pair(key0, key1, ts[p], sub / 2, j, N);
                    n = sub % 2 == 0 ? make_float2(npair[p].x, npair[p].y) : make_float2(npair[p].z, npair[p].w);
                } else {
                    n = act ? nz[p][(size_t)sub * N] : make_float2(0.f, 0.f);
                }
                q.IE = fmaf(q.GJ, coupling, fmaf(q.wEE, q.S_E, C::w_E__I_0)) - q.wIE * q.S_I;
                q.II = fmaf(q.wEI, q.S_E, C::w_I__I_0) - q.S_I;
                q.rE = rate(fmaf(C::a_E, q.IE, -C::b_E), C::d_E, 1.0f / C::d_E, -C::d_E * LOG2E);
                q.rI = rate(fmaf(C::a_I, q.II, -C::b_I), C::d_I, 1.0f / C::d_I, -C::d_I * LOG2E);
                // S += sigma sqrt(dt) xi + dt ((1-S_E) gamma_E r_E - S_E/tau_E), constants folded;
                // __saturatef clips to [0, 1] and maps NaN to 0 like std::max(0, std::min(S, 1))
                const float aE = fmaf(-kDtGammaE, q.S_E, kDtGammaE);
                const float dSE = fmaf(aE, q.rE, fmaf(-kDtInvTauE, q.S_E, SQ * n.x));
                const float dSI = fmaf(kDtGammaI, q.rI, fmaf(-kDtInvTauI, q.S_I, SQ * n.y));
                q.S_E = __saturatef(q.S_E + dSE);
                q.S_I = __saturatef(q.S_I + dSI);
                if (act) S_buf[(p * 2 + (cur ^ 1)) * LD + pos_j] = q.S_E;
            }
#endif
            __syncthreads();
            cur ^= 1;
        }

#pragma unroll
        for (int p = 0; p < P; p++) {
            if (!live[p]) continue;
            Slot& q = sl[p];
            c_cons[p]++;  // this millisecond's noise stage is free again
            q.bw.step(q.S_E);
            if (--to_frame[p] == 0) {  // ts % TR == 0
                to_frame[p] = a.TR;
                if (act) {
                    a.bold[((size_t)sim[p] * a.frames + frame[p]) * N + j] = q.bw.bold();
                    if (frame[p] >= a.n_vols_remove) {
                        double* e = ext + (size_t)p * 6 * blockDim.x + threadIdx.x;
                        e[0 * blockDim.x] += q.S_E;
                        e[1 * blockDim.x] += q.IE;
                        e[2 * blockDim.x] += q.rE;
                        e[3 * blockDim.x] += q.S_I;
                        e[4 * blockDim.x] += q.II;
                        e[5 * blockDim.x] += q.rI;
                    }
                }
                frame[p]++;
            }
            ts[p]++;
            if (adjusting[p]) {
                if (ts[p] >= a.samp_start && ts[p] <= a.samp_end) q.mean_IE += (double)q.IE;
                if (ts[p] == a.samp_end) {
                    bool needs = false;
                    if (act) {
                        const double diff = q.mean_IE / duration - (double)C::b_a_ratio_E;
                        if (fabs(diff + 0.026) > 0.005) {
                            needs = true;
                            if (trial[p] < a.max_trials) {
                                if (diff < -0.026) {
                                    q.wIE -= q.delta;
                                    q.delta = fmaxf(q.delta - 0.001f, 0.001f);
                                } else {
                                    q.wIE += q.delta;
                                }
                            }
                        }
                    }
                    if (__syncthreads_or(needs)) {
                        if (trial[p] < a.max_trials) {
                            q.S_E = q.S_I = 0.001f;
                            q.bw = BW();
                            q.mean_IE = 0.0;
#pragma unroll
                            for (int e = 0; e < 6; e++) ext[((size_t)p * 6 + e) * blockDim.x + threadIdx.x] = 0.0;
                            if (act) S_buf[(p * 2 + cur) * LD + pos_j] = q.S_E;
                            ts[p] = 0;
                            frame[p] = 0;
                            to_frame[p] = 1;
                            trial[p]++;
                            if (!NZI) {
                                // the copies already in flight hold milliseconds after
                                // the restart point: let them land, then refetch from 0
                                if (threadIdx.x == 0) s_flag = (int)c_issue[p];
                                __syncthreads();
                                const uint32_t in_flight_end = (uint32_t)s_flag;
                                bool lt = false;
                                for (; c_cons[p] < in_flight_end; c_cons[p]++) lt |= !wait_copy(p, c_cons[p]);
                                if (threadIdx.x == 0) ms_next[p] = 0;
                                if (__syncthreads_or(lt)) timed_out = true;
                            }
                        } else {
                            failed[p] = true;
                            adjusting[p] = false;
                        }
                    } else {
                        adjusting[p] = false;
                    }
                    __syncthreads();
                }
            }
            if (ts[p] > a.T) {  // particle done: write it out, take the next one
                if (act) {
                    a.wIE_out[(size_t)sim[p] * N + j] = (double)q.wIE;
                    const double kept = (double)(frame[p] - a.n_vols_remove);
#pragma unroll
                    for (int e = 0; e < 6; e++)
                        a.ext[((size_t)sim[p] * 6 + e) * N + j] = ext[((size_t)p * 6 + e) * blockDim.x + threadIdx.x] / kept;
                }
                if (threadIdx.x == 0) {
                    a.trials[sim[p]] = trial[p];
                    a.failed[sim[p]] = failed[p] ? 1 : 0;
                }
                load(p);
            }
        }
        if (timed_out) break;
    }
    if (timed_out) {
        if (threadIdx.x == 0) {
            atomicOr(a.status, kStatusTimeout);
            // bounded wait for this CTA's own copies before the CTA exits
#pragma unroll
            for (int p = 0; p < P; p++)
                for (uint32_t c = c_cons[p]; c < c_issue[p]; c++) wait_copy(p, c);
        }
        __syncthreads();
    }
}

template <int K, int KC, int P, bool NZI>
static size_t fast_smem(int N, int threads) {
    return (NZI ? 0 : (size_t)P * kStages * 10 * N * sizeof(float2)) + (size_t)N * 4 * K * sizeof(float) +
           (size_t)P * 2 * 4 * K * sizeof(float) + (size_t)P * 6 * threads * sizeof(double) +
           (1 + P * kStages) * sizeof(uint64_t);
}

template <int K, int KC, int P>
static cudaError_t launch_fast(const SimArgs& a, int grid, cudaStream_t st) {
    const int threads = ((a.N + 31) / 32) * 32;
    if (!a.noise) {  // noise drawn in the kernel
        const size_t smem = fast_smem<K, KC, P, true>(a.N, threads);
        cudaError_t e = cudaFuncSetAttribute(integrate_fast_kernel<K, KC, P, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        integrate_fast_kernel<K, KC, P, true><<<grid, threads, smem, st>>>(a);
        return cudaGetLastError();
    }
    const size_t smem = fast_smem<K, KC, P, false>(a.N, threads);
    if constexpr (P == 1) {
        if (a.order) {  // placement
            cudaError_t e = cudaFuncSetAttribute(integrate_fast_kernel<K, KC, 1, false, true>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            integrate_fast_kernel<K, KC, 1, false, true><<<grid, threads, smem, st>>>(a);
            return cudaGetLastError();
        }
    }
    cudaError_t e = cudaFuncSetAttribute(integrate_fast_kernel<K, KC, P, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    integrate_fast_kernel<K, KC, P, false><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int K, int KC, int P, bool NZI>
static double share_fast_t(const SimArgs& a, int grid, int num_sms) {
    const int threads = ((a.N + 31) / 32) * 32;
    const size_t smem = fast_smem<K, KC, P, NZI>(a.N, threads);
    int per_sm = 0;
    if (cudaFuncSetAttribute(integrate_fast_kernel<K, KC, P, NZI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, integrate_fast_kernel<K, KC, P, NZI>, threads, smem) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return 1.0;
    }
    const double cap = (double)per_sm * num_sms;
    return grid >= cap ? 1.0 : grid / cap;
}

template <int K, int KC, int P>
static double share_fast(const SimArgs& a, int grid, int num_sms) {
    return a.noise ? share_fast_t<K, KC, P, false>(a, grid, num_sms) : share_fast_t<K, KC, P, true>(a, grid, num_sms);
}

}  // namespace bnm

// Columns per lane of the register kernel: ceil(N / 4) rounded up to even.
static int fast_kc(int N) { return ((N + 3) / 4 + 1) / 2 * 2; }

// Padded SC row length (4K) of the register kernel for a node count (0 = the
// register kernel does not cover it).
extern "C" int bnm_fast_kmax(int N) {
    if (N <= 0 || N > 128) return 0;
    const int K = ((N + 3) / 4 + 3) / 4 * 4;
    return 4 * K;
}

// Launches one integrator shape (IntegratorShape in kernels.h).
cudaError_t bnm_launch_integrate_shape(const bnm::SimArgs& a, const bnm::IntegratorShape& sh, int num_sms,
                                       cudaStream_t st) {
    using namespace bnm;
    if (sh.kind == 0) {
        const int ld = bnm_fast_kmax(a.N);
        if (!ld || a.sc_ld != ld || (sh.slots != 1 && sh.slots != 2)) return cudaErrorInvalidValue;
        if (a.noise && a.noise_ld != a.N) return cudaErrorInvalidValue;
        // CTAs are persistent over the batch: two per SM with one slot, one with two
        const int P = sh.slots;
        int grid = (a.n_sims + P - 1) / P;
        const int max_grid = P == 1 ? 2 * num_sms : num_sms;
        if (grid > max_grid) grid = max_grid;
        const int kc = fast_kc(a.N);
        switch ((ld / 4) * 8 + (ld / 4 - kc) * 2 + P) {
#define BNM_K(K)                                                            \
    case K * 8 + 1: return launch_fast<K, K, 1>(a, grid, st);            \
    case K * 8 + 2: return launch_fast<K, K, 2>(a, grid, st);            \
    case K * 8 + 4 + 1: return launch_fast<K, K - 2, 1>(a, grid, st); \
    case K * 8 + 4 + 2: return launch_fast<K, K - 2, 2>(a, grid, st);
            BNM_K(4) BNM_K(8) BNM_K(12) BNM_K(16) BNM_K(20) BNM_K(24) BNM_K(28) BNM_K(32)
#undef BNM_K
            default: return cudaErrorInvalidValue;
        }
    }
    if (sh.kind == 1) {
        if (a.noise && a.noise_ld != a.N) return cudaErrorInvalidValue;
        return bnm_launch_integrate_cluster(a, sh.csize, sh.rpw, sh.kr, st);
    }
    if (sh.kind == 3 || sh.kind == 4) {
        // an odd node count runs with one padding node: the plan's noise table
        // and SC carry its column (and SC row)
        SimArgs b = a;
        b.N = a.N + (a.N & 1);
        if ((a.noise && a.noise_ld != b.N) || a.sc_ld < b.N) return cudaErrorInvalidValue;
        return bnm_launch_integrate_colsplit(b, sh.csize, sh.rpw, sh.slots, sh.kr, sh.kind == 4 ? 2 : 1, st);
    }
    if (sh.kind != 2 || !a.noise) return cudaErrorInvalidValue;  // the reference-order kernel reads a table
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

double bnm_integrator_share(const bnm::SimArgs& a, const bnm::IntegratorShape& sh, int num_sms) {
    using namespace bnm;
    if (sh.kind == 0) {
        const int ld = bnm_fast_kmax(a.N);
        if (!ld || (sh.slots != 1 && sh.slots != 2)) return 1.0;
        const int P = sh.slots;
        int grid = (a.n_sims + P - 1) / P;
        const int max_grid = P == 1 ? 2 * num_sms : num_sms;
        if (grid > max_grid) grid = max_grid;
        const int kc = fast_kc(a.N);
        switch ((ld / 4) * 8 + (ld / 4 - kc) * 2 + P) {
#define BNM_K(K)                                                                  \
    case K * 8 + 1: return share_fast<K, K, 1>(a, grid, num_sms);              \
    case K * 8 + 2: return share_fast<K, K, 2>(a, grid, num_sms);              \
    case K * 8 + 4 + 1: return share_fast<K, K - 2, 1>(a, grid, num_sms); \
    case K * 8 + 4 + 2: return share_fast<K, K - 2, 2>(a, grid, num_sms);
            BNM_K(4) BNM_K(8) BNM_K(12) BNM_K(16) BNM_K(20) BNM_K(24) BNM_K(28) BNM_K(32)
#undef BNM_K
            default: return 1.0;
        }
    }
    if (sh.kind == 1) return bnm_cluster_share(a.N, sh.csize, sh.rpw, sh.kr, a.n_sims);
    if (sh.kind == 3 || sh.kind == 4)
        return bnm_colsplit_share(a.N + (a.N & 1), sh.csize, sh.rpw, sh.slots, sh.kr, sh.kind == 4 ? 2 : 1, a.n_sims);
    return 1.0;  // the reference-order kernel fills the GPU (two CTAs per SM, persistent)
}

int bnm_integrator_candidates(int N, bnm::IntegratorShape* out, int max) {
    using namespace bnm;
    int n = 0;
    auto add = [&](IntegratorShape s) {
        if (n < max) out[n] = s;
        n++;
    };
    if (bnm_fast_kmax(N)) {
        add({0, 1, 0, 0, 0});
        add({0, 2, 0, 0, 0});
        return n < max ? n : max;
    }
    const int kc = (N + 31) / 32;
    const int kr_all = kc < 8 ? kc : 8;
    const int shapes[3][2] = {{8, 4}, {8, kr_all}, {16, 4}};
    for (int cs : {1, 2, 4, 8})
        for (int v = 0; v < 3; v++) {
            if (v == 1 && kr_all == 4) continue;  // same as {8, 4}
            int threads, rows;
            size_t smem;
            if (bnm_cluster_shape(N, cs, shapes[v][0], shapes[v][1], &threads, &rows, &smem))
                add({1, 0, cs, shapes[v][0], shapes[v][1]});
        }
    int vs[4 * 64];
    const int nv = bnm_colsplit_variants(vs, 64);
    const int Nc = N + (N & 1);  // column-split shapes of an odd N include one padding node
    for (int cs : {1, 2, 4, 8})
        for (int v = 0; v < nv && v < 64; v++) {
            int threads, rows;
            size_t smem;
            const int rpl = vs[4 * v], k2 = vs[4 * v + 1], krp = vs[4 * v + 2], np = vs[4 * v + 3];
            bool dup = false;  // the variant table repeats (rpl, k2, k2) when k2 <= 8
            for (int u = 0; u < v; u++)
                dup |= vs[4 * u] == rpl && vs[4 * u + 1] == k2 && vs[4 * u + 2] == krp && vs[4 * u + 3] == np;
            if (!dup && bnm_colsplit_shape(Nc, cs, rpl, k2, krp, np, &threads, &rows, &smem))
                add({np == 2 ? 4 : 3, k2, cs, rpl, krp});
        }
    add({2, 0, 0, 0, 0});
    return n < max ? n : max;
}
