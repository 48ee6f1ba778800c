// FP32 integrator for 128 < N <= 512: one thread-block cluster per particle.
//
// Same model, time loop, FIC restarts, BOLD and extended outputs as the
// reference's bnm kernel (bnm.cu:72-315) and CPU path (bnm.cpp:167-290), and
// the same arithmetic as the register integrator of integrate_fast.cu.  What
// changes is where SC lives: at N = 400 one SC matrix is 640 KB, more than an
// SM's registers and shared memory together, so a cluster of C CTAs (C picked
// by the autotuner) splits it by rows:
//   * CTA rank c owns nodes [c R, c R + R); warp w of it owns RPW consecutive
//     nodes.  Lane l holds, for each of those rows, the columns l + 32 k
//     (k < KC = N/32 rounded up): chunks k < KR in registers as row pairs
//     for packed FMA (fma.rn.f32x2), the rest in shared memory
//     (conflict-free, one float2 per lane per row pair and chunk);
//   * each substep a lane reads its KC entries of S_E once (shared memory),
//     forms RPW partial row sums, and a butterfly reduce-scatter over the 32
//     lanes leaves every row's full sum in the 32/RPW lanes l / (32/RPW) ==
//     row, which update that node redundantly (no divergence);
//   * the new S_E of a node goes to the S_E buffer of every CTA of the
//     cluster by asynchronous distributed-shared-memory stores (st.async, one
//     replica lane per destination rank) that count their bytes on the
//     destination's mbarrier; S_E is double buffered and a CTA waits only for
//     its own buffer to fill (no cluster-wide barrier per substep).  A remote
//     CTA can refill a buffer only after it has this CTA's next S_E, which is
//     sent after this CTA has read the buffer, so the double buffer is safe;
//   * noise arrives one simulated millisecond ahead through a 4-stage
//     shared-memory ring of bulk copies (each CTA copies only its own nodes:
//     ten contiguous runs of R x (E, I) per millisecond), tracked by
//     mbarriers with bounded waits;
//   * cluster-wide decisions (a late noise copy, the numerical-FIC restart)
//     are exchanged as flags through distributed shared memory and read after
//     a cluster barrier, so every CTA of a cluster takes the same branch and
//     meets the same barriers.
#include <cstdlib>
#include <cstring>
#include <vector>
#include "kernels.h"
#include "fp32_model.cuh"
#include "noise.cuh"
#include "cluster_util.cuh"

namespace bnm {
namespace {

constexpr int kRing = 4;  // noise ring stages (milliseconds)
// A late noise copy or S_E exchange is agreed on cluster-wide every kAgreeMs
// milliseconds (and at the FIC decision and the last millisecond), not every
// millisecond: a CTA that saw a wait run out stops issuing copies and waiting
// but keeps computing and sending until the next agreement point, so every
// CTA reaches the same points.  A CTA that stopped arming its S_E barriers
// collects at most kAgreeMs * 5 * 4 N <= 163840 bytes of negative tx-count
// per barrier (N <= 512), inside the mbarrier's 2^20 - 1 range.
constexpr int kAgreeMs = 16;

// Shared-memory layout (bytes), in this order:
//   S      [2][32 KC] float          S_E of every node, double buffered
//   SCs    [W][RPW/2][KC-KR][32] float2  shared-memory part of the SC slice
//   ring   [kRing][10][R] float2     noise of the own nodes, per millisecond
//   ext    [6][W RPW] double         extended-output sums of the own nodes
//   flags  [32] int                  late[2][8], fic[8]
//   mbar   [kRing + 2] uint64       noise stages, then S_E buffers 0 and 1
template <int RPW, int KC, int KR>
struct ClusterLayout {
    static constexpr int kNP = 32 * KC;
    __host__ __device__ static size_t sc_bytes(int W) { return (size_t)W * (RPW / 2) * (KC - KR) * 32 * sizeof(float2); }
    __host__ __device__ static size_t ring_off(int W) { return 2 * kNP * sizeof(float) + sc_bytes(W); }
    __host__ __device__ static size_t ext_off(int W, int R) { return ring_off(W) + (size_t)kRing * 10 * R * sizeof(float2); }
    __host__ __device__ static size_t flags_off(int W, int R) { return ext_off(W, R) + (size_t)6 * W * RPW * sizeof(double); }
    __host__ __device__ static size_t mbar_off(int W, int R) { return flags_off(W, R) + 32 * sizeof(int); }
    __host__ __device__ static size_t bytes(int W, int R) { return mbar_off(W, R) + (kRing + 2) * sizeof(uint64_t); }
};

template <int RPW, int KC, int KR>
__global__ void integrate_cluster_kernel(SimArgs a, int R) {
    static_assert(RPW == 4 || RPW == 8 || RPW == 16, "RPW");
    static_assert(KR >= 0 && KR <= KC, "KR");
    constexpr int NP = 32 * KC;
    constexpr int NREP = 32 / RPW;  // lanes holding each row after the reduction
    constexpr int NPAIR = RPW / 2;
    constexpr int KS = KC - KR;     // chunks in shared memory
    typedef Model<float> C;
    typedef ClusterLayout<RPW, KC, KR> L;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int N = a.N;
    const int W = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t crank = cluster_rank(), csize = cluster_size();
    const int sim = blockIdx.x / csize;
    const int r0 = (int)crank * R;
    const int r_own = max(0, min(N - r0, R));  // nodes this CTA updates

    float* S_buf = reinterpret_cast<float*>(smem_raw);
    float2* SCs = reinterpret_cast<float2*>(smem_raw + 2 * NP * sizeof(float));
    float2* ring = reinterpret_cast<float2*>(smem_raw + L::ring_off(W));
    double* ext = reinterpret_cast<double*>(smem_raw + L::ext_off(W, R));
    int* flags = reinterpret_cast<int*>(smem_raw + L::flags_off(W, R));  // late[2][8] at 0, fic[8] at 16, issue at 24
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + L::mbar_off(W, R));

    const int rho = lane / NREP, rep = lane % NREP;
    const int lr = w * RPW + rho;  // local row (node r0 + lr) this lane updates
    const int node = r0 + lr;
    const bool act = lr < r_own;
    const bool owner = act && rep == 0;  // writes outputs
    const bool every_warp_owns = (W - 1) * RPW < r_own;  // the last warp holds a node of this CTA
    const long long kSpin = kWaitNs;  // wall-clock limit of each bounded wait

    // every CTA of the cluster is running before any distributed shared memory access
    cluster_sync();
    if (threadIdx.x == 0) {
        for (int b = 0; b < kRing + 2; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar + b)) : "memory");
        // buffer 1 receives S_E after the first substep: N values of 4 bytes
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar + kRing + 1)),
                     "r"(4 * N)
                     : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = threadIdx.x; k < 2 * NP; k += blockDim.x) S_buf[k] = (k % NP) < N ? 0.001f : 0.f;
    for (int k = threadIdx.x; k < 6 * W * RPW; k += blockDim.x) ext[k] = 0.0;
    if (threadIdx.x < 32) flags[threadIdx.x] = 0;

    // SC slice: rows r0 + w RPW + 2p (+1), columns k 32 + lane; zero outside the matrix
    float2 scr[NPAIR][KR > 0 ? KR : 1];
#pragma unroll
    for (int p = 0; p < NPAIR; p++) {
        const int ra = w * RPW + 2 * p, rb = ra + 1;
#pragma unroll
        for (int k = 0; k < KC; k++) {
            const int col = k * 32 + lane;
            const float va = (ra < r_own && col < N) ? a.sc_f32[(size_t)(r0 + ra) * a.sc_ld + col] : 0.f;
            const float vb = (rb < r_own && col < N) ? a.sc_f32[(size_t)(r0 + rb) * a.sc_ld + col] : 0.f;
            if (k < KR)
                scr[p][k < KR ? k : 0] = make_float2(va, vb);
            else
                SCs[((size_t)(w * NPAIR + p) * KS + (k - KR)) * 32 + lane] = make_float2(va, vb);
        }
    }
    // buffers initialised in every CTA before anyone writes remote S_E
    cluster_sync();

    // per-lane distributed-shared-memory targets: replica `rep` serves ranks rep, rep + NREP, ...
    const uint32_t s_local = smem_addr(S_buf);
    const uint32_t flags_local = smem_addr(flags);

    const char* noise_bytes = reinterpret_cast<const char*>(a.noise);  // NULL: Philox noise drawn in place
    const uint32_t key0 = (uint32_t)a.noise_seed, key1 = (uint32_t)(a.noise_seed >> 32);
    const uint32_t run_bytes = (uint32_t)(r_own * sizeof(float2));  // one substep of the own nodes
    const double duration = (double)(a.samp_end - a.samp_start + 1);
    const float SQ = C::sigma_model * C::sqrt_dt;
    const float LOG2E = 1.4426950408889634f;
    const float kDtGammaE = C::dt * C::gamma_E, kDtInvTauE = C::dt / C::tau_E;
    const float kDtGammaI = C::dt * C::gamma_I, kDtInvTauI = C::dt / C::tau_I;

    float GJ = (float)a.G[sim] * C::J_NMDA;
    float wEE = act ? (float)a.wEE[(size_t)sim * N + node] : 0.f;
    float wEI = act ? (float)a.wEI[(size_t)sim * N + node] : 0.f;
    float wIE = act ? (float)a.wIE[(size_t)sim * N + node] : 0.f;
    float delta = (float)a.init_delta;
    float S_E = 0.001f, S_I = 0.001f, IE = 0.f, II = 0.f, rE = 0.f, rI = 0.f;
    double mean_IE = 0.0;
    BW bw;
    int ts = 0, frame = 0, to_frame = 1, trial = 0, ms_next = 0;
    bool failed = false, adjusting = a.adjust_fic != 0, timed_out = false;
    uint32_t c_cons = 0, c_issue = 0;
    int cur = 0;
    // S_E exchange: buffer b's mbarrier (mbar[kRing + b]) completes a phase
    // when all N values of the next S_E have landed there; ph bit b is the
    // parity this CTA waits for next.  Buffer 0 starts filled locally.
    uint32_t ph = 0;
    bool skip_wait = true;
    const uint32_t sbar_local = smem_addr(mbar + kRing);
    auto wait_s = [&](int b) -> bool {
        const bool ok = mbar_wait(sbar_local + 8u * b, (ph >> b) & 1u, kSpin);
        ph ^= 1u << b;
        return ok;
    };

    auto wait_copy = [&](uint32_t c) -> bool {
        return mbar_wait(smem_addr(mbar + c % kRing), (c / kRing) & 1, kSpin);
    };
    auto issue = [&]() {  // thread 0: keep up to kRing milliseconds in flight
        while (c_issue < c_cons + kRing && ms_next <= a.T) {
            const uint32_t st = c_issue % kRing;
            const uint32_t bar = smem_addr(mbar + st);
            if (run_bytes) {
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(10 * run_bytes)
                             : "memory");
                for (int sub = 0; sub < 10; sub++)
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                            smem_addr(ring + ((size_t)st * 10 + sub) * R)),
                        "l"(noise_bytes + (((size_t)ms_next * 10 + sub) * N + r0) * sizeof(float2)), "r"(run_bytes),
                        "r"(bar)
                        : "memory");
            } else {  // a CTA without nodes still keeps the phase sequence
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
            }
            c_issue++;
            ms_next++;
        }
    };
    // flags[slot] of every CTA <- v (threads 0 .. csize-1 each write one rank)
    auto broadcast_flag = [&](int slot, int v) {
        if (threadIdx.x < csize) st_cluster_s32(map_rank(flags_local + 4u * slot, threadIdx.x), v);
    };

    bool late = false;  // sticky; block-uniform after each __syncthreads_or
    int since_agree = 0, n_agree = 0;
    while (ts <= a.T) {
        if (a.noise) {
            if (threadIdx.x == 0 && !late) issue();
            late = __syncthreads_or(late || !wait_copy(c_cons));
        } else {  // Philox noise drawn by the block instead of copied from a table
            philox_fill_stage(ring + (size_t)(c_cons % kRing) * 10 * R, R, r0, r_own, a.n_real, ts, key0, key1);
            late = __syncthreads_or(late);
        }
        const float2* nz = ring + (size_t)(c_cons % kRing) * 10 * R + (act ? lr : 0);

#pragma unroll 1
        for (int sub = 0; sub < 10; sub++) {
            if (!skip_wait && !late) late = !wait_s(cur);
            skip_wait = false;
            // A warp sends its nodes' next S_E only after all its lanes have read
            // buffer cur and passed its wait, and the other CTAs need every node's
            // S_E before this buffer's next phase can fill: where every warp of
            // the CTA owns a node, no block barrier is needed here.  A CTA with
            // a warp that owns none (the last rank of some shapes) keeps one.
            if (!every_warp_owns) __syncthreads();
            if (threadIdx.x == 0 && !late)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sbar_local + 8u * cur),
                             "r"(4 * N)
                             : "memory");
            const float* Sc = S_buf + cur * NP;
            float s[KC];
#pragma unroll
            for (int k = 0; k < KC; k++) s[k] = Sc[k * 32 + lane];
            float2 acc[NPAIR];
#pragma unroll
            for (int p = 0; p < NPAIR; p++) acc[p] = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < KC; k++) {
                const float2 ss = make_float2(s[k], s[k]);
#pragma unroll
                for (int p = 0; p < NPAIR; p++) {
                    const float2 m = (k < KR) ? scr[p][k < KR ? k : 0]
                                              : SCs[((size_t)(w * NPAIR + p) * KS + (k - KR)) * 32 + lane];
                    acc[p] = __ffma2_rn(m, ss, acc[p]);
                }
            }
            // butterfly reduce-scatter: after the step on lane bit b the lane keeps the
            // half of its rows selected by that bit; the row left is lane / NREP
            float v[RPW];
#pragma unroll
            for (int p = 0; p < NPAIR; p++) {
                v[2 * p] = acc[p].x;
                v[2 * p + 1] = acc[p].y;
            }
#pragma unroll
            for (int m = RPW, b = 16; m > 1; m >>= 1, b >>= 1) {
                const bool hi = (lane & b) != 0;
#pragma unroll
                for (int i = 0; i < m / 2; i++) {
                    const float keep = hi ? v[i + m / 2] : v[i];
                    const float send = hi ? v[i] : v[i + m / 2];
                    v[i] = keep + __shfl_xor_sync(0xffffffffu, send, b);
                }
            }
#pragma unroll
            for (int b = NREP / 2; b >= 1; b >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], b);
            const float coupling = v[0];

            const float2 n = act ? nz[(size_t)sub * R] : make_float2(0.f, 0.f);
            IE = fmaf(GJ, coupling, fmaf(wEE, S_E, C::w_E__I_0)) - wIE * S_I;
            II = fmaf(wEI, S_E, C::w_I__I_0) - S_I;
            rE = rate(fmaf(C::a_E, IE, -C::b_E), C::d_E, 1.0f / C::d_E, -C::d_E * LOG2E);
            rI = rate(fmaf(C::a_I, II, -C::b_I), C::d_I, 1.0f / C::d_I, -C::d_I * LOG2E);
            const float aE = fmaf(-kDtGammaE, S_E, kDtGammaE);
            const float dSE = fmaf(aE, rE, fmaf(-kDtInvTauE, S_E, SQ * n.x));
            const float dSI = fmaf(kDtGammaI, rI, fmaf(-kDtInvTauI, S_I, SQ * n.y));
            S_E = __saturatef(S_E + dSE);
            S_I = __saturatef(S_I + dSI);
            if (act) {  // to buffer cur^1 of every CTA; its mbarrier counts the bytes
                const uint32_t dst = s_local + (uint32_t)(((cur ^ 1) * NP + node) * sizeof(float));
                const uint32_t bar = sbar_local + 8u * (cur ^ 1);
                for (uint32_t t = rep; t < csize; t += NREP) st_async_f32(map_rank(dst, t), S_E, map_rank(bar, t));
            }
            cur ^= 1;
        }
        // a late noise copy or S_E exchange anywhere stops the whole cluster at
        // the next agreement point (ts, adjusting and the counters are the
        // same in every CTA, so all of them stop here together)
        if (++since_agree == kAgreeMs || ts == a.T || (adjusting && ts + 1 == a.samp_end)) {
            since_agree = 0;
            const int lslot = (n_agree++ & 1) * 8;
            broadcast_flag(lslot + (int)crank, __syncthreads_or(late) ? 1 : 0);
            cluster_sync();
            bool any_late = false;
            for (uint32_t t = 0; t < csize; t++) any_late |= flags[lslot + t] != 0;
            if (any_late) {
                timed_out = true;
                break;
            }
        }
        c_cons++;
        bw.step(S_E);
        if (--to_frame == 0) {  // ts % TR == 0
            to_frame = a.TR;
            if (owner) {
                a.bold[((size_t)sim * a.frames + frame) * N + node] = bw.bold();
                if (frame >= a.n_vols_remove) {
                    double* e = ext + lr;
                    const int ld = W * RPW;
                    e[0 * ld] += S_E;
                    e[1 * ld] += IE;
                    e[2 * ld] += rE;
                    e[3 * ld] += S_I;
                    e[4 * ld] += II;
                    e[5 * ld] += rI;
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
                broadcast_flag(16 + (int)crank, __syncthreads_or(needs) ? 1 : 0);
                cluster_sync();
                bool any = false;
                for (uint32_t t = 0; t < csize; t++) any |= flags[16 + t] != 0;
                if (any) {
                    if (trial < a.max_trials) {
                        S_E = S_I = 0.001f;
                        bw = BW();
                        mean_IE = 0.0;
                        if (owner)
                            for (int e = 0; e < 6; e++) ext[e * W * RPW + lr] = 0.0;
                        // the S_E the next substep would read is in flight: let it land,
                        // then overwrite the buffer locally with the restart state
                        bool lt = !wait_s(cur);
                        skip_wait = true;
                        __syncthreads();
                        for (int k = threadIdx.x; k < N; k += blockDim.x) S_buf[cur * NP + k] = 0.001f;
                        ts = 0;
                        frame = 0;
                        to_frame = 1;
                        trial++;
                        // copies in flight hold milliseconds after the restart point:
                        // let them land, then refetch from millisecond 0 (thread 0
                        // issues, so it publishes how far it got)
                        if (threadIdx.x == 0) flags[24] = (int)c_issue;
                        __syncthreads();
                        const uint32_t in_flight_end = (uint32_t)flags[24];
                        for (; c_cons < in_flight_end; c_cons++) lt |= !wait_copy(c_cons);
                        ms_next = 0;
                        if (lt && threadIdx.x == 0) atomicOr(a.status, kStatusTimeout);
                    } else {
                        failed = true;
                        adjusting = false;
                    }
                } else {
                    adjusting = false;
                }
                cluster_sync();  // fic flags may be rewritten only after every CTA read them
            }
        }
    }
    if (!timed_out && owner) {
        a.wIE_out[(size_t)sim * N + node] = (double)wIE;
        const double kept = (double)(frame - a.n_vols_remove);
        for (int e = 0; e < 6; e++) a.ext[((size_t)sim * 6 + e) * N + node] = ext[e * W * RPW + lr] / kept;
    }
    if (!timed_out && crank == 0 && threadIdx.x == 0) {
        a.trials[sim] = trial;
        a.failed[sim] = failed ? 1 : 0;
    }
    if (timed_out) {
        if (threadIdx.x == 0) {
            atomicOr(a.status, kStatusTimeout);
            // own copies land before exit: once a wait ran out no copy was
            // issued, so only the last one of each ring stage can be in flight
            for (uint32_t c = c_issue > (uint32_t)kRing ? c_issue - kRing : 0; c < c_issue; c++) wait_copy(c);
        }
        __syncthreads();
    }
    // the S_E sent at the last substep lands before anyone leaves: no CTA
    // exits while another may still write its shared memory
    if (!skip_wait) wait_s(cur);
    cluster_sync();
}

// ---------------------------------------------------------------- launch

struct Variant {
    int rpw, kc, kr;
    const void* fn;
    size_t (*bytes)(int W, int R);
};

template <int RPW, int KC, int KR>
Variant make_variant() {
    return {RPW, KC, KR, (const void*)&integrate_cluster_kernel<RPW, KC, KR>, &ClusterLayout<RPW, KC, KR>::bytes};
}

// KC in 5..16 (N in 129..512); rows per warp 8 or 16; 4 or 8 column chunks in registers
#define BNM_V(KC) make_variant<8, KC, 4>(), make_variant<8, KC, (KC < 8 ? KC : 8)>(), make_variant<16, KC, 4>()
const std::vector<Variant>& variants() {
    static const std::vector<Variant> v = {BNM_V(5),  BNM_V(6),  BNM_V(7),  BNM_V(8),  BNM_V(9),  BNM_V(10),
                                           BNM_V(11), BNM_V(12), BNM_V(13), BNM_V(14), BNM_V(15), BNM_V(16)};
    return v;
}
#undef BNM_V

}  // namespace
}  // namespace bnm

using namespace bnm;

// Checks one cluster configuration for node count N and fills its launch
// shape; returns false when it cannot run (too many threads, registers or
// shared memory, or no cluster of that size fits).
extern "C" int bnm_cluster_shape(int N, int csize, int rpw, int kr, int* threads, int* rows, size_t* smem) {
    if (N <= 0 || N > 512 || (N & 1) || csize < 1 || csize > 8) return 0;
    const int kc = (N + 31) / 32;
    for (const Variant& v : variants()) {
        if (v.rpw != rpw || v.kc != kc || v.kr != kr || v.kr > v.kc) continue;
        int R = (N + csize - 1) / csize;
        R += R & 1;  // bulk copies of the own nodes' noise need even node runs
        if ((csize - 1) * R >= N) return 0;  // a rank without nodes
        const int W = (R + rpw - 1) / rpw;
        if (W * 32 > 1024) return 0;
        // the register file is split over the SM's four partitions, so the
        // kernel's own limit (not 65536 / registers) bounds the block size
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, v.fn) != cudaSuccess) return 0;
        if (W * 32 > fa.maxThreadsPerBlock) return 0;
        const size_t sm = v.bytes(W, R);
        if (sm > 227 * 1024) return 0;
        *threads = W * 32;
        *rows = R;
        *smem = sm;
        return 1;
    }
    return 0;
}

// Diagnostics of one cluster shape for n_sims particles: out[0] threads,
// out[1] rows per CTA, out[2] shared-memory bytes, out[3] registers per
// thread, out[4] the kernel's maximum threads per block, out[5] clusters that
// can be resident at once (negative: the CUDA error of that query).
extern "C" int bnm_cluster_probe(int N, int csize, int rpw, int kr, int n_sims, int* out) {
    for (int i = 0; i < 6; i++) out[i] = 0;
    int threads = 0, R = 0;
    size_t smem = 0;
    const int kc = (N + 31) / 32;
    const void* fn = nullptr;
    for (const Variant& v : variants())
        if (v.rpw == rpw && v.kc == kc && v.kr == kr) fn = v.fn;
    if (!fn) return 1;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return 2;
    out[3] = fa.numRegs;
    out[4] = fa.maxThreadsPerBlock;
    if (!bnm_cluster_shape(N, csize, rpw, kr, &threads, &R, &smem)) return 3;
    out[0] = threads;
    out[1] = R;
    out[2] = (int)smem;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return 4;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3((unsigned)(n_sims * csize));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
    out[5] = e == cudaSuccess ? clusters : -(int)e;
    cudaGetLastError();
    return 0;
}

// Fraction of the GPU one launch of this shape fills: its clusters over the
// clusters that can be resident at once (1 when the query fails).
extern "C" double bnm_cluster_share(int N, int csize, int rpw, int kr, int n_sims) {
    int out[6];
    if (bnm_cluster_probe(N, csize, rpw, kr, n_sims, out) || out[5] < 1) return 1.0;
    return n_sims >= out[5] ? 1.0 : (double)n_sims / out[5];
}

cudaError_t bnm_launch_integrate_cluster(const SimArgs& a, int csize, int rpw, int kr, cudaStream_t st) {
    int threads = 0, R = 0;
    size_t smem = 0;
    if (!bnm_cluster_shape(a.N, csize, rpw, kr, &threads, &R, &smem)) return cudaErrorInvalidValue;
    if (a.sc_ld < a.N) return cudaErrorInvalidValue;
    const int kc = (a.N + 31) / 32;
    const void* fn = nullptr;
    for (const Variant& v : variants())
        if (v.rpw == rpw && v.kc == kc && v.kr == kr) fn = v.fn;
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3((unsigned)(a.n_sims * csize));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
    if (e != cudaSuccess) return e;
    if (clusters < 1) return cudaErrorInvalidConfiguration;
    void* args[] = {(void*)&a, (void*)&R};
    return cudaLaunchKernelExC(&cfg, fn, args);
}
