// FP32 integrator for 128 < N <= 1024, column-split layout: one
// thread-block cluster per particle, one thread per node for the update.  An
// odd node count runs as N + 1 nodes: the padding node has a zero SC row and
// column (it neither drives nor feels the network), zero weights, its own
// column of the noise table, no part in the FIC decision and no outputs; the
// real nodes' results are those of the unpadded system.
//
// Same model, time loop, FIC restarts, BOLD and extended outputs as the
// reference's bnm kernel (bnm.cu:72-315) and CPU path (bnm.cpp:167-290), and
// the same arithmetic as integrate_fast.cu / integrate_cluster.cu; the
// cluster protocol (S_E exchange by st.async on mbarriers, noise ring,
// cluster-uniform flags) is the one of integrate_cluster.cu.  What differs is
// the coupling mat-vec:
//   * CTA rank c owns nodes [c R, c R + R) (R <= 32 RPL).  Warp w owns the
//     column block [2 K2 w, 2 K2 (w+1)) of all R rows; lane l holds rows
//     l, l + 32, ... (RPL of them) as column pairs for fma.rn.f32x2, the first
//     KRP pairs in registers and the rest in shared memory;
//   * every lane of a warp reads the same S_E pairs (broadcast loads), forms
//     RPL partial row sums with no shuffles, and stores them to a [warp][row]
//     table; after one barrier thread t < R adds the W partials of row t and
//     updates node r0 + t alone (the row-split layout updates each node in
//     32/RPW lanes);
//   * one CTA barrier per substep, between partials and sums: each thread
//     waits for the S_E buffer on its mbarrier itself and the partial table
//     alternates with the substep, so nothing else needs the whole block;
//   * a cluster of one CTA (N up to 32 RPL, all of SC in registers) skips the
//     asynchronous exchange: owners store S_E straight into the other buffer
//     and a second barrier at the start of the next substep orders it (the
//     buffer being written was last read before the partial-table barrier of
//     the previous substep).
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
// collects at most kAgreeMs * 5 * 4 N P bytes of negative tx-count per
// barrier (P particles per cluster; N <= 1024, P = 2: 655360), inside the
// mbarrier's 2^20 - 1 range.
constexpr int kAgreeMs = 16;

// Shared-memory layout (bytes), in this order:
//   S      [2][P][2 K2 W] float          S_E of every node, double buffered, per particle
//   red    [2][P][W][32 RPL] float       per-warp partial row sums, by substep parity
//   SCs    [W][RPL][K2-KRP][32] float2   shared-memory part of the SC slice
//   ring   [kRing][10][R] float2         noise of the own nodes, per millisecond
//   ext    [P][6][32 RPL] double         extended-output sums of the own nodes
//   flags  [48] int                      late[2][8], fic[P][8], issue
//   mbar   [kRing + 2] uint64            noise stages, then S_E buffers 0 and 1
template <int RPL, int K2, int KRP, int P>
struct ColLayout {
    static constexpr int kRP = 32 * RPL;
    __host__ __device__ static size_t red_off(int W) { return (size_t)2 * P * W * 2 * K2 * sizeof(float); }
    __host__ __device__ static size_t sc_off(int W) { return red_off(W) + (size_t)2 * P * W * kRP * sizeof(float); }
    __host__ __device__ static size_t ring_off(int W) {
        return sc_off(W) + (size_t)W * RPL * (K2 - KRP) * 32 * sizeof(float2);
    }
    __host__ __device__ static size_t ext_off(int W, int R) { return ring_off(W) + (size_t)kRing * 10 * R * sizeof(float2); }
    __host__ __device__ static size_t flags_off(int W, int R) {
        return ext_off(W, R) + (size_t)P * 6 * kRP * sizeof(double);
    }
    __host__ __device__ static size_t mbar_off(int W, int R) { return flags_off(W, R) + 48 * sizeof(int); }
    __host__ __device__ static size_t bytes(int W, int R) { return mbar_off(W, R) + (kRing + 2) * sizeof(uint64_t); }
};
constexpr int kFicFlags = 16, kIssueFlag = 40;  // flags[16 + 8 p + rank], flags[40]

// P particles per cluster (1 or 2).  With P = 2 the two particles share the
// SC slice in registers: every warp forms the partial sums of both from one
// pass over its columns, and the two halves of the block update one particle
// each (thread t of half h owns node r0 + t of particle 2 c + h, c the
// cluster index).  The two particles advance in lockstep and read the same
// noise (every particle reads the same stream, bnm.cu:202-205): when either
// one's FIC check asks for a restart, both restart.  A particle that did not
// ask keeps its wIE, trial count and FIC state, and its rerun from
// millisecond 0 repeats its trajectory bit for bit (same state, noise and
// arithmetic), so its results are those of a run alone.  An odd batch leaves
// the last cluster's second half on a copy of the first particle, with no
// outputs written.
template <int RPL, int K2, int KRP, int P>
__global__ void integrate_colsplit_kernel(SimArgs a, int R) {
    static_assert(RPL >= 1 && RPL <= 8, "RPL");
    static_assert(KRP >= 0 && KRP <= K2, "KRP");
    static_assert(P == 1 || P == 2, "P");
    constexpr int KS = K2 - KRP;  // column pairs in shared memory
    constexpr int RP = 32 * RPL;
    typedef Model<float> C;
    typedef ColLayout<RPL, K2, KRP, P> L;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int N = a.N;
    const int W = blockDim.x >> 5;
    const int NC = 2 * K2 * W;  // padded column count
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, t = threadIdx.x;
    const uint32_t crank = cluster_rank(), csize = cluster_size();
    const int HB = (int)blockDim.x / P;         // threads per particle (the update roles)
    const int slot = P == 1 ? 0 : t / HB;       // particle of the cluster this thread updates
    const int tu = P == 1 ? t : t - slot * HB;  // own node index of this thread
    const int sim_raw = (int)(blockIdx.x / csize) * P + slot;
    const bool live = P == 1 || sim_raw < a.n_sims;
    // with a placement order, cluster c integrates particles order[P c ..]: the
    // order lists them by predicted work, so the particles a cluster advances
    // in lockstep need about the same number of substeps
    const int sim = a.order ? a.order[live ? sim_raw : sim_raw - slot] : (live ? sim_raw : sim_raw - slot);
    const int r0 = (int)crank * R;
    const int r_own = max(0, min(N - r0, R));  // nodes this CTA updates
    const int upd_warps = (r_own + 31) >> 5;    // warps (per particle) holding node owners

    float* S_buf = reinterpret_cast<float*>(smem_raw);
    float* red = reinterpret_cast<float*>(smem_raw + L::red_off(W));
    float2* SCs = reinterpret_cast<float2*>(smem_raw + L::sc_off(W));
    float2* ring = reinterpret_cast<float2*>(smem_raw + L::ring_off(W));
    double* ext_all = reinterpret_cast<double*>(smem_raw + L::ext_off(W, R));
    double* ext = ext_all + (size_t)slot * 6 * RP;  // this thread's particle
    int* flags = reinterpret_cast<int*>(smem_raw + L::flags_off(W, R));
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + L::mbar_off(W, R));

    const int node = r0 + tu;
    const int NR = a.n_real;      // nodes of the simulation: an odd count runs with one padding node
    const bool act = tu < r_own;  // thread owns node r0 + tu of its particle
    const bool real = act && node < NR;  // ... a node of the simulation (not the padding node)
    const bool wr = real && live;  // ... and writes its outputs
    const bool solo = csize == 1;  // S_E exchange through local shared memory
    const long long kSpin = kWaitNs;  // wall-clock limit of each bounded wait

    cluster_sync();  // every CTA of the cluster runs before any distributed shared memory access
    if (t == 0) {
        for (int b = 0; b < kRing + 2; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar + b)) : "memory");
        // buffer 1 receives S_E after the first substep: P N values of 4 bytes
        if (!solo)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar + kRing + 1)),
                         "r"(4 * N * P)
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = t; k < 2 * P * NC; k += blockDim.x) S_buf[k] = (k % NC) < N ? 0.001f : 0.f;
    for (int k = t; k < P * 6 * RP; k += blockDim.x) ext_all[k] = 0.0;
    for (int k = t; k < 48; k += blockDim.x) flags[k] = 0;

    // SC slice: rows r0 + lane + 32 i, column pairs 2 K2 w + 2 j (+1); zero outside the matrix
    float2 scr[RPL][KRP > 0 ? KRP : 1];
#pragma unroll
    for (int i = 0; i < RPL; i++) {
        const int row = lane + 32 * i;
#pragma unroll
        for (int j = 0; j < K2; j++) {
            const int col = 2 * K2 * w + 2 * j;
            float va = 0.f, vb = 0.f;
            if (row < r_own) {
                const float* src = a.sc_f32 + (size_t)(r0 + row) * a.sc_ld;
                if (col < N) va = src[col];
                if (col + 1 < N) vb = src[col + 1];
            }
            if (j < KRP)
                scr[i][j < KRP ? j : 0] = make_float2(va, vb);
            else
                SCs[((size_t)(w * RPL + i) * KS + (j - KRP)) * 32 + lane] = make_float2(va, vb);
        }
    }
    cluster_sync();  // buffers initialised in every CTA before anyone writes remote S_E

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

    const float GJ = (float)a.G[sim] * C::J_NMDA;
    // the padding node (zero SC row and column) integrates with zero weights and takes no part in FIC
    const float wEE = real ? (float)a.wEE[(size_t)sim * NR + node] : 0.f;
    const float wEI = real ? (float)a.wEI[(size_t)sim * NR + node] : 0.f;
    float wIE = real ? (float)a.wIE[(size_t)sim * NR + node] : 0.f;
    float delta = (float)a.init_delta;
    float S_E = 0.001f, S_I = 0.001f, IE = 0.f, II = 0.f, rE = 0.f, rI = 0.f;
    double mean_IE = 0.0;
    BW bw;
    // time and copies are shared by the cluster's particles; the FIC state is per particle
    int ts = 0, frame = 0, to_frame = 1, ms_next = 0;
    int trial[P];
    bool failed[P], adj[P];
#pragma unroll
    for (int p = 0; p < P; p++) {
        trial[p] = 0;
        failed[p] = false;
        adj[p] = a.adjust_fic != 0;
    }
    bool adjusting = a.adjust_fic != 0, timed_out = false;
    uint32_t c_cons = 0, c_issue = 0;
    int cur = 0;
    // S_E exchange as in integrate_cluster.cu: buffer b's mbarrier completes a
    // phase when all P N values of the next S_E have landed; ph bit b is the
    // parity this CTA waits for next; buffer 0 starts filled locally
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
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(10 * run_bytes)
                         : "memory");
            for (int sub = 0; sub < 10; sub++)
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_addr(ring + ((size_t)st * 10 + sub) * R)),
                    "l"(noise_bytes + (((size_t)ms_next * 10 + sub) * N + r0) * sizeof(float2)), "r"(run_bytes),
                    "r"(bar)
                    : "memory");
            c_issue++;
            ms_next++;
        }
    };
    // flags[base + 8 p + crank] of every CTA <- v_p (thread p csize + r writes rank r)
    auto broadcast_flags = [&](int base, bool v0, bool v1) {
        if (solo) {
            if (t < P) flags[base + 8 * t] = (t ? v1 : v0) ? 1 : 0;
        } else if (t < P * (int)csize) {
            const int p = t / (int)csize;
            st_cluster_s32(map_rank(flags_local + 4u * (base + 8 * p + (int)crank), (uint32_t)(t - p * (int)csize)),
                           (p ? v1 : v0) ? 1 : 0);
        }
    };
    // cluster-wide agreement point: a one-CTA cluster needs only a block
    // barrier (no release fence at cluster scope)
    auto agree = [&]() {
        if (solo)
            __syncthreads();
        else
            cluster_sync();
    };

    bool late = false;  // sticky; block-uniform after each __syncthreads_or
    int since_agree = 0, n_agree = 0;
    while (ts <= a.T) {
        if (a.noise) {
            if (t == 0 && !late) issue();
            late = __syncthreads_or(late || !wait_copy(c_cons));
        } else {  // Philox noise drawn by the block instead of copied from a table
            philox_fill_stage(ring + (size_t)(c_cons % kRing) * 10 * R, R, r0, r_own, a.n_real, ts, key0, key1);
            late = __syncthreads_or(late);
        }
        const float2* nz = ring + (size_t)(c_cons % kRing) * 10 * R + (act ? tu : 0);

#pragma unroll 1
        for (int sub = 0; sub < 10; sub++) {
            if (!solo && !skip_wait && !late) late = !wait_s(cur);
            skip_wait = false;
            // A one-CTA cluster stored S_E locally: a block barrier orders those
            // stores before the reads below.  A cluster of several CTAs needs
            // none here: every thread waited on buffer cur's mbarrier itself;
            // the next phase of that buffer (S_E two substeps on) cannot
            // complete, nor land in the buffer, before the other CTAs have this
            // CTA's next S_E, which is sent after the block barrier below, when
            // every thread has read buffer cur and passed this wait; and the
            // partial table alternates with the substep, so this substep's
            // partials never overwrite ones a slower thread is still adding.
            if (solo) __syncthreads();
            if (!solo && t == 0 && !late)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sbar_local + 8u * cur),
                             "r"(4 * N * P)
                             : "memory");
            float2 acc[P][RPL];
#pragma unroll
            for (int p = 0; p < P; p++)
#pragma unroll
                for (int i = 0; i < RPL; i++) acc[p][i] = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < K2; j++) {
                float2 s2[P];  // same address in every lane: broadcast
#pragma unroll
                for (int p = 0; p < P; p++)
                    s2[p] = reinterpret_cast<const float2*>(S_buf + (cur * P + p) * NC + 2 * K2 * w)[j];
#pragma unroll
                for (int i = 0; i < RPL; i++) {
                    const float2 m = (j < KRP) ? scr[i][j < KRP ? j : 0]
                                               : SCs[((size_t)(w * RPL + i) * KS + (j - KRP)) * 32 + lane];
#pragma unroll
                    for (int p = 0; p < P; p++) acc[p][i] = __ffma2_rn(m, s2[p], acc[p][i]);
                }
            }
#pragma unroll
            for (int p = 0; p < P; p++)
#pragma unroll
                for (int i = 0; i < RPL; i++)
                    red[((cur * P + p) * W + w) * RP + lane + 32 * i] = acc[p][i].x + acc[p][i].y;
            __syncthreads();
            if ((tu >> 5) < upd_warps) {
                const float* rp = red + (cur * P + slot) * W * RP + tu;
                float coupling = 0.f;
                for (int w2 = 0; w2 < W; w2++) coupling += rp[w2 * RP];
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
                const int dst_idx = ((cur ^ 1) * P + slot) * NC + node;
                if (act && solo) {
                    S_buf[dst_idx] = S_E;
                } else if (act) {  // to buffer cur^1 of every CTA; its mbarrier counts the bytes
                    const uint32_t dst = s_local + (uint32_t)(dst_idx * sizeof(float));
                    const uint32_t bar = sbar_local + 8u * (cur ^ 1);
                    for (uint32_t r = 0; r < csize; r++) st_async_f32(map_rank(dst, r), S_E, map_rank(bar, r));
                }
            }
            cur ^= 1;
        }
        // a late noise copy or S_E exchange anywhere stops the whole cluster at
        // the next agreement point (ts, adjusting and the counters are the
        // same in every CTA, so all of them stop here together)
        if (++since_agree == kAgreeMs || ts == a.T || (adjusting && ts + 1 == a.samp_end)) {
            since_agree = 0;
            const int lslot = (n_agree++ & 1) * 8;
            const bool lt_blk = __syncthreads_or(late);
            if (solo) {
                if (t == 0) flags[lslot] = lt_blk ? 1 : 0;
            } else if (t < (int)csize) {
                st_cluster_s32(map_rank(flags_local + 4u * (lslot + (int)crank), (uint32_t)t), lt_blk ? 1 : 0);
            }
            agree();
            bool any_late = false;
            for (uint32_t r = 0; r < csize; r++) any_late |= flags[lslot + r] != 0;
            if (any_late) {
                timed_out = true;
                break;
            }
        }
        c_cons++;
        bw.step(S_E);
        if (--to_frame == 0) {  // ts % TR == 0
            to_frame = a.TR;
            if (act) {
                if (wr) a.bold[((size_t)sim * a.frames + frame) * NR + node] = bw.bold();
                if (frame >= a.n_vols_remove) {
                    double* e = ext + tu;
                    e[0 * RP] += S_E;
                    e[1 * RP] += IE;
                    e[2 * RP] += rE;
                    e[3 * RP] += S_I;
                    e[4 * RP] += II;
                    e[5 * RP] += rI;
                }
            }
            frame++;
        }
        ts++;
        if (adjusting) {
            if (ts >= a.samp_start && ts <= a.samp_end) mean_IE += (double)IE;
            if (ts == a.samp_end) {
                const bool my_adj = P == 1 ? adj[0] : (slot ? adj[P - 1] : adj[0]);
                const int my_trial = P == 1 ? trial[0] : (slot ? trial[P - 1] : trial[0]);
                bool needs = false;
                if (real && my_adj) {
                    const double diff = mean_IE / duration - (double)C::b_a_ratio_E;
                    if (fabs(diff + 0.026) > 0.005) {
                        needs = true;
                        if (my_trial < a.max_trials) {
                            if (diff < -0.026) {
                                wIE -= delta;
                                delta = fmaxf(delta - 0.001f, 0.001f);
                            } else {
                                wIE += delta;
                            }
                        }
                    }
                }
                const bool blk0 = __syncthreads_or(needs && slot == 0);
                const bool blk1 = P == 2 ? __syncthreads_or(needs && slot == 1) : false;
                broadcast_flags(kFicFlags, blk0, blk1);
                agree();
                bool restart = false;
#pragma unroll
                for (int p = 0; p < P; p++) {
                    bool any = false;
                    for (uint32_t r = 0; r < csize; r++) any |= flags[kFicFlags + 8 * p + r] != 0;
                    if (!adj[p]) continue;
                    if (!any) {
                        adj[p] = false;
                    } else if (trial[p] < a.max_trials) {
                        restart = true;
                        trial[p]++;
                    } else {
                        failed[p] = true;
                        adj[p] = false;
                    }
                }
                adjusting = false;
#pragma unroll
                for (int p = 0; p < P; p++) adjusting |= adj[p];
                if (restart) {
                    S_E = S_I = 0.001f;
                    bw = BW();
                    mean_IE = 0.0;
                    if (act)
                        for (int e = 0; e < 6; e++) ext[e * RP + tu] = 0.0;
                    // the S_E the next substep would read is in flight: let it land,
                    // then overwrite the buffer locally with the restart state
                    bool lt = false;
                    if (!solo) {
                        lt = !wait_s(cur);
                        skip_wait = true;
                    }
                    __syncthreads();
#pragma unroll
                    for (int p = 0; p < P; p++)
                        for (int k = t; k < N; k += blockDim.x) S_buf[(cur * P + p) * NC + k] = 0.001f;
                    ts = 0;
                    frame = 0;
                    to_frame = 1;
                    // copies in flight hold milliseconds after the restart point:
                    // let them land, then refetch from millisecond 0 (thread 0
                    // issues, so it publishes how far it got)
                    if (t == 0) flags[kIssueFlag] = (int)c_issue;
                    __syncthreads();
                    const uint32_t in_flight_end = (uint32_t)flags[kIssueFlag];
                    for (; c_cons < in_flight_end; c_cons++) lt |= !wait_copy(c_cons);
                    ms_next = 0;
                    if (lt && t == 0) atomicOr(a.status, kStatusTimeout);
                }
                agree();  // fic flags may be rewritten only after every CTA read them
            }
        }
    }
    if (!timed_out && wr) {
        a.wIE_out[(size_t)sim * NR + node] = (double)wIE;
        const double kept = (double)(frame - a.n_vols_remove);
        for (int e = 0; e < 6; e++) a.ext[((size_t)sim * 6 + e) * NR + node] = ext[e * RP + tu] / kept;
    }
    if (!timed_out && crank == 0 && tu == 0 && live) {
        a.trials[sim] = P == 1 ? trial[0] : (slot ? trial[P - 1] : trial[0]);
        a.failed[sim] = (P == 1 ? failed[0] : (slot ? failed[P - 1] : failed[0])) ? 1 : 0;
    }
    if (timed_out) {
        if (t == 0) {
            atomicOr(a.status, kStatusTimeout);
            // own copies land before exit: once a wait ran out no copy was
            // issued, so only the last one of each ring stage can be in flight
            for (uint32_t c = c_issue > (uint32_t)kRing ? c_issue - kRing : 0; c < c_issue; c++) wait_copy(c);
        }
        __syncthreads();
    }
    // the S_E sent at the last substep lands before anyone leaves: no CTA
    // exits while another may still write its shared memory
    if (!solo && !skip_wait) wait_s(cur);
    cluster_sync();
}

// ---------------------------------------------------------------- launch

struct Variant {
    int rpl, k2, krp, np;
    const void* fn;
    size_t (*bytes)(int W, int R);
};

template <int RPL, int K2, int KRP, int P = 1>
Variant make_variant() {
    return {RPL, K2, KRP, P, (const void*)&integrate_colsplit_kernel<RPL, K2, KRP, P>,
            &ColLayout<RPL, K2, KRP, P>::bytes};
}

// One particle per cluster: rows per lane 2 or 4; column pairs per warp 8,
// 10, 13, 16, 25; all pairs in registers, or 8 in registers and the rest in
// shared memory.  Plus row-heavy shapes with all of SC in registers for
// one-CTA clusters up to N = 160 / 192 / 208 (5, 6, 7 rows per lane).  Two
// particles per cluster: the same column blocks with the two particles'
// partial sums sharing the SC registers (also with fewer pairs in registers,
// which leaves room for the second particle's accumulators).
#define BNM_V(K2)                                                                                        \
    make_variant<2, K2, K2>(), make_variant<4, K2, K2>(), make_variant<2, K2, (K2 < 8 ? K2 : 8)>(), \
        make_variant<4, K2, (K2 < 8 ? K2 : 8)>()
const std::vector<Variant>& variants() {
    static const std::vector<Variant> v = {
        BNM_V(8), BNM_V(10), BNM_V(13), BNM_V(16), BNM_V(25), make_variant<5, 10, 10>(), make_variant<6, 12, 12>(),
        make_variant<7, 13, 13>(),
        // N above 512 (76 to 96 rows per CTA of an 8-CTA cluster): 3 or 4 rows per
        // lane, 25 column pairs per warp, 12 or 16 of them in registers
        make_variant<3, 25, 16>(), make_variant<3, 25, 12>(), make_variant<4, 25, 12>(),
        // two particles per cluster
        make_variant<2, 10, 10, 2>(), make_variant<4, 10, 10, 2>(), make_variant<2, 13, 13, 2>(),
        make_variant<4, 13, 13, 2>(), make_variant<2, 16, 16, 2>(), make_variant<4, 16, 16, 2>(),
        make_variant<2, 25, 25, 2>(), make_variant<4, 25, 25, 2>(), make_variant<4, 25, 20, 2>(),
        make_variant<4, 25, 16, 2>()};
    return v;
}
#undef BNM_V

const Variant* find(int rpl, int k2, int krp, int np) {
    for (const Variant& v : variants())
        if (v.rpl == rpl && v.k2 == k2 && v.krp == krp && v.np == np) return &v;
    return nullptr;
}

}  // namespace
}  // namespace bnm

using namespace bnm;

// Checks one column-split configuration for node count N: rows per CTA R
// (even, at most 32 RPL, with a node in every rank), warps W = N / (2 K2)
// rounded up (at least R threads per particle; with two particles an even W
// so that each half of the block is whole warps), the kernel's own
// block-size limit and shared memory.  Returns 1 and the launch shape when it
// can run.
extern "C" int bnm_colsplit_shape(int N, int csize, int rpl, int k2, int krp, int np, int* threads, int* rows,
                                  size_t* smem) {
    if (N <= 0 || N > 1024 || (N & 1) || csize < 1 || csize > 8) return 0;
    const Variant* v = find(rpl, k2, krp, np);
    if (!v) return 0;
    int R = (N + csize - 1) / csize;
    R += R & 1;  // bulk copies of the own nodes' noise need even node runs
    if (R > 32 * rpl || (csize - 1) * R >= N) return 0;
    const int W = (N + 2 * k2 - 1) / (2 * k2);
    if (W * 32 > 1024) return 0;
    if (np == 1 && W * 32 < R) return 0;
    if (np == 2 && ((W & 1) || W * 16 < R)) return 0;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, v->fn) != cudaSuccess) return 0;
    if (W * 32 > fa.maxThreadsPerBlock) return 0;
    const size_t sm = v->bytes(W, R);
    if (sm > 227 * 1024) return 0;
    *threads = W * 32;
    *rows = R;
    *smem = sm;
    return 1;
}

// The (rows per lane, column pairs per warp, pairs in registers, particles
// per cluster) variants built.
extern "C" int bnm_colsplit_variants(int* out4, int max) {
    int n = 0;
    for (const Variant& v : variants()) {
        if (n < max) {
            out4[4 * n] = v.rpl;
            out4[4 * n + 1] = v.k2;
            out4[4 * n + 2] = v.krp;
            out4[4 * n + 3] = v.np;
        }
        n++;
    }
    return n;
}

static void colsplit_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr, int clusters, int csize, int threads,
                            size_t smem) {
    std::memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3((unsigned)(clusters * csize));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
}

// Fraction of the GPU one launch of this shape fills: its clusters over the
// clusters that can be resident at once (1 when the query fails).
extern "C" double bnm_colsplit_share(int N, int csize, int rpl, int k2, int krp, int np, int n_sims) {
    int threads = 0, R = 0;
    size_t smem = 0;
    if (!bnm_colsplit_shape(N, csize, rpl, k2, krp, np, &threads, &R, &smem)) return 1.0;
    const Variant* v = find(rpl, k2, krp, np);
    const int needed = (n_sims + np - 1) / np;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    colsplit_config(cfg, attr, needed, csize, threads, smem);
    int clusters = 0;
    if (cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveClusters(&clusters, v->fn, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return 1.0;
    }
    return needed >= clusters ? 1.0 : (double)needed / clusters;
}

cudaError_t bnm_launch_integrate_colsplit(const SimArgs& a, int csize, int rpl, int k2, int krp, int np,
                                          cudaStream_t st) {
    int threads = 0, R = 0;
    size_t smem = 0;
    if (!bnm_colsplit_shape(a.N, csize, rpl, k2, krp, np, &threads, &R, &smem)) return cudaErrorInvalidValue;
    if (a.sc_ld < a.N) return cudaErrorInvalidValue;
    const Variant* v = find(rpl, k2, krp, np);
    cudaError_t e = cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    colsplit_config(cfg, attr, (a.n_sims + np - 1) / np, csize, threads, smem);
    cfg.stream = st;
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, v->fn, &cfg);
    if (e != cudaSuccess) return e;
    if (clusters < 1) return cudaErrorInvalidConfiguration;
    void* args[] = {(void*)&a, (void*)&R};
    return cudaLaunchKernelExC(&cfg, v->fn, args);
}
