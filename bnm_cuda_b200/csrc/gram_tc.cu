// FC and FCD Grams on the fifth-generation tensor cores (tcgen05.mma with the
// accumulator in tensor memory), BF16 or split-BF16 operands, FP32
// accumulation.
//
// Reference computations (CPU path, check_fit.cpp; GPU path, bnm.cu):
//   FC   Pearson of node BOLD series over the kept frames, pairs i > j
//        (check_fit.cpp:19-62; bold_stats + fc, bnm.cu:317-347, 382-434)
//   FCD  Pearson of window-FC vectors, windows a > b
//        (check_fit.cpp:110-134; window_fc_stats + fcd, bnm.cu:436-551)
// Both are Grams of rows that are centred and scaled to unit norm in FP64
// first: FC rows are nodes (K = kept frames), FCD rows are windows (K = pairs).
//
// Operands live in HBM already in the layout the tensor core reads from
// shared memory: tiles of 128 rows x 64 BF16 (16 KB), each row one 128-byte
// line whose 16-byte chunks are XOR-swizzled by row % 8 (the canonical
// K-major SWIZZLE_128B layout).  A tile therefore moves HBM -> shared memory
// with one bulk copy (cp.async.bulk on an mbarrier) and no tensor map.
// Split BF16 stores x = hi + lo, hi = bf16(x), lo = bf16(x - hi), and
// accumulates hi.hi + hi.lo + lo.hi; the dropped lo.lo term is ~2^-18 of a
// product, below FP32 rounding of the sum.
//
// gram_tc_kernel: one CTA (6 warps) per 128 x 128 lower-triangle output tile.
//   warp 4 lane 0   producer: K tiles through a ring of shared-memory stages
//   warp 5 lane 0   MMA issuer: 4 (12 split) tcgen05.mma of K = 16 per K tile;
//                   tcgen05.commit frees each stage once its MMAs have read it.
//                   Every 2 K tiles form a partial sum in one of two TMEM
//                   accumulators (double-buffered)
//   warps 0-3       drain each partial (tcgen05.ld; warp w owns TMEM lanes
//                   32w..32w+31 = tile rows) into FP32 registers while the
//                   next partial accumulates, then write the finished tile to
//                   shared memory for the epilogue
//   all 6 warps     epilogue: lower-triangle store (coalesced along rows) and,
//                   for FCD, the KS rank histogram of analysis.cu.
// Diagonal tiles load one operand and use it as both A and B.  Every wait is
// bounded; a timeout sets kStatusTimeout, stops the other roles through a
// shared flag, lets in-flight copies and MMAs finish (bounded again), frees
// tensor memory and returns.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "kernels.h"

namespace bnm {
namespace {

constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s; a stage normally lands in microseconds
constexpr uint32_t kTmemCols = 256;           // two 128 x 128 FP32 partial accumulators

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Parity wait on an mbarrier, bounded by kWaitNs of wall time; gives up early
// when *stop is set.
__device__ __noinline__ bool bar_wait(uint32_t bar, uint32_t parity, const volatile int* stop) {
    uint64_t t0 = 0;
    for (uint32_t i = 0;; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (stop && *stop) return false;
        if ((i & 63) == 0) {
            const uint64_t t = global_ns();
            if (i == 0)
                t0 = t;
            else if (t - t0 > kWaitNs)
                return false;
        }
    }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Shared-memory matrix descriptor of a K-major SWIZZLE_128B operand:
// start address >> 4 (bits 0-13); leading byte offset 1 (bits 16-29, unused
// by swizzled K-major layouts); stride byte offset 1024 B >> 4 between 8-row
// groups (bits 32-45); descriptor version 1 (bits 46-47); base offset 0, as
// every tile starts on a 1024-byte boundary; layout 2 = SWIZZLE_128B
// (bits 61-63).  Stepping K by 16 BF16 inside the 128-byte row adds 32 bytes
// to the start address; the swizzle is applied to the computed address.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, bits 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 (bits 17-22), M >> 4 (bits 24-28); M = N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

// Arrive on bar once every tcgen05 operation this thread issued so far is done.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

template <bool Split>
struct GramRing {
    static constexpr int kParts = Split ? 2 : 1;  // hi (+ lo) per operand
    static constexpr int kStages = Split ? 3 : 4;
    static constexpr int kStageBytes = 2 * kParts * kGramTileBytes;
    static constexpr int kRingBytes = kStages * kStageBytes;
    static constexpr int kTileLd = kGramTileRows + 1;  // padded FP32 output tile, reuses the ring
    static constexpr int kSmemBytes =
        (kRingBytes > kGramTileRows * kTileLd * 4 ? kRingBytes : kGramTileRows * kTileLd * 4) + 1024;
};

// K tiles per partial accumulator.  The tensor core's FP32 accumulation loses
// about half an ulp of the running sum per MMA, so long K chains (79,800 pairs
// is 4,988 MMAs) drift; partial sums over 128 K are drained into FP32
// registers, which bounds that loss by the partial's own size.
constexpr int kDrainTiles = 2;

template <bool Split>
__global__ void __launch_bounds__(192, 1) gram_tc_kernel(GramArgs a) {
    using R = GramRing<Split>;
    constexpr int kStages = R::kStages, kParts = R::kParts;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int stop, skip;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int t = blockIdx.x, ta = 0;  // lower-triangle tile (ta >= tb)
    while (t > ta) {
        t -= ta + 1;
        ta++;
    }
    const int tb = t, sim = blockIdx.y;
    const bool diag = ta == tb;
    const int groups = (a.kblocks + kDrainTiles - 1) / kDrainTiles;
    // stages start on a 1024-byte boundary of the shared address space
    const uint32_t raw = saddr(smem_raw);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
    const uint32_t ring = raw + pad;

    // once any CTA has timed out the rest return at once (before taking tensor memory)
    if (threadIdx.x == 0) skip = *(volatile int*)a.status & kStatusTimeout;
    __syncthreads();
    if (skip) return;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&empty[s])) : "memory");
        }
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&acc_full[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(saddr(&acc_empty[b])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&done)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        stop = 0;
    }
    if (warp == 0) {  // warp-wide allocation; the address lands in tmem_slot
        __syncwarp();
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    volatile int* vstop = &stop;
    auto give_up = [&]() {
        atomicOr(a.status, kStatusTimeout);
        *vstop = 1;
    };

    float acc[kGramTileRows];  // drain warps: this thread's tile row, summed over partials
    if (warp == 4) {
        if (lane == 0) {  // producer
            const size_t tile_a = ((size_t)sim * a.row_blocks + ta) * a.kblocks;
            const size_t tile_b = ((size_t)sim * a.row_blocks + tb) * a.kblocks;
            const uint32_t bytes = (uint32_t)((diag ? 1 : 2) * kParts * kGramTileBytes);
            int issued = 0;
            for (int kb = 0; kb < a.kblocks; kb++) {
                const int s = kb % kStages;
                if (kb >= kStages && !bar_wait(saddr(&empty[s]), ((kb / kStages) - 1) & 1, vstop)) {
                    give_up();
                    break;
                }
                const uint32_t fb = saddr(&full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(bytes)
                             : "memory");
                const uint32_t st = ring + (uint32_t)(s * R::kStageBytes);
                bulk_g2s(st, a.hi + (tile_a + kb) * kGramTileBytes, kGramTileBytes, fb);
                if (Split) bulk_g2s(st + kGramTileBytes, a.lo + (tile_a + kb) * kGramTileBytes, kGramTileBytes, fb);
                if (!diag) {
                    const uint32_t sb = st + kParts * kGramTileBytes;
                    bulk_g2s(sb, a.hi + (tile_b + kb) * kGramTileBytes, kGramTileBytes, fb);
                    if (Split) bulk_g2s(sb + kGramTileBytes, a.lo + (tile_b + kb) * kGramTileBytes, kGramTileBytes, fb);
                }
                issued++;
            }
            // copies still in flight land before the CTA's shared memory is reused or freed
            for (int kb = issued > kStages ? issued - kStages : 0; kb < issued; kb++)
                bar_wait(saddr(&full[kb % kStages]), (kb / kStages) & 1, nullptr);
        }
        __syncwarp();
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer: group g accumulates K tiles [g*D, g*D+D) into buffer g % 2
            bool failed = false;
            for (int g = 0; g < groups && !failed; g++) {
                const int b = g & 1;
                if (g >= 2 && !bar_wait(saddr(&acc_empty[b]), ((g >> 1) - 1) & 1, vstop)) {
                    give_up();
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * kGramTileRows);
                const int kb_end = min(a.kblocks, (g + 1) * kDrainTiles);
                for (int kb = g * kDrainTiles; kb < kb_end; kb++) {
                    const int s = kb % kStages;
                    if (!bar_wait(saddr(&full[s]), (kb / kStages) & 1, vstop)) {
                        give_up();
                        failed = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = ring + (uint32_t)(s * R::kStageBytes);
                    const uint32_t a_hi = st, a_lo = st + kGramTileBytes;
                    const uint32_t b_hi = diag ? a_hi : st + kParts * kGramTileBytes;
                    const uint32_t b_lo = diag ? a_lo : b_hi + kGramTileBytes;
                    const bool first = kb == g * kDrainTiles;
#pragma unroll
                    for (int ks = 0; ks < kGramTileK / 16; ks++) {
                        const uint32_t off = 32u * ks;
                        mma_bf16(d, sw128_desc(a_hi + off), sw128_desc(b_hi + off), !(first && ks == 0));
                        if (Split) {
                            mma_bf16(d, sw128_desc(a_hi + off), sw128_desc(b_lo + off), 1u);
                            mma_bf16(d, sw128_desc(a_lo + off), sw128_desc(b_hi + off), 1u);
                        }
                    }
                    mma_commit(saddr(&empty[s]));
                }
                if (!failed) mma_commit(saddr(&acc_full[b]));
            }
            mma_commit(saddr(&done));  // arrives when every MMA above has completed
        }
        __syncwarp();
    } else {  // warps 0-3 drain TMEM lanes 32w..32w+31 (tile rows) after every group
#pragma unroll
        for (int j = 0; j < kGramTileRows; j++) acc[j] = 0.f;
        for (int g = 0; g < groups; g++) {
            const int b = g & 1;
            const bool ok = bar_wait(saddr(&acc_full[b]), (g >> 1) & 1, vstop);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) give_up();
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int c = 0; c < kGramTileRows / 32; c++) {
                float v[32];
                tmem_load32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(b * kGramTileRows + 32 * c), v);
#pragma unroll
                for (int j = 0; j < 32; j++) acc[32 * c + j] += v[j];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(&acc_empty[b])) : "memory");
        }
    }

    // every MMA has completed (or the wait gave up) before the ring is reused
    const bool ok = bar_wait(saddr(&done), 0, nullptr);
    if (__syncthreads_or(!ok || *vstop)) {
        if (threadIdx.x == 0) atomicOr(a.status, kStatusTimeout);
        if (!ok) bar_wait(saddr(&done), 0, nullptr);  // outstanding MMAs still write tensor memory
    } else {
        // ---- epilogue: row sums -> padded shared tile -> lower triangle / KS histogram ----
        float* tile = reinterpret_cast<float*>(smem_raw + pad);
        if (warp < 4) {
            float* row = tile + (32 * warp + lane) * R::kTileLd;
#pragma unroll
            for (int j = 0; j < kGramTileRows; j++) row[j] = acc[j];
        }
        __syncthreads();
        const int a0 = ta * kGramTileRows, b0 = tb * kGramTileRows;
        bool any_nan = false;
        unsigned int* hist = a.hist ? a.hist + (size_t)sim * (a.m + 1) : nullptr;
        unsigned int* eq = a.hist ? a.eq + (size_t)sim * (a.m + 1) : nullptr;
        float* out = a.out ? a.out + (size_t)sim * a.out_ld : nullptr;
        // consecutive threads take consecutive columns of a row: coalesced stores
        for (int e = threadIdx.x; e < kGramTileRows * kGramTileRows; e += blockDim.x) {
            const int r = e / kGramTileRows, j = e % kGramTileRows;
            const int wa = a0 + r, wb = b0 + j;
            if (wa >= a.rows || wb >= wa) continue;
            const float x = tile[r * R::kTileLd + j];
            if (!(x == x) || isinf(x)) {
                any_nan = true;
                continue;
            }
            if (out) {
                const long long idx = (long long)wa * (wa - 1) / 2 + wb;
                const long long o = a.tril_map ? a.tril_map[idx] : idx;
                if (o >= 0) out[o] = x;
            }
            if (hist) {
                int c;
                bool equal;
                if (a.ks_lut)
                    ks_bucket_lut(a.emp_sorted, a.ks_lut, a.m, (double)x, c, equal);
                else
                    ks_bucket(a.emp_sorted, a.m, (double)x, c, equal);
                atomicAdd(&hist[c], 1u);
                if (equal) atomicAdd(&eq[c], 1u);
            }
        }
        if (any_nan) atomicOr(&a.nan_flag[sim], 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// ------------------------------------------------------------ operands

// byte offset of (row r, 16-byte chunk c) inside a tile: SWIZZLE_128B
__device__ __forceinline__ uint32_t tile_offset(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 x, __nv_bfloat16 y) {
    return (uint32_t)__bfloat16_as_ushort(x) | ((uint32_t)__bfloat16_as_ushort(y) << 16);
}

// Writes 8 consecutive K values of one row as hi (and lo) BF16 chunks.
__device__ __forceinline__ void store_chunk(const OperandArgs& a, int sim, int row, int chunk, const float (&x)[8]) {
    __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        h[e] = __float2bfloat16_rn(x[e]);
        l[e] = __float2bfloat16_rn(x[e] - __bfloat162float(h[e]));
    }
    const size_t tile = ((size_t)sim * a.row_blocks + row / kGramTileRows) * a.kblocks + chunk / 8;
    const size_t off = tile * kGramTileBytes + tile_offset(row % kGramTileRows, chunk % 8);
    *reinterpret_cast<uint4*>(a.hi + off) =
        make_uint4(pack2(h[0], h[1]), pack2(h[2], h[3]), pack2(h[4], h[5]), pack2(h[6], h[7]));
    if (a.lo)
        *reinterpret_cast<uint4*>(a.lo + off) =
            make_uint4(pack2(l[0], l[1]), pack2(l[2], l[3]), pack2(l[4], l[5]), pack2(l[6], l[7]));
}

// FCD rows: window a of a simulation, z = (wfc - mean) / ||wfc - mean|| over
// pairs with FP64 centring (same normalisation as fcd_gram_kernel).
// grid (row_blocks * 128, n_sims); padding rows and K are zero.
__global__ void __launch_bounds__(256) fcd_operand_kernel(OperandArgs a) {
    const int row = blockIdx.x, sim = blockIdx.y;
    const bool valid = row < a.rows;
    double mean = 0.0, inv = 0.0;
    if (valid) window_norm(a.wsum + ((size_t)sim * a.rows + row) * 2, a.K, mean, inv);
    const float* src = a.wfc + ((size_t)sim * a.rows + (valid ? row : 0)) * a.K;
    for (int ch = threadIdx.x; ch < a.kblocks * 8; ch += blockDim.x) {
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int k = ch * 8 + e;
            x[e] = (valid && k < a.K) ? (float)(((double)src[k] - mean) * inv) : 0.f;
        }
        store_chunk(a, sim, row, ch, x);
    }
}

__device__ double block_sum256(double v, double* sh) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    return s;
}

// FC rows: node i's BOLD over the kept frames, centred on its FP64 mean and
// scaled by 1 / sqrt(sum of squared deviations) (bold_stats, bnm.cu:317-347).
// grid (row_blocks * 128, n_sims).
template <typename TB>
__global__ void __launch_bounds__(256) fc_operand_kernel(OperandArgs a, const TB* __restrict__ bold) {
    __shared__ double sh[8];
    const int row = blockIdx.x, sim = blockIdx.y;
    const bool valid = row < a.rows;
    const int N = a.rows, L = a.K;
    const TB* src = bold + ((size_t)sim * a.frames + a.n_vols_remove) * N + (valid ? row : 0);
    double mean = 0.0, inv = 0.0;
    if (valid) {  // block-uniform
        double s = 0.0;
        for (int t = threadIdx.x; t < L; t += blockDim.x) s += (double)src[(size_t)t * N];
        mean = block_sum256(s, sh) / L;
        double ss = 0.0;
        for (int t = threadIdx.x; t < L; t += blockDim.x) {
            const double d = (double)src[(size_t)t * N] - mean;
            ss += d * d;
        }
        inv = 1.0 / sqrt(block_sum256(ss, sh));
    }
    for (int ch = threadIdx.x; ch < a.kblocks * 8; ch += blockDim.x) {
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int t = ch * 8 + e;
            x[e] = (valid && t < L) ? (float)(((double)src[(size_t)t * N] - mean) * inv) : 0.f;
        }
        store_chunk(a, sim, row, ch, x);
    }
}

}  // namespace
}  // namespace bnm

using namespace bnm;

cudaError_t bnm_launch_fcd_operand(const OperandArgs& a, cudaStream_t st) {
    if (a.row_blocks * kGramTileRows < a.rows || a.kblocks * kGramTileK < a.K) return cudaErrorInvalidValue;
    dim3 grid(a.row_blocks * kGramTileRows, a.n_sims);
    fcd_operand_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t bnm_launch_fc_operand(const OperandArgs& a, cudaStream_t st) {
    if (a.row_blocks * kGramTileRows < a.rows || a.kblocks * kGramTileK < a.K) return cudaErrorInvalidValue;
    dim3 grid(a.row_blocks * kGramTileRows, a.n_sims);
    if (a.bold_f64)
        fc_operand_kernel<double><<<grid, 256, 0, st>>>(a, a.bold_f64);
    else
        fc_operand_kernel<float><<<grid, 256, 0, st>>>(a, a.bold);
    return cudaGetLastError();
}

template <bool Split>
static cudaError_t launch_gram(const GramArgs& a, cudaStream_t st) {
    constexpr int smem = GramRing<Split>::kSmemBytes;
    cudaError_t e = cudaFuncSetAttribute(gram_tc_kernel<Split>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.row_blocks * (a.row_blocks + 1) / 2, a.n_sims);
    gram_tc_kernel<Split><<<grid, 192, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t bnm_launch_gram_tc(const GramArgs& a, int split, cudaStream_t st) {
    if (a.kblocks < 1 || a.row_blocks < 1 || a.row_blocks * kGramTileRows < a.rows || (split && !a.lo))
        return cudaErrorInvalidValue;
    // bulk copies need 16-byte aligned global sources
    if (((uintptr_t)a.hi | (uintptr_t)a.lo) & 15) return cudaErrorInvalidValue;
    return split ? launch_gram<true>(a, st) : launch_gram<false>(a, st);
}
