// Argument blocks and launchers of the device stages (shared by the .cu files
// and the plan code in capi.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "bnm_common.cuh"

namespace bnm {

struct FcArgs {
    int N, n_sims, frames, n_vols_remove, corr_len;
    int P;                    // pairs
    const int* pair_i;        // [P]
    const int* pair_j;        // [P]
    int W, win_len, win_step; // windows: start k*step, length win_len (relative to first kept frame)
    const float* bold;        // [n][frames][N] (FP32 integrators)
    const double* bold_f64;   // [n][frames][N] (FP64 integrator); exactly one is set
    float* fc;                // [n][P]
    float* wfc;               // [n][W][P] raw window FC
    double* wsum;             // [n][W][2] sum, sum of squares over pairs (written after the window FC)
    int* nan_flag;            // [n]
    int ppt;                  // pairs per thread: a CTA of 256 threads covers 256 ppt pairs (0: 4)
};

struct FcdArgs {
    int n_sims, W, P;
    const float* wfc;       // [n][W][P]
    const double* wsum;     // [n][W][2]
    float* fcd;             // [n][W(W-1)/2] or null
    int n_fcd;
    const double* emp_sorted;  // [m] ascending
    int m;
    unsigned int* hist;     // [n][m+1] counts by upper_bound rank, or null (no KS)
    unsigned int* eq;       // [n][m+1] sim values equal to emp_sorted[c-1]
    const int* ks_lut;      // bucket table of emp_sorted (kKsBuckets + 1), or null
    int* nan_flag;
    int tiles;              // tiles per side
    int p0, p1;             // pair range [p0, p1) of the window-FC rows (wsum holds its sums)
};

struct GofArgs {
    int n_sims, N, P, n_fcd, m;
    const float* fc;               // [n][P]
    const double* emp_fc;          // [P]
    double emp_fc_mean;
    const unsigned int* hist;      // [n][m+1]
    const unsigned int* eq;        // [n][m+1]
    const unsigned char* valid;    // [m+1] emp rank c is a jump point (c==0 or e[c-1] < e[c])
    const double* ext;             // [n][6][N]
    const int* failed;             // [n]
    const int* nan_flag;           // [n]
    int use_fc_diff, calc_fic_penalty, fic_reject_failed, no_fcd;
    double max_cost, fic_penalty_scale;
    double* cost;          // [n]
    double* fic_penalty;   // [n]
    double* fc_corr;       // [n]
    double* fc_diff;       // [n]
    double* fcd_ks;        // [n]
};

// Mean and 1/||z - mean|| of one window-FC vector from its pair sums
// (window_fc_stats, bnm.cu:436-467).
__device__ __forceinline__ void window_norm(const double* wsum, int P, double& mean, double& inv_ssd) {
    mean = wsum[0] / P;
    const double v = wsum[1] - wsum[0] * mean;
    inv_ssd = 1.0 / sqrt(v);
}

// KS bucket of x: c = #emp <= x; also whether x equals emp[c-1].
__device__ __forceinline__ void ks_bucket(const double* e, int m, double x, int& c, bool& equal) {
    int lo = 0, hi = m;  // upper_bound
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (e[mid] <= x) lo = mid + 1; else hi = mid;
    }
    c = lo;
    equal = (c > 0) && (e[c - 1] == x);
}

// Bucket table over the sorted empirical FCD for the KS rank search: bucket b
// covers [edge(b), edge(b+1)) with edge(b) = -1 + b 2^-15 (exact in double),
// bucket 0 extends to -inf and the last to +inf; lut[b] = #emp < edge(b)
// (lut[0] = 0, lut[kKsBuckets] = m).  A correlation's rank is then found by
// two table loads and an upper_bound over the few values of its bucket.
constexpr int kKsBuckets = 1 << 16;
__host__ __device__ __forceinline__ double ks_edge(int b) { return -1.0 + b * (1.0 / 32768.0); }

__device__ __forceinline__ void ks_bucket_lut(const double* e, const int* lut, int m, double x, int& c, bool& equal) {
    const double t = (x + 1.0) * 32768.0;
    int b = t < 1.0 ? 0 : (t >= (double)(kKsBuckets - 1) ? kKsBuckets - 1 : (int)t);
    // x + 1 can round across an edge when |x| is tiny: settle b on the exact edges
    if (b > 0 && x < ks_edge(b)) b--;
    if (b < kKsBuckets - 1 && x >= ks_edge(b + 1)) b++;
    int lo = lut[b], hi = lut[b + 1];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (e[mid] <= x) lo = mid + 1; else hi = mid;
    }
    c = lo;
    equal = (c > 0) && (e[c - 1] == x);
    (void)m;
}

// Tensor-core Gram operands: rows x K values as BF16 tiles of 128 rows x 64 K
// (16 KB, the tcgen05 K-major SWIZZLE_128B layout), tile (sim, row block,
// k block) at ((sim * row_blocks + rb) * kblocks + kb) * 16384 bytes.
constexpr int kGramTileRows = 128, kGramTileK = 64, kGramTileBytes = kGramTileRows * kGramTileK * 2;

struct OperandArgs {
    int n_sims, rows, K, row_blocks, kblocks;
    const float* wfc;         // FCD rows: [n][W][P] window FC ...
    const double* wsum;       // ... and its [n][W][2] pair sums
    const float* bold;        // FC rows: [n][frames][N] BOLD (FP32 integrators) ...
    const double* bold_f64;   // ... or FP64 (one of the two)
    int frames, n_vols_remove;
    unsigned char* hi;        // bf16(x) tiles
    unsigned char* lo;        // bf16(x - hi) tiles, split only (else null)
};

struct GramArgs {
    int n_sims, rows, row_blocks, kblocks;
    const unsigned char* hi;  // operand tiles (OperandArgs layout)
    const unsigned char* lo;  // split only
    float* out;               // lower triangle i > j: out[sim * out_ld + map(i(i-1)/2 + j)], or null
    const int* tril_map;      // null: identity; else output index, or -1 to drop the entry
    long long out_ld;
    const double* emp_sorted; // KS histogram (FCD) as in FcdArgs, or hist == null
    int m;
    unsigned int* hist;
    unsigned int* eq;
    const int* ks_lut;        // bucket table (see ks_bucket_lut), or null
    int* nan_flag;            // [n]
    int* status;
};

struct FicArgs {
    int n_sims, N;
    const double* sc;   // [N][N] (values as the chosen precision rounds them)
    const double* G;    // [n]
    const double* wEE;  // [n][N]
    const double* wEI;  // [n][N]
    double* wIE;        // [n][N] out
    int* unstable;      // [n] out
    int fp32_consts;    // use float-rounded model constants (reference USE_FLOATS build)
};

}  // namespace bnm

namespace bnm {
// One FP32 integrator configuration.  kind 0: register-SC kernel (N <= 128)
// with `slots` particles per CTA; kind 1: row-split cluster kernel (N <= 512,
// even) with `csize` CTAs per particle, `rpw` nodes per warp and `kr` SC
// column chunks in registers; kind 2: the reference-order kernel in FP32 (any
// N); kind 3: column-split cluster kernel (N > 128, an odd N launched with one
// padding node, up to the node count whose SC slice fits an SM) with `csize` CTAs
// per particle, `slots` column pairs per warp, `rpw` rows per lane and `kr`
// column pairs in registers; kind 4: column-split cluster kernel with two
// particles per cluster (fields as kind 3).
struct IntegratorShape {
    int kind, slots, csize, rpw, kr;
};
}  // namespace bnm
cudaError_t bnm_launch_integrate_shape(const bnm::SimArgs& a, const bnm::IntegratorShape& s, int num_sms,
                                       cudaStream_t st);
// Fraction of the GPU (0, 1] one launch of shape s for a.n_sims particles
// fills, by the kernel's own occupancy limit: the SM share a tuner weighs
// when several plans run side by side.
double bnm_integrator_share(const bnm::SimArgs& a, const bnm::IntegratorShape& s, int num_sms);
extern "C" double bnm_cluster_share(int N, int csize, int rpw, int kr, int n_sims);
extern "C" double bnm_colsplit_share(int N, int csize, int rpl, int k2, int krp, int np, int n_sims);
// Candidate shapes for N nodes (those that compile to a launchable kernel); returns the count.
int bnm_integrator_candidates(int N, bnm::IntegratorShape* out, int max);
cudaError_t bnm_launch_integrate_cluster(const bnm::SimArgs& a, int csize, int rpw, int kr, cudaStream_t st);
cudaError_t bnm_launch_integrate_colsplit(const bnm::SimArgs& a, int csize, int rpl, int k2, int krp, int np,
                                          cudaStream_t st);
extern "C" int bnm_colsplit_shape(int N, int csize, int rpl, int k2, int krp, int np, int* threads, int* rows,
                                  size_t* smem);
extern "C" int bnm_colsplit_variants(int* out4, int max);
extern "C" int bnm_cluster_shape(int N, int csize, int rpw, int kr, int* threads, int* rows, size_t* smem);
cudaError_t bnm_launch_integrate_exact(const bnm::SimArgs& a, int fp64, int num_sms, cudaStream_t st);
cudaError_t bnm_launch_fc_window(const bnm::FcArgs& a, cudaStream_t st);
cudaError_t bnm_launch_fcd(bnm::FcdArgs a, cudaStream_t st);
// Per-window sum and sum of squares of window FC over pairs [p0, p1) (FP64):
// wsum_out [n][W][2].
cudaError_t bnm_launch_window_sums(const float* wfc, int n_sims, int W, int P, int p0, int p1, double* wsum_out,
                                   cudaStream_t st);
cudaError_t bnm_launch_gof(const bnm::GofArgs& a, cudaStream_t st);
cudaError_t bnm_launch_fcd_operand(const bnm::OperandArgs& a, cudaStream_t st);
cudaError_t bnm_launch_fc_operand(const bnm::OperandArgs& a, cudaStream_t st);
cudaError_t bnm_launch_gram_tc(const bnm::GramArgs& a, int split, cudaStream_t st);
cudaError_t bnm_launch_analytic_fic(const bnm::FicArgs& a, cudaStream_t st);
cudaError_t bnm_launch_philox(float* out, uint64_t n, int N, int ld, uint64_t seed, int num_sms, cudaStream_t st);
extern "C" int bnm_fast_kmax(int N);
