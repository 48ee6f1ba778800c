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
    double* wsum;             // [n][W][2] sum, sum of squares over pairs (zeroed)
    int* nan_flag;            // [n]
};

struct FcdArgs {
    int n_sims, W, P;
    const float* wfc;       // [n][W][P]
    const double* wsum;     // [n][W][2]
    float* fcd;             // [n][W(W-1)/2] or null
    int n_fcd;
    const double* emp_sorted;  // [m] ascending
    int m;
    unsigned int* hist;     // [n][m+1] counts by upper_bound rank
    unsigned int* eq;       // [n][m+1] sim values equal to emp_sorted[c-1]
    int* nan_flag;
    int tiles;              // tiles per side
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

cudaError_t bnm_launch_integrate_f32(const bnm::SimArgs& a, int num_sms, cudaStream_t st);
cudaError_t bnm_launch_integrate_exact(const bnm::SimArgs& a, int fp64, int num_sms, cudaStream_t st);
cudaError_t bnm_launch_fc_window(const bnm::FcArgs& a, cudaStream_t st);
cudaError_t bnm_launch_fcd(bnm::FcdArgs a, cudaStream_t st);
cudaError_t bnm_launch_gof(const bnm::GofArgs& a, cudaStream_t st);
cudaError_t bnm_launch_analytic_fic(const bnm::FicArgs& a, cudaStream_t st);
cudaError_t bnm_launch_philox(float* out, uint64_t n, uint64_t seed, int num_sms, cudaStream_t st);
extern "C" int bnm_fast_kmax(int N);
