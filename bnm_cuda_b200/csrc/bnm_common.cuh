// Shared definitions for the B200 simulate-and-fit kernels.
//
// Model constants are those of the reference's constants.h:24-90 (reduced
// Wong-Wang excitatory/inhibitory pools, Deco et al. 2014; Balloon-Windkessel
// with the 3 T coefficients of Demirtas 2019).  They are instantiated per
// arithmetic type exactly as the reference declares them (`const u_real x =
// literal`), so the FP64 and reference-order FP32 kernels see the same
// rounded values as the reference's double and USE_FLOATS builds.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bnm {

template <typename R>
struct Model {
    static constexpr R dt = 0.1, model_dt = 0.001, sqrt_dt = 0.316227;
    static constexpr R J_NMDA = 0.15, a_E = 310, b_E = 125, d_E = 0.16, a_I = 615, b_I = 177, d_I = 0.087;
    static constexpr R b_a_ratio_E = b_E / a_E;
    static constexpr R gamma_E = (R)0.641 / (R)1000.0, gamma_I = (R)1.0 / (R)1000.0;
    static constexpr R tau_E = 100, tau_I = 10;
    static constexpr R sigma_model = 0.01, I_0 = 0.382, w_E = 1.0, w_I = 0.7, w_II = 1.0, I_ext = 0.0;
    static constexpr R w_E__I_0 = w_E * I_0, w_I__I_0 = w_I * I_0;
    static constexpr R rho = 0.34, alpha = 0.32, tau = 0.98, y = 1.0 / 0.41, kappa = 1.0 / 0.65;
    static constexpr R V_0 = 0.02 * 100, ialpha = 1.0 / alpha, itau = 1.0 / tau, oneminrho = (1.0 - rho);
    static constexpr R k1 = 3.72, k2 = 0.527, k3 = 0.53;
};

// Status word bits written by kernels (host maps them to BNM_E* codes).
enum : int {
    kStatusOk = 0,
    kStatusBadArgs = 1,
    kStatusTimeout = 2,  // a bounded device wait gave up
};

// Launch-time description of one batch of simulations (all device pointers).
struct SimArgs {
    int N;            // nodes
    int n_sims;       // particles in this call
    int T;            // simulated ms; the loop runs ts = 0..T inclusive
    int TR;           // BOLD sampling period in ms
    int frames;       // T / TR + 1
    int n_vols_remove;
    int adjust_fic, max_trials, samp_start, samp_end;
    double init_delta;
    const double* G;       // [n]
    const double* wEE;     // [n][N]
    const double* wEI;     // [n][N]
    const double* wIE;     // [n][N] initial wIE (analytic FIC or fixed)
    const float* noise;    // [(T+1)*10][N][2] standard normals, or NULL: drawn in the kernel (Philox, noise.cuh)
    uint64_t noise_seed;   // Philox key when noise == NULL
    int noise_ld;          // node stride of the noise table (N, or N + 1 when padded for an odd N)
    int n_real;            // nodes of the simulation; the kernel's N may add one padding node
    const float* sc_f32;   // [N][sc_ld] row-major, zero padded
    const double* sc_f64;  // [N][N]
    int sc_ld;
    // outputs
    float* bold;        // [n][frames][N] (fp32 kernels)
    double* bold_f64;   // [n][frames][N] (fp64 kernel)
    double* wIE_out;    // [n][N]
    int* trials;        // [n]
    int* failed;        // [n]
    double* ext;        // [n][6][N] means of S_E, I_E, r_E, S_I, I_I, r_I over kept frames
    int* work_counter;  // persistent scheduling (zeroed before launch)
    const int* order;   // optional placement: particles by predicted work, heaviest first
    int* place_ws;      // with order: [0, 2) a 64-bit two-ended claim word, [2, 2 + 256) CTAs per SM (zeroed)
    int* status;
};

}  // namespace bnm

#define BNM_CUDA_TRY(expr)                                 \
    do {                                                   \
        cudaError_t _e = (expr);                           \
        if (_e != cudaSuccess) return bnm_fail_cuda(_e, #expr, __FILE__, __LINE__); \
    } while (0)
