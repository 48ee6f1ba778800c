/*
 * bnm.cu for amnsbr/bnm_cuda, backed by libbnm_b200.
 *
 * The reference's GPU driver, run_CMAES.cpp, is one translation unit that
 * #includes "bnm.cu" when nvcc compiles it (run_CMAES.cpp:55-59).  Put this
 * file in place of the reference's bnm.cu, next to run_CMAES.cpp, and build
 * the driver the reference's way plus this library:
 *
 *     cp run_CMAES.cpp run_CMAES.cu
 *     nvcc run_CMAES.cu -o run_CMAES_gpu -I<repo>/include \
 *          -L<repo>/bnm_cuda_b200 -lbnm_b200 -Xlinker -rpath,<repo>/bnm_cuda_b200 \
 *          -lm -lgsl -lgslcblas <path-to-libks>/libks.so -I <path-to-libks>/include
 *
 * The driver is unchanged; every generation's call to run_simulations (at
 * run_CMAES.cpp:758-780, and the best-particle rerun at 875-897) runs on the
 * B200 kernels through the C ABI.  This file provides what the driver uses
 * from the reference's bnm.cu (bnm.cu:20-70, 560-617): its headers, the
 * CUDA_CHECK_RETURN macro, the device symbols the driver sets with
 * cudaMemcpyToSymbol, get_device_prop and run_simulations with the same
 * signature.  run_simulations keeps one plan (device buffers, the noise table
 * uploaded once, the tuned integrator) across calls and rebuilds it only when
 * the configuration changes; it writes the driver's outputs in place (corr,
 * fic_penalties, w_IE_fic, FIC_failed, fic_n_trials, BOLD_ex, the extended
 * means S_E .. r_I) and, with save_output, the best-simulation files in the
 * reference's formats (bnm.cu:771-833).  The jagged scratch arrays of the
 * reference (mean_bold, windows_fc_trils, fcd_trils, ...) are not touched.
 * Errors print the library's message and exit(1), as the reference does.
 *
 * BNM_B200_PRECISION=f64|f32ref selects the reference-order kernels instead
 * of the FP32 product path (as for run_CMAES_gpu).
 */
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#include <string.h>
#include <math.h>
#include <sys/stat.h>
#include <iostream>
#include <fstream>
#include <cmath>
#include <string>
#include <cstdlib>
#include <cuda_runtime.h>
#include <random>
#include <algorithm>
#include <cassert>
#include <vector>
#include "constants.h"
#include "fic.cpp"
#include <gsl/gsl_statistics.h>
extern "C" {
#include "ks.h"
};
#include "bnm_b200.h"

// The driver checks every CUDA call it makes itself with this macro (e.g. its
// cudaMallocManaged calls) and expects the process to end on an error.
#define CUDA_CHECK_RETURN(value)                                                                          \
    {                                                                                                     \
        cudaError_t _bnm_b200_e = (value);                                                                \
        if (_bnm_b200_e != cudaSuccess) {                                                                 \
            fprintf(stderr, "Error %s at line %d in file %s\n", cudaGetErrorString(_bnm_b200_e), __LINE__, \
                    __FILE__);                                                                            \
            exit(1);                                                                                      \
        }                                                                                                 \
    }
#define CUDA_CHECK_LAST_ERROR() CUDA_CHECK_RETURN(cudaGetLastError())

// Set by the driver with cudaMemcpyToSymbol (run_CMAES.cpp:449-452).  The
// library reads the same BNM_* values from the environment itself.
__device__ int d_I_SAMPLING_START, d_I_SAMPLING_END, d_I_SAMPLING_DURATION;
__device__ u_real d_init_delta;

cudaDeviceProp get_device_prop(bool verbose = true) {
    int count = 0;
    cudaDeviceProp prop;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
        std::cout << "No CUDA devices found" << std::endl;
        exit(1);
    }
    CUDA_CHECK_RETURN(cudaGetDeviceProperties(&prop, 0));
    if (verbose)
        std::cout << "\nDevice # 0: " << prop.name << ", " << prop.multiProcessorCount << " SMs, "
                  << prop.totalGlobalMem << " bytes, compute capability " << prop.major << "." << prop.minor
                  << " (simulations run on libbnm_b200)" << std::endl;
    return prop;
}

namespace bnm_b200_binding {

[[noreturn]] inline void fail(const char* what) {
    fprintf(stderr, "Error: %s: %s\n", what, bnm_last_error());
    exit(1);
}

struct Cached {
    bnm_plan* plan = nullptr;
    bnm_config cfg;
    const void *sc = nullptr, *noise = nullptr, *emp_fc = nullptr, *emp_fcd = nullptr;
};

inline Cached& cached() {
    static Cached c;
    return c;
}

inline bool same_config(const bnm_config& a, const bnm_config& b) {
    return a.nodes == b.nodes && a.time_steps == b.time_steps && a.bold_tr == b.bold_tr &&
           a.window_step == b.window_step && a.window_size == b.window_size && a.do_fic == b.do_fic &&
           a.numerical_fic == b.numerical_fic && a.max_fic_trials == b.max_fic_trials &&
           a.calculate_fic_penalty == b.calculate_fic_penalty && a.no_fcd == b.no_fcd &&
           a.precision == b.precision && a.gram == b.gram;
}

}  // namespace bnm_b200_binding

void run_simulations(
    double* corr, u_real* fic_penalties, u_real* G_list, u_real* w_EE_list, u_real* w_EI_list, u_real* w_IE_list,
    u_real** w_IE_fic, u_real* SC, int nodes, bool calculate_fic_penalty, int time_steps, int BOLD_TR,
    int _max_fic_trials, bool sim_only, gsl_vector* emp_FC_tril, gsl_vector* emp_FCD_tril, int window_size,
    bool save_output, bool extended_output, std::string sims_out_prefix, int N_SIMS, u_real* noise, int output_ts,
    cudaDeviceProp prop, u_real** BOLD_ex, u_real** S_E, u_real** I_E, u_real** r_E, u_real** S_I, u_real** I_I,
    u_real** r_I, bool do_fic, bool adjust_fic, bool* FIC_failed, int* fic_n_trials, int n_vols_remove,
    int corr_len, u_real** mean_bold, u_real** ssd_bold, int n_windows, int* window_starts, int* window_ends,
    u_real** windows_mean_bold, u_real** windows_ssd_bold, u_real** fc_trils, u_real** windows_fc_trils,
    u_real** windows_mean_fc, u_real** windows_ssd_fc, int n_pairs, int* pairs_i, int* pairs_j,
    int n_window_pairs, int* window_pairs_i, int* window_pairs_j, u_real** fcd_trils, double** d_fc_trils,
    double** d_fcd_trils, gsl_vector* emp_FCD_tril_copy) {
    using namespace bnm_b200_binding;
    (void)prop;
    // ---- configuration: the driver's arguments plus BNM_* (read by the library like the reference)
    bnm_config cfg;
    bnm_config_default(&cfg);
    bnm_config_from_env(&cfg);
    cfg.nodes = nodes;
    cfg.max_sims = N_SIMS;
    cfg.time_steps = time_steps;
    cfg.bold_tr = BOLD_TR;
    cfg.window_size = window_size;
    // the driver lays out its windows from argv[14] (run_CMAES.cpp:531-556); the step is their spacing
    cfg.window_step = n_windows > 1 ? window_starts[1] - window_starts[0] : 1;
    cfg.do_fic = do_fic;
    cfg.numerical_fic = adjust_fic;
    cfg.max_fic_trials = _max_fic_trials;
    cfg.calculate_fic_penalty = calculate_fic_penalty;
    cfg.no_fcd = emp_FCD_tril == NULL || emp_FCD_tril->size == 0;
    cfg.noise_mode = BNM_NOISE_HOST;  // the driver's mt19937 stream (run_CMAES.cpp:640-657)
    if (const char* p = getenv("BNM_B200_PRECISION")) {
        if (!strcmp(p, "f64")) cfg.precision = BNM_PREC_F64;
        else if (!strcmp(p, "f32ref")) cfg.precision = BNM_PREC_F32_REF;
    }
    bnm_sizes s;
    if (bnm_config_sizes(&cfg, &s) != BNM_OK) fail("run_simulations: configuration");
    if (s.frames != output_ts || s.n_vols_remove != n_vols_remove || s.corr_len != corr_len ||
        s.n_pairs != n_pairs || s.n_windows != n_windows || (!cfg.no_fcd && s.n_fcd != n_window_pairs) ||
        (n_windows > 0 && window_starts[0] != n_vols_remove)) {
        fprintf(stderr, "Error: run_simulations: the driver's frame / pair / window tables differ from the library's "
                        "(frames %d/%d, pairs %d/%d, windows %d/%d)\n",
                output_ts, s.frames, n_pairs, s.n_pairs, n_windows, s.n_windows);
        exit(1);
    }

    // ---- the plan, kept while the configuration and the driver's arrays stay the same
    Cached& c = cached();
    const bool reuse = c.plan && same_config(c.cfg, cfg) && N_SIMS <= c.cfg.max_sims && c.sc == SC &&
                       c.noise == noise && c.emp_fc == emp_FC_tril && c.emp_fcd == emp_FCD_tril;
    if (!reuse) {
        if (c.plan) bnm_plan_destroy(c.plan);
        c.plan = nullptr;
        std::vector<double> sc(SC, SC + (size_t)nodes * nodes);
        std::vector<float> nz(noise, noise + s.noise_len);  // the driver's values are floats (run_CMAES.cpp:648-652)
        const double* efcd = cfg.no_fcd ? NULL : emp_FCD_tril->data;
        if (bnm_plan_create(&cfg, sc.data(), emp_FC_tril->data, (int32_t)emp_FC_tril->size, efcd,
                            cfg.no_fcd ? 0 : (int32_t)emp_FCD_tril->size, nz.data(), s.noise_len,
                            &c.plan) != BNM_OK)
            fail("run_simulations: plan");
        c.cfg = cfg;
        c.sc = SC;
        c.noise = noise;
        c.emp_fc = emp_FC_tril;
        c.emp_fcd = emp_FCD_tril;
    }

    // ---- one batch
    const size_t nN = (size_t)N_SIMS * nodes;
    std::vector<double> G(G_list, G_list + N_SIMS), wee(w_EE_list, w_EE_list + nN), wei(w_EI_list, w_EI_list + nN),
        wie(nN), cost(N_SIMS), pen(N_SIMS), ext(nN * 6), bold(nN * output_ts);
    for (int i = 0; i < N_SIMS; i++)  // with FIC, w_IE_fic holds the driver's analytic start (run_CMAES.cpp:144-174)
        for (int j = 0; j < nodes; j++)
            wie[(size_t)i * nodes + j] = do_fic ? (double)w_IE_fic[i][j] : (double)w_IE_list[(size_t)i * nodes + j];
    std::vector<int32_t> failed(N_SIMS), trials(N_SIMS);
    bnm_batch_out out;
    memset(&out, 0, sizeof out);
    out.cost = cost.data();
    out.fic_penalty = pen.data();
    out.w_ie = wie.data();
    out.fic_failed = failed.data();
    out.fic_ntrials = trials.data();
    out.ext_means = ext.data();
    out.bold = bold.data();
    if (bnm_run(c.plan, N_SIMS, G.data(), wee.data(), wei.data(), wie.data(), &out) != BNM_OK)
        fail("run_simulations");

    // ---- outputs in the driver's arrays
    u_real** ext_out[6] = {S_E, I_E, r_E, S_I, I_I, r_I};
    for (int i = 0; i < N_SIMS; i++) {
        if (!sim_only) {
            corr[i] = cost[i];
            if (calculate_fic_penalty) fic_penalties[i] = (u_real)pen[i];
        }
        FIC_failed[i] = failed[i] != 0;
        fic_n_trials[i] = trials[i];
        for (size_t k = 0; k < (size_t)output_ts * nodes; k++)
            BOLD_ex[i][k] = (u_real)bold[(size_t)i * output_ts * nodes + k];
        for (int j = 0; j < nodes; j++) {
            if (do_fic) w_IE_fic[i][j] = (u_real)wie[(size_t)i * nodes + j];
            if (extended_output)
                for (int e = 0; e < 6; e++) ext_out[e][i][j] = (u_real)ext[((size_t)i * 6 + e) * nodes + j];
        }
    }

    // ---- best-simulation files (bnm.cu:771-833)
    if (save_output) {
        if (N_SIMS != 1) {
            printf("Saving multiple simulations output not implemented\n");
            exit(1);
        }
        auto open = [&](const char* name) {
            FILE* f = fopen((sims_out_prefix + name).c_str(), "w");
            if (!f) {
                fprintf(stderr, "Error: cannot write %s%s\n", sims_out_prefix.c_str(), name);
                exit(1);
            }
            return f;
        };
        FILE* f = open("bold.txt");
        for (int t = 0; t < output_ts; t++) {
            for (int j = 0; j < nodes; j++) fprintf(f, "%f ", BOLD_ex[0][t * nodes + j]);
            fprintf(f, "\n");
        }
        fclose(f);
        const char* ext_names[6] = {"S_E.txt", "I_E.txt", "r_E.txt", "S_I.txt", "I_I.txt", "r_I.txt"};
        for (int e = 0; e < 6; e++) {
            f = open(ext_names[e]);
            for (int j = 0; j < nodes; j++) fprintf(f, "%f ", ext_out[e][0][j]);
            fclose(f);
        }
        f = open("w_EE.txt");
        for (int j = 0; j < nodes; j++) fprintf(f, "%f ", w_EE_list[j]);
        fclose(f);
        f = open("w_EI.txt");
        for (int j = 0; j < nodes; j++) fprintf(f, "%f ", w_EI_list[j]);
        fclose(f);
        if (do_fic) {
            f = open("w_IE.txt");
            for (int j = 0; j < nodes; j++) fprintf(f, "%f ", w_IE_fic[0][j]);
            fclose(f);
            if (adjust_fic) {
                f = open("fic_failed.txt");
                fprintf(f, "%d", (int)FIC_failed[0]);
                fclose(f);
                f = open("fic_ntrials.txt");
                fprintf(f, "%d of max %d", fic_n_trials[0], _max_fic_trials);
                fclose(f);
            }
        }
    }
}
