// C ABI of the library (include/bnm_b200.h): configuration, plans, the batch
// entry point and its one-shot run_simulations mirror.
//
// A plan allocates every device buffer once for max_sims particles and then
// runs a generation as a fixed sequence of launches on its own stream:
//   analytic FIC (optional) -> integrate -> FC + window FC -> FCD + KS histogram -> GOF
// (the reference runs bnm, bold_stats, window_bold_stats, fc, window_fc_stats,
// fcd, float2double with a device-wide sync after each, then a host GOF loop,
// bnm.cu:623-769).  Errors come back as status codes, never exit().
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/bnm_b200.h"
#include "kernels.h"

using namespace bnm;

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}
int bnm_fail_cuda(cudaError_t e, const char* expr, const char* file, int line) {
    return fail(e == cudaErrorMemoryAllocation ? BNM_ENOMEM : BNM_ECUDA, "%s failed: %s (%s:%d)", expr,
                cudaGetErrorString(e), file, line);
}

int bnm_fail_msg(int code, const char* msg) { return fail(code, "%s", msg); }

extern "C" const char* bnm_last_error(void) { return g_err.c_str(); }

extern "C" int bnm_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" void bnm_config_default(bnm_config* c) {
    std::memset(c, 0, sizeof *c);
    c->nodes = 100;
    c->max_sims = 1;
    c->time_steps = 60000;
    c->bold_tr = 1000;
    c->window_step = 2;
    c->window_size = 10;
    c->bold_remove_s = 30;
    c->exc_interhem = 1;
    c->do_fic = 1;
    c->numerical_fic = 1;
    c->max_fic_trials = 10;
    c->i_sampling_start = 1000;
    c->i_sampling_end = 10000;
    c->init_delta = (double)(float)0.02;
    c->use_fc_diff = 1;
    c->fic_reject_failed = 0;
    c->fic_penalty_scale = 2.0;
    c->max_cost = 2.0;
    c->calculate_fic_penalty = 1;
    c->no_fcd = 0;
    c->precision = BNM_PREC_F32;
    c->noise_mode = BNM_NOISE_PHILOX;
    c->noise_seed = 410;
    c->device = 0;
    c->gram = BNM_GRAM_AUTO;
}

// helpers.cpp:4-19: ints through atoi; doubles through atof, returned as float.
static int env_int(const char* k, int d) {
    const char* v = std::getenv(k);
    return v ? std::atoi(v) : d;
}
static double env_dbl(const char* k, double d) {
    const char* v = std::getenv(k);
    return v ? (double)(float)std::atof(v) : (double)(float)d;
}

extern "C" void bnm_config_from_env(bnm_config* c) {
    c->bold_remove_s = env_int("BNM_BOLD_REMOVE", c->bold_remove_s);
    c->max_cost = (double)env_int("BNM_MAX_COST", (int)c->max_cost);
    c->i_sampling_start = env_int("BNM_I_SAMPLING_START", c->i_sampling_start);
    c->i_sampling_end = env_int("BNM_I_SAMPLING_END", c->i_sampling_end);
    c->numerical_fic = env_int("BNM_NUMERICAL_FIC", c->numerical_fic) != 0;
    c->max_fic_trials = env_int("BNM_MAX_FIC_TRIALS_CMAES", c->max_fic_trials);
    c->init_delta = env_dbl("BNM_INIT_DELTA", 0.02);
    c->use_fc_diff = env_int("BNM_USE_FC_DIFF", c->use_fc_diff) != 0;
    c->exc_interhem = env_int("BNM_EXC_INTERHEM", c->exc_interhem) != 0;
    c->fic_penalty_scale = env_dbl("BNM_CMAES_FIC_PENALTY_SCALE", 2.0);
    c->fic_reject_failed = env_int("BNM_CMAES_FIC_REJECT_FAILED", c->fic_reject_failed) != 0;
}

// Sizes of run_CMAES.cpp:476-594.
extern "C" int bnm_config_sizes(const bnm_config* c, bnm_sizes* s) {
    if (c->nodes < 2 || c->nodes > 1024) return fail(BNM_EINVAL, "nodes must be in [2, 1024] (got %d)", c->nodes);
    if (c->bold_tr <= 0 || c->time_steps < 0) return fail(BNM_EINVAL, "time_steps >= 0 and BOLD_TR > 0 required");
    if (c->window_step <= 0 || c->window_size < 0) return fail(BNM_EINVAL, "window_step > 0 and window_size >= 0 required");
    if (c->exc_interhem && (c->nodes % 2)) return fail(BNM_EINVAL, "exc_interhem needs an even node count");
    std::memset(s, 0, sizeof *s);
    s->frames = c->time_steps / c->bold_tr + 1;
    // the reference sizes its buffers with a floating-point quotient
    // (run_CMAES.cpp:476-477); frames are written at ts % TR == 0, so the two
    // must agree or the reference itself would under/overrun.
    const double tr_s = (double)c->bold_tr / 1000;
    const int ref_frames = (int)(c->time_steps / (tr_s / 0.001)) + 1;
    if (ref_frames != s->frames)
        return fail(BNM_EINVAL, "time_steps/BOLD_TR gives %d frames but the reference sizes %d", s->frames, ref_frames);
    s->n_vols_remove = c->bold_remove_s * 1000 / c->bold_tr;
    s->corr_len = s->frames - s->n_vols_remove;
    if (s->corr_len < 2) return fail(BNM_EINVAL, "fewer than 2 BOLD frames left after removing %d", s->n_vols_remove);
    const int N = c->nodes;
    s->n_pairs = N * (N - 1) / 2 - (c->exc_interhem ? (N / 2) * (N / 2) : 0);
    const int h = c->window_size / 2;
    s->window_len = 2 * h + 1;
    const int first = h, last = s->corr_len - 1 - h;
    s->n_windows = last >= first ? (last - first) / c->window_step + 1 : 0;
    s->n_fcd = s->n_windows * (s->n_windows - 1) / 2;
    if (!c->no_fcd && s->n_windows < 2) return fail(BNM_EINVAL, "need at least 2 FCD windows (got %d)", s->n_windows);
    s->noise_len = (int64_t)N * (c->time_steps + 1) * 10 * 2;
    return BNM_OK;
}

constexpr int kPlaceWs = 2 + 256;  // placement claim word + CTAs per SM

struct bnm_plan {
    bnm_config cfg;
    bnm_sizes sz;
    int num_sms = 0, kmax = 0, sc_ld = 0, m = 0;
    int pad = 0, noise_ld = 0;  // padding node of an odd N (column-split kernel); node stride of the noise table
    cudaStream_t st = nullptr;
    cudaEvent_t ev[6] = {}, tev[2] = {};
    double emp_fc_mean = 0;
    float* d_sc32 = nullptr;
    double *d_sc64 = nullptr, *d_sc_fic = nullptr;
    float* d_noise = nullptr;
    int *d_pi = nullptr, *d_pj = nullptr;
    double *d_emp_fc = nullptr, *d_emp_sorted = nullptr;
    int* d_ks_lut = nullptr;
    unsigned char* d_valid = nullptr;
    double *d_G = nullptr, *d_wEE = nullptr, *d_wEI = nullptr, *d_wIE = nullptr, *d_wIE_out = nullptr;
    int* d_unstable = nullptr;
    float* d_bold = nullptr;
    double* d_bold64 = nullptr;
    int *d_trials = nullptr, *d_failed = nullptr, *d_nan = nullptr, *d_counter = nullptr, *d_status = nullptr;
    double* d_ext = nullptr;
    float *d_fc = nullptr, *d_wfc = nullptr, *d_fcd = nullptr;
    double* d_wsum = nullptr;
    unsigned int *d_hist = nullptr, *d_eq = nullptr;
    double *d_cost = nullptr, *d_pen = nullptr, *d_fcc = nullptr, *d_fcdiff = nullptr, *d_ks = nullptr;
    // tensor-core Grams: BF16 operand tiles (FCD for gram_chunk sims at a time,
    // FC for all), and the map from the full lower triangle to pair order
    unsigned char *d_fcd_hi = nullptr, *d_fcd_lo = nullptr, *d_fc_hi = nullptr, *d_fc_lo = nullptr;
    int* d_tril_map = nullptr;
    int fcd_rb = 0, fcd_kb = 0, fc_rb = 0, fc_kb = 0, gram_chunk = 0;
    // hemisphere FCDs (optional outputs; allocated on first request)
    float* d_fcd_hemi = nullptr;
    double* d_wsum_hemi = nullptr;
    // FP32 integrator picked by the autotuner for batches of tuned_n particles
    IntegratorShape shape{};
    int tuned_n = 0, n_tried = 0;
    // pinned host staging for graph-captured (group) runs
    unsigned char* pinned = nullptr;
    double *io_G = nullptr, *io_wEE = nullptr, *io_wEI = nullptr, *io_cost = nullptr, *io_pen = nullptr,
           *io_fcc = nullptr, *io_fcdiff = nullptr, *io_ks = nullptr, *io_wie = nullptr;
    int *io_failed = nullptr, *io_trials = nullptr, *io_unstable = nullptr, *io_status = nullptr;
    bool capturing = false;
    // bnm_run's generation as one CUDA graph (captured for batches of run_graph_n particles)
    cudaGraph_t run_graph = nullptr;
    cudaGraphExec_t run_exec = nullptr;
    int run_graph_n = 0, last_graph = 0;
    // window-FC tile (pairs per thread) picked by the tuner for batches of win_tuned_n particles
    int win_ppt = 0, win_tuned_n = 0, win_tried = 0;
    // placement of particles on the register kernel's CTAs by predicted FIC work (on by
    // default; BNM_B200_PLACE=0 turns it off): the predicted order, the claim counters,
    // and the parameters and FIC restart counts of the particles simulated so far
    bool place = false;
    bool last_placed = false;  // the last run's order came from the history
    int* d_order = nullptr;
    int* d_place_ws = nullptr;  // kPlaceWs ints, zeroed before each launch
    int* io_order = nullptr;  // pinned [max_sims]
    std::vector<float> hist_x;  // G, mean wEE, mean wEI per simulated particle
    std::vector<int> hist_tr;
    size_t hist_next = 0;
    double timings[6] = {0, 0, 0, 0, 0, 0};
    // tensor-core Gram kernels alone: one event pair per launch (FC, then each FCD chunk)
    std::vector<cudaEvent_t> gev;
    int n_gram = 0, launches = 0;
    double gram_ms[2] = {0, 0};
    std::vector<void*> allocs;
};

template <typename T>
static cudaError_t dalloc(bnm_plan* p, T** ptr, size_t count) {
    cudaError_t e = cudaMalloc((void**)ptr, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) p->allocs.push_back(*ptr);
    return e;
}

extern "C" void bnm_plan_destroy(bnm_plan* p) {
    if (!p) return;
    cudaSetDevice(p->cfg.device);
    if (p->st) cudaStreamSynchronize(p->st);
    for (void* a : p->allocs) cudaFree(a);
    if (p->run_exec) cudaGraphExecDestroy(p->run_exec);
    if (p->run_graph) cudaGraphDestroy(p->run_graph);
    if (p->pinned) cudaFreeHost(p->pinned);
    if (p->io_order) cudaFreeHost(p->io_order);
    for (auto& e : p->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : p->tev)
        if (e) cudaEventDestroy(e);
    for (auto& e : p->gev)
        if (e) cudaEventDestroy(e);
    if (p->st) cudaStreamDestroy(p->st);
    delete p;
}

static int plan_create(const bnm_config* cfg, const double* sc, const double* emp_fc, int n_emp_fc,
                       const double* emp_fcd, int n_emp_fcd, const float* host_noise, int64_t n_host_noise,
                       bnm_plan* p) {
    p->cfg = *cfg;
    int rc = bnm_config_sizes(cfg, &p->sz);
    if (rc) return rc;
    const bnm_sizes& s = p->sz;
    const int N = cfg->nodes;
    if (cfg->max_sims < 1) return fail(BNM_EINVAL, "max_sims must be >= 1");
    if (!sc) return fail(BNM_EINVAL, "SC is required");
    if (!emp_fc || n_emp_fc != s.n_pairs)
        return fail(BNM_EINVAL, "empirical FC has %d values; %d nodes with exc_interhem=%d need %d", n_emp_fc, N,
                    cfg->exc_interhem, s.n_pairs);
    if (!cfg->no_fcd && (!emp_fcd || n_emp_fcd < 1)) return fail(BNM_EINVAL, "empirical FCD is required");
    if (cfg->noise_mode == BNM_NOISE_HOST && (!host_noise || n_host_noise < s.noise_len))
        return fail(BNM_EINVAL, "host noise needs %lld values (got %lld)", (long long)s.noise_len,
                    (long long)n_host_noise);
    if (cfg->precision < 0 || cfg->precision > 2) return fail(BNM_EINVAL, "unknown precision %d", cfg->precision);
    if (cfg->gram < BNM_GRAM_AUTO || cfg->gram > 2) return fail(BNM_EINVAL, "unknown gram arithmetic %d", cfg->gram);
    // AUTO: tensor-core split BF16 for the FP32 product path, the FP32 / FP64
    // SIMT analysis for the reference-order precisions
    if (p->cfg.gram == BNM_GRAM_AUTO)
        p->cfg.gram = cfg->precision == BNM_PREC_F32 ? BNM_GRAM_BF16_SPLIT : BNM_GRAM_F32;
    for (int i = 0; i < N * N; i++)
        if (!std::isfinite(sc[i])) return fail(BNM_EINVAL, "SC has a non-finite entry at %d", i);

    BNM_CUDA_TRY(cudaSetDevice(cfg->device));
    BNM_CUDA_TRY(cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, cfg->device));
    BNM_CUDA_TRY(cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking));
    for (auto& e : p->ev) BNM_CUDA_TRY(cudaEventCreate(&e));
    for (auto& e : p->tev) BNM_CUDA_TRY(cudaEventCreate(&e));

    // SC: FP32 rows padded for the register kernel, FP64 for the exact kernel,
    // and the FIC copy rounded like the chosen precision's u_real.
    p->kmax = (cfg->precision == BNM_PREC_F32) ? bnm_fast_kmax(N) : 0;
    // an odd N above the register kernel's range runs the column-split kernel
    // with one padding node (zero SC row and column, its own noise column)
    p->pad = (cfg->precision == BNM_PREC_F32 && !p->kmax && (N & 1)) ? 1 : 0;
    p->sc_ld = p->kmax ? p->kmax : N + p->pad;
    std::vector<float> sc32((size_t)(N + p->pad) * p->sc_ld, 0.f);
    std::vector<double> scfic((size_t)N * N);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            sc32[(size_t)i * p->sc_ld + j] = (float)sc[(size_t)i * N + j];
            scfic[(size_t)i * N + j] =
                cfg->precision == BNM_PREC_F32_REF ? (double)(float)sc[(size_t)i * N + j] : sc[(size_t)i * N + j];
        }
    BNM_CUDA_TRY(dalloc(p, &p->d_sc32, sc32.size()));
    BNM_CUDA_TRY(dalloc(p, &p->d_sc64, (size_t)N * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_sc_fic, (size_t)N * N));
    BNM_CUDA_TRY(cudaMemcpy(p->d_sc32, sc32.data(), sc32.size() * 4, cudaMemcpyHostToDevice));
    BNM_CUDA_TRY(cudaMemcpy(p->d_sc64, sc, (size_t)N * N * 8, cudaMemcpyHostToDevice));
    BNM_CUDA_TRY(cudaMemcpy(p->d_sc_fic, scfic.data(), scfic.size() * 8, cudaMemcpyHostToDevice));

    // noise: the caller's table (HOST), or Philox values.  The FP32 kernels can
    // draw those where they use them (no table): the cluster kernels (N > 128)
    // do by default, one millisecond per block at a time; the register kernel
    // (N <= 128) reads a table by default, because drawing in place lengthens
    // its substep (measured at N = 100, 256 particles: 149.2 against 170.7
    // sims/s).  The reference-order kernels always read a table.
    // BNM_B200_NOISE_SOURCE=table|inline overrides the FP32 default.
    bool can_inline = cfg->precision == BNM_PREC_F32 && bnm_fast_kmax(N);
    if (cfg->precision == BNM_PREC_F32 && !can_inline) {
        IntegratorShape cand[128];
        const int nc = bnm_integrator_candidates(N, cand, 128);
        for (int i = 0; i < nc; i++) can_inline |= cand[i].kind != 2;
    }
    bool inline_noise = can_inline && !bnm_fast_kmax(N);
    if (const char* ns = std::getenv("BNM_B200_NOISE_SOURCE")) {
        if (!std::strcmp(ns, "table")) inline_noise = false;
        else if (!std::strcmp(ns, "inline")) inline_noise = can_inline;
        else return fail(BNM_EINVAL, "BNM_B200_NOISE_SOURCE must be table or inline");
    }
    const bool table = cfg->noise_mode == BNM_NOISE_HOST || !inline_noise;
    p->noise_ld = N + p->pad;
    if (table) {
        const size_t rows = (size_t)(cfg->time_steps + 1) * 10;  // substeps; a row holds (E, I) of every node
        BNM_CUDA_TRY(dalloc(p, &p->d_noise, rows * p->noise_ld * 2));
        if (p->pad) BNM_CUDA_TRY(cudaMemset(p->d_noise, 0, rows * p->noise_ld * 2 * 4));
        if (cfg->noise_mode == BNM_NOISE_HOST)
            BNM_CUDA_TRY(cudaMemcpy2D(p->d_noise, (size_t)p->noise_ld * 8, host_noise, (size_t)N * 8, (size_t)N * 8,
                                      rows, cudaMemcpyHostToDevice));
        else
            BNM_CUDA_TRY(bnm_launch_philox(p->d_noise, (uint64_t)s.noise_len, N, p->noise_ld, cfg->noise_seed,
                                           p->num_sms, p->st));
    }

    // particle placement (numerical FIC, FP32: the register kernel with a noise table, the
    // column-split clusters; BNM_B200_PLACE=0 turns it off)
    {
        const char* pl = std::getenv("BNM_B200_PLACE");
        p->place = !(pl && !std::strcmp(pl, "0")) && cfg->precision == BNM_PREC_F32 && cfg->do_fic &&
                   cfg->numerical_fic && (p->kmax ? p->d_noise != nullptr : true);
    }
    if (p->place) {
        BNM_CUDA_TRY(dalloc(p, &p->d_place_ws, kPlaceWs));
        BNM_CUDA_TRY(dalloc(p, &p->d_order, (size_t)cfg->max_sims));
        BNM_CUDA_TRY(cudaMallocHost((void**)&p->io_order, (size_t)cfg->max_sims * sizeof(int)));
        for (int i = 0; i < cfg->max_sims; i++) p->io_order[i] = i;
        BNM_CUDA_TRY(cudaMemcpy(p->d_order, p->io_order, (size_t)cfg->max_sims * 4, cudaMemcpyHostToDevice));
    }

    // pair table (run_CMAES.cpp:505-524)
    std::vector<int> pi, pj;
    const int rh = N / 2;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < i; j++) {
            if (cfg->exc_interhem && ((i < rh) ^ (j < rh))) continue;
            pi.push_back(i);
            pj.push_back(j);
        }
    BNM_CUDA_TRY(dalloc(p, &p->d_pi, pi.size()));
    BNM_CUDA_TRY(dalloc(p, &p->d_pj, pj.size()));
    BNM_CUDA_TRY(cudaMemcpy(p->d_pi, pi.data(), pi.size() * 4, cudaMemcpyHostToDevice));
    BNM_CUDA_TRY(cudaMemcpy(p->d_pj, pj.data(), pj.size() * 4, cudaMemcpyHostToDevice));

    // targets: empirical FC and its mean; empirical FCD sorted, with jump flags
    double mfc = 0;
    for (int i = 0; i < n_emp_fc; i++) mfc += emp_fc[i];
    p->emp_fc_mean = mfc / n_emp_fc;
    BNM_CUDA_TRY(dalloc(p, &p->d_emp_fc, n_emp_fc));
    BNM_CUDA_TRY(cudaMemcpy(p->d_emp_fc, emp_fc, (size_t)n_emp_fc * 8, cudaMemcpyHostToDevice));
    p->m = cfg->no_fcd ? 1 : n_emp_fcd;
    std::vector<double> es(p->m, 0.0);
    if (!cfg->no_fcd) {
        es.assign(emp_fcd, emp_fcd + n_emp_fcd);
        std::sort(es.begin(), es.end());
    }
    std::vector<unsigned char> valid(p->m + 1, 0);
    valid[0] = 1;  // sims below every empirical value
    for (int c = 1; c <= p->m; c++) valid[c] = (c == p->m) || (es[c - 1] < es[c]);
    BNM_CUDA_TRY(dalloc(p, &p->d_emp_sorted, es.size()));
    BNM_CUDA_TRY(dalloc(p, &p->d_valid, valid.size()));
    BNM_CUDA_TRY(cudaMemcpy(p->d_emp_sorted, es.data(), es.size() * 8, cudaMemcpyHostToDevice));
    std::vector<int> lut(kKsBuckets + 1, 0);
    for (int b = 1; b < kKsBuckets; b++)
        lut[b] = (int)(std::lower_bound(es.begin(), es.end(), ks_edge(b)) - es.begin());
    lut[kKsBuckets] = p->m;
    BNM_CUDA_TRY(dalloc(p, &p->d_ks_lut, lut.size()));
    BNM_CUDA_TRY(cudaMemcpy(p->d_ks_lut, lut.data(), lut.size() * 4, cudaMemcpyHostToDevice));
    BNM_CUDA_TRY(cudaMemcpy(p->d_valid, valid.data(), valid.size(), cudaMemcpyHostToDevice));

    // per-particle work space
    const size_t n = cfg->max_sims;
    BNM_CUDA_TRY(dalloc(p, &p->d_G, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_wEE, n * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_wEI, n * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_wIE, n * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_wIE_out, n * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_unstable, n));
    if (cfg->precision == BNM_PREC_F64)
        BNM_CUDA_TRY(dalloc(p, &p->d_bold64, n * s.frames * N));
    else
        BNM_CUDA_TRY(dalloc(p, &p->d_bold, n * s.frames * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_trials, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_failed, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_nan, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_counter, 4));
    BNM_CUDA_TRY(dalloc(p, &p->d_status, 4));
    BNM_CUDA_TRY(dalloc(p, &p->d_ext, n * 6 * N));
    BNM_CUDA_TRY(dalloc(p, &p->d_fc, n * s.n_pairs));
    BNM_CUDA_TRY(dalloc(p, &p->d_wfc, n * (size_t)std::max(s.n_windows, 1) * s.n_pairs));
    BNM_CUDA_TRY(dalloc(p, &p->d_wsum, n * (size_t)std::max(s.n_windows, 1) * 2));
    BNM_CUDA_TRY(dalloc(p, &p->d_fcd, n * (size_t)std::max(s.n_fcd, 1)));
    BNM_CUDA_TRY(dalloc(p, &p->d_hist, n * (size_t)(p->m + 1)));
    BNM_CUDA_TRY(dalloc(p, &p->d_eq, n * (size_t)(p->m + 1)));
    BNM_CUDA_TRY(dalloc(p, &p->d_cost, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_pen, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_fcc, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_fcdiff, n));
    BNM_CUDA_TRY(dalloc(p, &p->d_ks, n));
    if (p->cfg.gram != BNM_GRAM_F32) {
        const int parts = p->cfg.gram == BNM_GRAM_BF16_SPLIT ? 2 : 1;
        auto blocks = [](int64_t x, int b) { return (int)((x + b - 1) / b); };
        p->fc_rb = blocks(N, kGramTileRows);
        p->fc_kb = blocks(s.corr_len, kGramTileK);
        const size_t fc_bytes = n * p->fc_rb * p->fc_kb * (size_t)kGramTileBytes;
        BNM_CUDA_TRY(dalloc(p, &p->d_fc_hi, fc_bytes));
        if (parts == 2) BNM_CUDA_TRY(dalloc(p, &p->d_fc_lo, fc_bytes));
        std::vector<int> map((size_t)N * (N - 1) / 2, -1);
        for (size_t q = 0; q < pi.size(); q++) map[(size_t)pi[q] * (pi[q] - 1) / 2 + pj[q]] = (int)q;
        BNM_CUDA_TRY(dalloc(p, &p->d_tril_map, map.size()));
        BNM_CUDA_TRY(cudaMemcpy(p->d_tril_map, map.data(), map.size() * 4, cudaMemcpyHostToDevice));
        if (!cfg->no_fcd) {
            // FCD operands are large (W x pairs per sim); stage at most 4 GiB of them
            p->fcd_rb = blocks(s.n_windows, kGramTileRows);
            p->fcd_kb = blocks(s.n_pairs, kGramTileK);
            const size_t per_sim = (size_t)p->fcd_rb * p->fcd_kb * kGramTileBytes;
            const size_t budget = (size_t)4 << 30;
            p->gram_chunk = (int)std::max<size_t>(1, std::min<size_t>(n, budget / (per_sim * parts)));
            // BNM_B200_GRAM_CHUNK caps the simulations per staged chunk
            if (const char* e = std::getenv("BNM_B200_GRAM_CHUNK"))
                if (std::atoi(e) > 0) p->gram_chunk = std::min(p->gram_chunk, std::atoi(e));
            BNM_CUDA_TRY(dalloc(p, &p->d_fcd_hi, per_sim * p->gram_chunk));
            if (parts == 2) BNM_CUDA_TRY(dalloc(p, &p->d_fcd_lo, per_sim * p->gram_chunk));
        }
        const int pairs = 1 + (cfg->no_fcd ? 0 : (int)((n + p->gram_chunk - 1) / std::max(p->gram_chunk, 1)));
        p->gev.assign(2 * pairs, nullptr);
        for (auto& e : p->gev) BNM_CUDA_TRY(cudaEventCreate(&e));
    }
    BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
    return BNM_OK;
}

extern "C" int bnm_plan_create(const bnm_config* cfg, const double* sc, const double* emp_fc, int32_t n_emp_fc,
                               const double* emp_fcd, int32_t n_emp_fcd, const float* host_noise,
                               int64_t n_host_noise, bnm_plan** out) {
    if (!cfg || !out) return fail(BNM_EINVAL, "null argument");
    *out = nullptr;
    bnm_plan* p = new bnm_plan();
    int rc = plan_create(cfg, sc, emp_fc, n_emp_fc, emp_fcd, n_emp_fcd, host_noise, n_host_noise, p);
    if (rc) {
        bnm_plan_destroy(p);
        return rc;
    }
    *out = p;
    return BNM_OK;
}

static std::vector<double> rounded(const double* v, size_t n, bool to_float) {
    std::vector<double> r(v, v + n);
    if (to_float)
        for (auto& x : r) x = (double)(float)x;
    return r;
}

template <typename T>
static int d2h(T* host, const T* dev, size_t n, cudaStream_t st) {
    if (!host) return BNM_OK;
    BNM_CUDA_TRY(cudaMemcpyAsync(host, dev, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    return BNM_OK;
}

static int f2d(double* host, const float* dev, size_t n, cudaStream_t st) {
    if (!host) return BNM_OK;
    std::vector<float> tmp(n);
    BNM_CUDA_TRY(cudaMemcpyAsync(tmp.data(), dev, n * 4, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < n; i++) host[i] = tmp[i];
    return BNM_OK;
}

static int launch_fic(bnm_plan* p, int n) {
    FicArgs fa;
    fa.n_sims = n;
    fa.N = p->cfg.nodes;
    fa.sc = p->d_sc_fic;
    fa.G = p->d_G;
    fa.wEE = p->d_wEE;
    fa.wEI = p->d_wEI;
    fa.wIE = p->d_wIE;
    fa.unstable = p->d_unstable;
    fa.fp32_consts = p->cfg.precision == BNM_PREC_F32_REF;
    BNM_CUDA_TRY(bnm_launch_analytic_fic(fa, p->st));
    return BNM_OK;
}

static int upload_params(bnm_plan* p, int n, const double* G, const double* w_ee, const double* w_ei) {
    const int N = p->cfg.nodes;
    const bool rf = p->cfg.precision == BNM_PREC_F32_REF;
    for (int i = 0; i < n; i++)
        if (!std::isfinite(G[i])) return fail(BNM_EINVAL, "G[%d] is not finite", i);
    for (size_t i = 0; i < (size_t)n * N; i++)
        if (!std::isfinite(w_ee[i]) || !std::isfinite(w_ei[i])) return fail(BNM_EINVAL, "wEE/wEI not finite at %zu", i);
    auto g = rounded(G, n, rf), we = rounded(w_ee, (size_t)n * N, rf), wi = rounded(w_ei, (size_t)n * N, rf);
    BNM_CUDA_TRY(cudaMemcpyAsync(p->d_G, g.data(), n * 8, cudaMemcpyHostToDevice, p->st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->d_wEE, we.data(), (size_t)n * N * 8, cudaMemcpyHostToDevice, p->st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->d_wEI, wi.data(), (size_t)n * N * 8, cudaMemcpyHostToDevice, p->st));
    BNM_CUDA_TRY(cudaStreamSynchronize(p->st));  // host vectors go out of scope
    return BNM_OK;
}

// Autotuner of the FP32 integrator: times every candidate shape of
// bnm_integrator_candidates on this batch size over 200 simulated
// milliseconds without FIC (the per-millisecond cost does not depend on the
// model time) and keeps the fastest.  With `share` (plans of a group, which
// run side by side and split the SMs) the score is the time weighted by the
// fraction of the GPU the launch fills (bnm_integrator_share): SM time, not
// latency.  A plan keeps the shape of its first tuning for a batch size,
// whichever path ran it, so the same inputs give the same results through
// bnm_run and through a group.  BNM_B200_SHAPE="kind,slots,csize,rpw,kr"
// forces a shape; BNM_B200_SLOTS forces the register kernel's slots;
// BNM_B200_TUNE=0 takes the first candidate untimed.
static int tune_integrator(bnm_plan* p, const SimArgs& a, bool share = false) {
    const int n = a.n_sims;
    if (p->tuned_n == n) return BNM_OK;
    IntegratorShape cand[128];
    const int nc = bnm_integrator_candidates(a.N, cand, 128);
    if (nc < 1) return fail(BNM_EINVAL, "no FP32 integrator for %d nodes", a.N);
    p->shape = cand[0];
    p->n_tried = 0;
    if (const char* e = std::getenv("BNM_B200_SHAPE")) {
        IntegratorShape s{};
        if (std::sscanf(e, "%d,%d,%d,%d,%d", &s.kind, &s.slots, &s.csize, &s.rpw, &s.kr) != 5)
            return fail(BNM_EINVAL, "BNM_B200_SHAPE must be kind,slots,csize,rpw,kr");
        p->shape = s;
        p->tuned_n = n;
        return BNM_OK;
    }
    const char* slots = std::getenv("BNM_B200_SLOTS");
    if (slots && p->shape.kind == 0) {
        p->shape.slots = std::atoi(slots) == 2 ? 2 : 1;
        p->tuned_n = n;
        return BNM_OK;
    }
    const char* tune = std::getenv("BNM_B200_TUNE");
    if ((tune && std::atoi(tune) == 0) || nc == 1) {
        p->tuned_n = n;
        return BNM_OK;
    }
    SimArgs t = a;
    t.T = std::min(a.T, 200);
    t.adjust_fic = 0;
    t.order = nullptr;  // shapes are timed on claim order
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_status, 0, 16, p->st));
    double best = 1e300;
    for (int i = 0; i < nc; i++) {
        // shapes that integrate two particles together compute an idle one for a batch of one
        if (n < 2 && ((cand[i].kind == 0 && cand[i].slots == 2) || cand[i].kind == 4)) continue;
        float ms = 0.f;
        bool ok = true;
        for (int rep = 0; rep < 2 && ok; rep++) {  // the first launch also loads the kernel
            BNM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, 16, p->st));
            BNM_CUDA_TRY(cudaEventRecord(p->tev[0], p->st));
            ok = bnm_launch_integrate_shape(t, cand[i], p->num_sms, p->st) == cudaSuccess;
            BNM_CUDA_TRY(cudaEventRecord(p->tev[1], p->st));
        }
        cudaGetLastError();  // a shape that cannot launch is skipped
        BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
        int st_word = 0;
        BNM_CUDA_TRY(cudaMemcpy(&st_word, p->d_status, 4, cudaMemcpyDeviceToHost));
        if (st_word)
            return fail(BNM_ETIMEOUT, "integrator tuning: shape %d,%d,%d,%d,%d for N=%d n=%d left status 0x%x",
                        cand[i].kind, cand[i].slots, cand[i].csize, cand[i].rpw, cand[i].kr, a.N, n, st_word);
        if (!ok) continue;
        BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->tev[0], p->tev[1]));
        p->n_tried++;
        const double score = share ? ms * bnm_integrator_share(t, cand[i], p->num_sms) : ms;
        if (score < best) {
            best = score;
            p->shape = cand[i];
        }
    }
    int status = 0;
    BNM_CUDA_TRY(cudaMemcpy(&status, p->d_status, 4, cudaMemcpyDeviceToHost));
    if (status) return fail(BNM_ETIMEOUT, "integrator tuning run reported status %d", status);
    p->tuned_n = n;
    return BNM_OK;
}

extern "C" int bnm_plan_integrator(bnm_plan* p, int32_t* out5, int32_t* n_tried) {
    if (!p || !out5) return fail(BNM_EINVAL, "null argument");
    out5[0] = p->shape.kind;
    out5[1] = p->shape.slots;
    out5[2] = p->shape.csize;
    out5[3] = p->shape.rpw;
    out5[4] = p->shape.kr;
    if (n_tried) *n_tried = p->n_tried;
    return BNM_OK;
}

extern "C" int bnm_analytic_fic(bnm_plan* p, int32_t n, const double* G, const double* w_ee, const double* w_ei,
                                double* w_ie_out, int32_t* unstable_out) {
    if (!p || n < 1 || n > p->cfg.max_sims) return fail(BNM_EINVAL, "n must be in [1, max_sims]");
    BNM_CUDA_TRY(cudaSetDevice(p->cfg.device));
    int rc = upload_params(p, n, G, w_ee, w_ei);
    if (rc) return rc;
    if ((rc = launch_fic(p, n))) return rc;
    if ((rc = d2h(w_ie_out, p->d_wIE, (size_t)n * p->cfg.nodes, p->st))) return rc;
    if ((rc = d2h(unstable_out, p->d_unstable, n, p->st))) return rc;
    BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
    return BNM_OK;
}

// Stage event: inside a graph capture it must become an event-record node
// (external record) to time anything when the graph runs.
static cudaError_t rec(bnm_plan* p, cudaEvent_t e) {
    return p->capturing ? cudaEventRecordWithFlags(e, p->st, cudaEventRecordExternal) : cudaEventRecord(e, p->st);
}

// FC + window FC (+ tensor-core FC Gram), FCD + KS histogram, goodness of
// fit, on the plan's BOLD buffer; events 3, 4, 5 close the stages.
// Hemisphere FCD buffers, allocated the first time a caller asks for them.
static int ensure_hemi(bnm_plan* p) {
    if (p->d_fcd_hemi) return BNM_OK;
    const int N = p->cfg.nodes, h = N / 2;
    if (p->cfg.no_fcd || h * (h - 1) / 2 < 2)
        return fail(BNM_EINVAL, "hemisphere FCDs need FCD and at least 3 nodes per hemisphere");
    const size_t n = p->cfg.max_sims, W = std::max(p->sz.n_windows, 1);
    BNM_CUDA_TRY(dalloc(p, &p->d_fcd_hemi, 2 * n * std::max(p->sz.n_fcd, 1)));
    BNM_CUDA_TRY(dalloc(p, &p->d_wsum_hemi, 2 * n * W * 2));
    return BNM_OK;
}

static int launch_analysis(bnm_plan* p, int n, int calc_fic_penalty, bool hemis = false);

// Window FC + static FC of the plan's BOLD buffer (fc_window_kernel).
static FcArgs fc_args(bnm_plan* p, int n) {
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    FcArgs fa;
    std::memset(&fa, 0, sizeof fa);
    fa.ppt = p->win_ppt;
    fa.N = c.nodes;
    fa.n_sims = n;
    fa.frames = s.frames;
    fa.n_vols_remove = s.n_vols_remove;
    fa.corr_len = s.corr_len;
    fa.P = s.n_pairs;
    fa.pair_i = p->d_pi;
    fa.pair_j = p->d_pj;
    fa.W = c.no_fcd ? 0 : s.n_windows;
    fa.win_len = s.window_len;
    fa.win_step = c.window_step;
    fa.bold = p->d_bold;
    fa.bold_f64 = p->d_bold64;
    fa.fc = p->d_fc;
    fa.wfc = p->d_wfc;
    fa.wsum = p->d_wsum;
    fa.nan_flag = p->d_nan;
    return fa;
}

static int launch_window_only(bnm_plan* p, int n) {
    BNM_CUDA_TRY(bnm_launch_fc_window(fc_args(p, n), p->st));
    return BNM_OK;
}

// Window-tile tuner: times the window-FC kernel with 1, 2, 4 and 8 pairs per
// thread (256, 512, 1024 and 2048 pairs per CTA) on this batch size and keeps
// the fastest, on the first run of each batch size (BNM_B200_TUNE=0: 4).  The
// timing launches accumulate into the NaN flags, which are cleared afterwards.
static int tune_window(bnm_plan* p, int n) {
    if (p->win_tuned_n == n) return BNM_OK;
    const char* tune = std::getenv("BNM_B200_TUNE");
    p->win_ppt = 4;
    p->win_tried = 0;
    if (!(tune && std::atoi(tune) == 0)) {
        double best = 1e300;
        for (int ppt : {1, 2, 4, 8}) {
            const int saved = p->win_ppt;
            p->win_ppt = ppt;
            float ms = 0.f;
            bool ok = true;
            for (int rep = 0; rep < 2 && ok; rep++) {  // the first launch also loads the kernel
                BNM_CUDA_TRY(cudaEventRecord(p->tev[0], p->st));
                const int launches = p->launches;
                ok = launch_window_only(p, n) == BNM_OK;
                p->launches = launches;
                BNM_CUDA_TRY(cudaEventRecord(p->tev[1], p->st));
            }
            cudaGetLastError();  // a tile that cannot launch is skipped
            BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
            if (!ok) {
                p->win_ppt = saved;
                continue;
            }
            BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->tev[0], p->tev[1]));
            p->win_tried++;
            if (ms < best) best = ms;
            else p->win_ppt = saved;
        }
    }
    const size_t W = std::max(p->sz.n_windows, 1);
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_wsum, 0, (size_t)n * W * 2 * 8, p->st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_nan, 0, n * 4, p->st));
    p->win_tuned_n = n;
    return BNM_OK;
}

static int launch_analysis(bnm_plan* p, int n, int calc_fic_penalty, bool hemis) {
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    const int N = c.nodes;
    cudaStream_t st = p->st;
    p->n_gram = 0;
    p->launches += c.no_fcd ? 2 : 3;  // window FC (+ window sums) and goodness of fit

    BNM_CUDA_TRY(bnm_launch_fc_window(fc_args(p, n), st));
    const int split = c.gram == BNM_GRAM_BF16_SPLIT;
    if (c.gram != BNM_GRAM_F32) {
        // FC again as a tensor-core Gram; it replaces the co-moment FC in d_fc
        OperandArgs oa;
        std::memset(&oa, 0, sizeof oa);
        oa.n_sims = n;
        oa.rows = N;
        oa.K = s.corr_len;
        oa.row_blocks = p->fc_rb;
        oa.kblocks = p->fc_kb;
        oa.bold = p->d_bold;
        oa.bold_f64 = p->d_bold64;
        oa.frames = s.frames;
        oa.n_vols_remove = s.n_vols_remove;
        oa.hi = p->d_fc_hi;
        oa.lo = p->d_fc_lo;
        BNM_CUDA_TRY(bnm_launch_fc_operand(oa, st));
        GramArgs ga;
        std::memset(&ga, 0, sizeof ga);
        ga.n_sims = n;
        ga.rows = N;
        ga.row_blocks = p->fc_rb;
        ga.kblocks = p->fc_kb;
        ga.hi = p->d_fc_hi;
        ga.lo = p->d_fc_lo;
        ga.out = p->d_fc;
        ga.tril_map = p->d_tril_map;
        ga.out_ld = s.n_pairs;
        ga.nan_flag = p->d_nan;
        ga.status = p->d_status;
        BNM_CUDA_TRY(rec(p, p->gev[0]));
        BNM_CUDA_TRY(bnm_launch_gram_tc(ga, split, st));
        BNM_CUDA_TRY(rec(p, p->gev[1]));
        p->n_gram = 1;
        p->launches += 2;
    }
    BNM_CUDA_TRY(rec(p, p->ev[3]));

    if (!c.no_fcd && c.gram != BNM_GRAM_F32) {
        for (int c0 = 0; c0 < n; c0 += p->gram_chunk) {
            const int cn = std::min(p->gram_chunk, n - c0);
            OperandArgs oa;
            std::memset(&oa, 0, sizeof oa);
            oa.n_sims = cn;
            oa.rows = s.n_windows;
            oa.K = s.n_pairs;
            oa.row_blocks = p->fcd_rb;
            oa.kblocks = p->fcd_kb;
            oa.wfc = p->d_wfc + (size_t)c0 * s.n_windows * s.n_pairs;
            oa.wsum = p->d_wsum + (size_t)c0 * s.n_windows * 2;
            oa.hi = p->d_fcd_hi;
            oa.lo = p->d_fcd_lo;
            BNM_CUDA_TRY(bnm_launch_fcd_operand(oa, st));
            GramArgs ga;
            std::memset(&ga, 0, sizeof ga);
            ga.n_sims = cn;
            ga.rows = s.n_windows;
            ga.row_blocks = p->fcd_rb;
            ga.kblocks = p->fcd_kb;
            ga.hi = p->d_fcd_hi;
            ga.lo = p->d_fcd_lo;
            ga.out = p->d_fcd + (size_t)c0 * s.n_fcd;
            ga.out_ld = s.n_fcd;
            ga.emp_sorted = p->d_emp_sorted;
            ga.ks_lut = p->d_ks_lut;
            ga.m = p->m;
            ga.hist = p->d_hist + (size_t)c0 * (p->m + 1);
            ga.eq = p->d_eq + (size_t)c0 * (p->m + 1);
            ga.nan_flag = p->d_nan + c0;
            ga.status = p->d_status;
            BNM_CUDA_TRY(rec(p, p->gev[2 * p->n_gram]));
            BNM_CUDA_TRY(bnm_launch_gram_tc(ga, split, st));
            BNM_CUDA_TRY(rec(p, p->gev[2 * p->n_gram + 1]));
            p->n_gram++;
            p->launches += 2;
        }
    } else if (!c.no_fcd) {
        FcdArgs da;
        da.n_sims = n;
        da.W = s.n_windows;
        da.P = s.n_pairs;
        da.wfc = p->d_wfc;
        da.wsum = p->d_wsum;
        da.fcd = p->d_fcd;
        da.n_fcd = s.n_fcd;
        da.emp_sorted = p->d_emp_sorted;
        da.ks_lut = p->d_ks_lut;
        da.p0 = 0;
        da.p1 = s.n_pairs;
        da.m = p->m;
        da.hist = p->d_hist;
        da.eq = p->d_eq;
        da.nan_flag = p->d_nan;
        BNM_CUDA_TRY(bnm_launch_fcd(da, st));
        p->launches++;
    }
    if (hemis) {
        // left / right hemisphere FCD over the first / last (N/2)(N/2-1)/2 pairs,
        // each centred over its own pairs (window_fc_stats + fcd with save_hemis,
        // bnm.cu:436-551); not part of the cost
        const int h = N / 2, nh = h * (h - 1) / 2;
        const size_t W = std::max(s.n_windows, 1), nmax = c.max_sims;
        for (int side = 0; side < 2; side++) {
            const int p0 = side == 0 ? 0 : s.n_pairs - nh, p1 = side == 0 ? nh : s.n_pairs;
            double* ws = p->d_wsum_hemi + side * nmax * W * 2;
            BNM_CUDA_TRY(bnm_launch_window_sums(p->d_wfc, n, s.n_windows, s.n_pairs, p0, p1, ws, st));
            FcdArgs da;
            std::memset(&da, 0, sizeof da);
            da.n_sims = n;
            da.W = s.n_windows;
            da.P = s.n_pairs;
            da.wfc = p->d_wfc;
            da.wsum = ws;
            da.fcd = p->d_fcd_hemi + side * nmax * s.n_fcd;
            da.n_fcd = s.n_fcd;
            da.p0 = p0;
            da.p1 = p1;
            BNM_CUDA_TRY(bnm_launch_fcd(da, st));
            p->launches += 2;
        }
    }
    BNM_CUDA_TRY(rec(p, p->ev[4]));

    GofArgs ga;
    ga.n_sims = n;
    ga.N = N;
    ga.P = s.n_pairs;
    ga.n_fcd = s.n_fcd;
    ga.m = p->m;
    ga.fc = p->d_fc;
    ga.emp_fc = p->d_emp_fc;
    ga.emp_fc_mean = p->emp_fc_mean;
    ga.hist = p->d_hist;
    ga.eq = p->d_eq;
    ga.valid = p->d_valid;
    ga.ext = p->d_ext;
    ga.failed = p->d_failed;
    ga.nan_flag = p->d_nan;
    ga.use_fc_diff = c.use_fc_diff;
    ga.calc_fic_penalty = calc_fic_penalty;
    ga.fic_reject_failed = c.fic_reject_failed;
    ga.no_fcd = c.no_fcd;
    ga.max_cost = c.max_cost;
    ga.fic_penalty_scale = c.fic_penalty_scale;
    ga.cost = p->d_cost;
    ga.fic_penalty = p->d_pen;
    ga.fc_corr = p->d_fcc;
    ga.fc_diff = p->d_fcdiff;
    ga.fcd_ks = p->d_ks;
    BNM_CUDA_TRY(bnm_launch_gof(ga, st));
    BNM_CUDA_TRY(rec(p, p->ev[5]));

    return BNM_OK;
}

// Copies the requested outputs back, reads the stage timings and the device
// status word.
static int finish(bnm_plan* p, int n, bnm_batch_out* out, bool integrated) {
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    const int N = c.nodes;
    cudaStream_t st = p->st;
    int rc;
    int status = 0;
    BNM_CUDA_TRY(cudaMemcpyAsync(&status, p->d_status, 4, cudaMemcpyDeviceToHost, st));
    if ((rc = d2h(out->cost, p->d_cost, n, st))) return rc;
    if ((rc = d2h(out->fic_penalty, p->d_pen, n, st))) return rc;
    if ((rc = d2h(out->fc_corr, p->d_fcc, n, st))) return rc;
    if ((rc = d2h(out->fc_diff, p->d_fcdiff, n, st))) return rc;
    if ((rc = d2h(out->fcd_ks, p->d_ks, n, st))) return rc;
    if (integrated) {
        if ((rc = d2h(out->w_ie, p->d_wIE_out, (size_t)n * N, st))) return rc;
        if ((rc = d2h(out->fic_failed, p->d_failed, n, st))) return rc;
        if ((rc = d2h(out->fic_ntrials, p->d_trials, n, st))) return rc;
        if ((rc = d2h(out->fic_unstable, p->d_unstable, n, st))) return rc;
        if ((rc = d2h(out->ext_means, p->d_ext, (size_t)n * 6 * N, st))) return rc;
    }
    if (integrated && out->bold) {
        if (c.precision == BNM_PREC_F64)
            rc = d2h(out->bold, p->d_bold64, (size_t)n * s.frames * N, st);
        else
            rc = f2d(out->bold, p->d_bold, (size_t)n * s.frames * N, st);
        if (rc) return rc;
    }
    if ((rc = f2d(out->fc, p->d_fc, (size_t)n * s.n_pairs, st))) return rc;
    if (!c.no_fcd && (rc = f2d(out->fcd, p->d_fcd, (size_t)n * s.n_fcd, st))) return rc;
    if (p->d_fcd_hemi) {
        const size_t nmax = c.max_sims;
        if ((rc = f2d(out->fcd_left, p->d_fcd_hemi, (size_t)n * s.n_fcd, st))) return rc;
        if ((rc = f2d(out->fcd_right, p->d_fcd_hemi + nmax * s.n_fcd, (size_t)n * s.n_fcd, st))) return rc;
    }
    BNM_CUDA_TRY(cudaStreamSynchronize(st));
    float ms;
    for (int i = 0; i < 5; i++) {
        BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->ev[i], p->ev[i + 1]));
        p->timings[i] = ms;
    }
    BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->ev[0], p->ev[5]));
    p->timings[5] = ms;
    p->gram_ms[0] = p->gram_ms[1] = 0;
    for (int g = 0; g < p->n_gram; g++) {
        BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->gev[2 * g], p->gev[2 * g + 1]));
        p->gram_ms[g == 0 ? 0 : 1] += ms;
    }
    if (status & kStatusTimeout) return fail(BNM_ETIMEOUT, "a device wait gave up (status %d)", status);
    if (status) return fail(BNM_ECUDA, "device status %d", status);
    return BNM_OK;
}

static SimArgs sim_args(bnm_plan* p, int n) {
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    SimArgs a;
    std::memset(&a, 0, sizeof a);
    a.N = c.nodes;
    a.n_sims = n;
    a.T = c.time_steps;
    a.TR = c.bold_tr;
    a.frames = s.frames;
    a.n_vols_remove = s.n_vols_remove;
    a.adjust_fic = c.do_fic && c.numerical_fic;
    a.max_trials = c.max_fic_trials;
    a.samp_start = c.i_sampling_start;
    a.samp_end = c.i_sampling_end;
    a.init_delta = c.init_delta;
    a.G = p->d_G;
    a.wEE = p->d_wEE;
    a.wEI = p->d_wEI;
    a.wIE = p->d_wIE;
    a.order = p->place ? p->d_order : nullptr;
    a.place_ws = p->d_place_ws;
    a.noise = p->d_noise;  // NULL: the register integrator draws Philox noise in place
    a.noise_seed = c.noise_seed;
    a.noise_ld = p->noise_ld;
    a.n_real = c.nodes;
    a.sc_f32 = p->d_sc32;
    a.sc_f64 = p->d_sc64;
    a.sc_ld = p->sc_ld;
    a.bold = p->d_bold;
    a.bold_f64 = p->d_bold64;
    a.wIE_out = p->d_wIE_out;
    a.trials = p->d_trials;
    a.failed = p->d_failed;
    a.ext = p->d_ext;
    a.work_counter = p->d_counter;
    a.status = p->d_status;
    return a;
}

static int ensure_pinned(bnm_plan* p);
static int enqueue_run(bnm_plan* p, int n);
static int read_timings(bnm_plan* p);

// Particle placement (on by default with numerical FIC on the FP32 path: the
// register kernel with a noise table, the column-split clusters;
// BNM_B200_PLACE=0 turns it off).  Column-split clusters of two particles
// integrate io_order's pairs, so the two particles they advance in lockstep
// need about the same number of substeps.  In the register kernel a
// particle that hits the numerical-FIC trial cap integrates about 1 M more
// substeps than one that needs no restart, and with more particles than SMs
// the CTAs share SMs (two per SM, each slower than alone), so the generation
// ends with the heavy particles that shared an SM.  The kernel hands out
// io_order from both ends: the second CTA on an SM takes the lightest
// particles, every other CTA the heaviest, so heavy particles run alone or
// beside light ones.  Work is predicted by the FIC restart count of the
// nearest particle simulated before by this plan (G, mean wEE, mean wEI, each
// scaled by its spread); io_order lists the particles heaviest first.
// Without history (fewer than 16 particles) the order is the identity.  Where
// a particle runs does not change its results.
static void place_particles(bnm_plan* p, int n, const double* G, const double* w_ee, const double* w_ei) {
    const int N = p->cfg.nodes;
    for (int i = 0; i < n; i++) p->io_order[i] = i;
    const size_t H = p->hist_tr.size();
    p->last_placed = H >= 16 && n > 1;
    if (!p->last_placed) return;
    double mu[3] = {0, 0, 0}, sd[3] = {0, 0, 0};
    for (size_t h = 0; h < H; h++)
        for (int d = 0; d < 3; d++) mu[d] += p->hist_x[3 * h + d];
    for (int d = 0; d < 3; d++) mu[d] /= H;
    for (size_t h = 0; h < H; h++)
        for (int d = 0; d < 3; d++) sd[d] += (p->hist_x[3 * h + d] - mu[d]) * (p->hist_x[3 * h + d] - mu[d]);
    for (int d = 0; d < 3; d++) sd[d] = sd[d] > 0 ? std::sqrt(sd[d] / H) : 1.0;
    std::vector<int> pred(n);
    for (int i = 0; i < n; i++) {
        double x[3] = {G[i], 0, 0};
        for (int j = 0; j < N; j++) {
            x[1] += w_ee[(size_t)i * N + j];
            x[2] += w_ei[(size_t)i * N + j];
        }
        x[1] /= N;
        x[2] /= N;
        double best = 1e300;
        for (size_t h = 0; h < H; h++) {
            double d2 = 0;
            for (int d = 0; d < 3; d++) {
                const double t = (x[d] - p->hist_x[3 * h + d]) / sd[d];
                d2 += t * t;
            }
            if (d2 < best) {
                best = d2;
                pred[i] = p->hist_tr[h];
            }
        }
    }
    std::stable_sort(p->io_order, p->io_order + n, [&](int a, int b) { return pred[a] > pred[b]; });
}

// Appends the last batch's particles and FIC restart counts to the placement history.
static void record_particles(bnm_plan* p, int n, const double* G, const double* w_ee, const double* w_ei,
                             const int* trials) {
    const int N = p->cfg.nodes;
    const size_t cap = 4096;  // the most recent particles (a few generations)
    for (int i = 0; i < n; i++) {
        float x[3] = {(float)G[i], 0.f, 0.f};
        double e = 0, f = 0;
        for (int j = 0; j < N; j++) {
            e += w_ee[(size_t)i * N + j];
            f += w_ei[(size_t)i * N + j];
        }
        x[1] = (float)(e / N);
        x[2] = (float)(f / N);
        if (p->hist_tr.size() < cap) {
            p->hist_x.insert(p->hist_x.end(), x, x + 3);
            p->hist_tr.push_back(trials[i]);
        } else {
            const size_t h = p->hist_next++ % cap;
            std::copy(x, x + 3, p->hist_x.begin() + 3 * h);
            p->hist_tr[h] = trials[i];
        }
    }
}

// A generation of a plan whose integrator is already tuned for n particles,
// with analytic FIC on the device: parameters staged through pinned host
// buffers, then one graph launch (the same stream operations as the eager
// path: parameter upload, analytic FIC, integrator, window FC, Grams, KS,
// goodness of fit, result download), captured on the first such call for n.
// Optional large outputs (BOLD, FC, FCD, extended means) are copied from the
// device buffers after the launch.
static int run_graph(bnm_plan* p, int n, const double* G, const double* w_ee, const double* w_ei,
                     bnm_batch_out* out) {
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    const int N = c.nodes;
    int rc = ensure_pinned(p);
    if (rc) return rc;
    for (int i = 0; i < n; i++) {
        if (!std::isfinite(G[i])) return fail(BNM_EINVAL, "G[%d] is not finite", i);
        p->io_G[i] = G[i];
    }
    for (size_t i = 0; i < (size_t)n * N; i++) {
        if (!std::isfinite(w_ee[i]) || !std::isfinite(w_ei[i])) return fail(BNM_EINVAL, "wEE/wEI not finite at %zu", i);
        p->io_wEE[i] = w_ee[i];
        p->io_wEI[i] = w_ei[i];
    }
    if (p->place) place_particles(p, n, G, w_ee, w_ei);
    cudaStream_t st = p->st;
    if (!p->run_exec || p->run_graph_n != n) {
        if (p->run_exec) cudaGraphExecDestroy(p->run_exec);
        if (p->run_graph) cudaGraphDestroy(p->run_graph);
        p->run_exec = nullptr;
        p->run_graph = nullptr;
        p->run_graph_n = 0;
        BNM_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        p->capturing = true;
        rc = enqueue_run(p, n);
        p->capturing = false;
        cudaGraph_t graph = nullptr;
        const cudaError_t e_end = cudaStreamEndCapture(st, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        BNM_CUDA_TRY(e_end);
        p->run_graph = graph;
        BNM_CUDA_TRY(cudaGraphInstantiate(&p->run_exec, graph, 0));
        p->run_graph_n = n;
    }
    BNM_CUDA_TRY(cudaGraphLaunch(p->run_exec, st));
    p->last_graph = 1;
    if (out->bold) rc = f2d(out->bold, p->d_bold, (size_t)n * s.frames * N, st);
    if (!rc) rc = d2h(out->ext_means, p->d_ext, (size_t)n * 6 * N, st);
    if (!rc) rc = f2d(out->fc, p->d_fc, (size_t)n * s.n_pairs, st);
    if (!rc && !c.no_fcd) rc = f2d(out->fcd, p->d_fcd, (size_t)n * s.n_fcd, st);
    if (rc) return rc;
    BNM_CUDA_TRY(cudaStreamSynchronize(st));
    if ((rc = read_timings(p))) return rc;
    const int status = *p->io_status;
    if (status & kStatusTimeout) return fail(BNM_ETIMEOUT, "a device wait gave up (status %d)", status);
    if (status) return fail(BNM_ECUDA, "device status %d", status);
    auto put = [](auto* dst, const auto* src, size_t cnt) {
        if (dst) std::copy(src, src + cnt, dst);
    };
    put(out->cost, p->io_cost, n);
    put(out->fic_penalty, p->io_pen, n);
    put(out->fc_corr, p->io_fcc, n);
    put(out->fc_diff, p->io_fcdiff, n);
    put(out->fcd_ks, p->io_ks, n);
    put(out->w_ie, p->io_wie, (size_t)n * N);
    put(out->fic_failed, p->io_failed, n);
    put(out->fic_ntrials, p->io_trials, n);
    put(out->fic_unstable, p->io_unstable, n);
    if (p->place) record_particles(p, n, G, w_ee, w_ei, p->io_trials);
    return BNM_OK;
}

extern "C" int bnm_run(bnm_plan* p, int32_t n, const double* G, const double* w_ee, const double* w_ei,
                       const double* w_ie, bnm_batch_out* out) {
    if (!p || !out || !G || !w_ee || !w_ei) return fail(BNM_EINVAL, "null argument");
    if (n < 1 || n > p->cfg.max_sims) return fail(BNM_EINVAL, "n=%d outside [1, max_sims=%d]", n, p->cfg.max_sims);
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    const int N = c.nodes;
    if (!c.do_fic && !w_ie) return fail(BNM_EINVAL, "w_ie is required when do_fic == 0");
    BNM_CUDA_TRY(cudaSetDevice(c.device));
    const bool hemis = out->fcd_left || out->fcd_right;
    const bool device_fic = c.do_fic && !w_ie;
    // after the first (tuning) run of a batch size, the generation is one graph launch
    const char* ge = std::getenv("BNM_B200_GRAPH");
    if (device_fic && !hemis && c.precision == BNM_PREC_F32 && p->tuned_n == n && p->win_tuned_n == n &&
        !(ge && !std::strcmp(ge, "0")))
        return run_graph(p, n, G, w_ee, w_ei, out);
    p->last_graph = 0;
    int rc = hemis ? ensure_hemi(p) : BNM_OK;
    if (rc) return rc;
    if ((rc = upload_params(p, n, G, w_ee, w_ei))) return rc;
    cudaStream_t st = p->st;
    BNM_CUDA_TRY(cudaEventRecord(p->ev[0], st));
    p->launches = device_fic ? 2 : 1;  // analytic FIC, integrator
    if (device_fic) {
        if ((rc = launch_fic(p, n))) return rc;
    } else {
        auto wi = rounded(w_ie, (size_t)n * N, c.precision == BNM_PREC_F32_REF);
        for (double v : wi)
            if (!std::isfinite(v)) return fail(BNM_EINVAL, "wIE not finite");
        BNM_CUDA_TRY(cudaMemcpyAsync(p->d_wIE, wi.data(), wi.size() * 8, cudaMemcpyHostToDevice, st));
        BNM_CUDA_TRY(cudaMemsetAsync(p->d_unstable, 0, n * 4, st));
        BNM_CUDA_TRY(cudaStreamSynchronize(st));
    }
    BNM_CUDA_TRY(cudaEventRecord(p->ev[1], st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, 16, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_status, 0, 16, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_nan, 0, n * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_wsum, 0, (size_t)n * std::max(s.n_windows, 1) * 2 * 8, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_hist, 0, (size_t)n * (p->m + 1) * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_eq, 0, (size_t)n * (p->m + 1) * 4, st));

    const SimArgs a = sim_args(p, n);
    if (c.precision == BNM_PREC_F32) {
        if ((rc = tune_integrator(p, a))) return rc;
        BNM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, 16, st));
        BNM_CUDA_TRY(cudaMemsetAsync(p->d_status, 0, 16, st));
        if (p->place) {
            BNM_CUDA_TRY(cudaStreamSynchronize(st));  // the tuner's launches may still read the order
            place_particles(p, n, G, w_ee, w_ei);
            BNM_CUDA_TRY(cudaMemcpyAsync(p->d_order, p->io_order, n * 4, cudaMemcpyHostToDevice, st));
            BNM_CUDA_TRY(cudaMemsetAsync(p->d_place_ws, 0, kPlaceWs * 4, st));
        }
        BNM_CUDA_TRY(bnm_launch_integrate_shape(a, p->shape, p->num_sms, st));
    }
    else
        BNM_CUDA_TRY(bnm_launch_integrate_exact(a, c.precision == BNM_PREC_F64, p->num_sms, st));
    if ((rc = tune_window(p, n))) return rc;
    BNM_CUDA_TRY(cudaEventRecord(p->ev[2], st));
    if ((rc = launch_analysis(p, n, c.calculate_fic_penalty, hemis))) return rc;
    rc = finish(p, n, out, true);
    if (!rc && p->place) {
        std::vector<int> tr(n);
        BNM_CUDA_TRY(cudaMemcpy(tr.data(), p->d_trials, n * 4, cudaMemcpyDeviceToHost));
        record_particles(p, n, G, w_ee, w_ei, tr.data());
    }
    return rc;
}

// Goodness of fit of given BOLD series (check_fit_bold, check_fit.cpp:138-217,
// for a batch): bold holds n series of corr_len kept frames x nodes (the
// frames after n_vols_remove), particle-major.  Same FC / FCD / KS / cost as
// bnm_run on the plan's configuration and targets; no FIC penalty (there is
// no r_E series), so cost = 1 - r(FC) (+ |dmean FC|) + KS.
extern "C" int bnm_check_fit_bold(bnm_plan* p, int32_t n, const double* bold, bnm_batch_out* out) {
    if (!p || !out || !bold) return fail(BNM_EINVAL, "null argument");
    if (n < 1 || n > p->cfg.max_sims) return fail(BNM_EINVAL, "n=%d outside [1, max_sims=%d]", n, p->cfg.max_sims);
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    const int N = c.nodes;
    BNM_CUDA_TRY(cudaSetDevice(c.device));
    cudaStream_t st = p->st;
    const size_t per = (size_t)s.corr_len * N, full = (size_t)s.frames * N;
    if (c.precision == BNM_PREC_F64) {
        for (int i = 0; i < n; i++)
            BNM_CUDA_TRY(cudaMemcpyAsync(p->d_bold64 + i * full + (size_t)s.n_vols_remove * N, bold + i * per,
                                         per * 8, cudaMemcpyHostToDevice, st));
    } else {
        std::vector<float> tmp((size_t)n * per);
        for (size_t k = 0; k < tmp.size(); k++) tmp[k] = (float)bold[k];
        for (int i = 0; i < n; i++)
            BNM_CUDA_TRY(cudaMemcpyAsync(p->d_bold + i * full + (size_t)s.n_vols_remove * N, tmp.data() + i * per,
                                         per * 4, cudaMemcpyHostToDevice, st));
        BNM_CUDA_TRY(cudaStreamSynchronize(st));  // tmp goes out of scope
    }
    int rc = tune_window(p, n);
    if (rc) return rc;
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_status, 0, 16, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_nan, 0, n * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_failed, 0, n * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_ext, 0, (size_t)n * 6 * N * 8, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_wsum, 0, (size_t)n * std::max(s.n_windows, 1) * 2 * 8, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_hist, 0, (size_t)n * (p->m + 1) * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_eq, 0, (size_t)n * (p->m + 1) * 4, st));
    for (int e = 0; e < 3; e++) BNM_CUDA_TRY(cudaEventRecord(p->ev[e], st));
    p->launches = 0;
    const bool hemis = out->fcd_left || out->fcd_right;
    rc = hemis ? ensure_hemi(p) : BNM_OK;
    if (rc) return rc;
    rc = launch_analysis(p, n, 0, hemis);
    if (rc) return rc;
    return finish(p, n, out, false);
}


// ------------------------------------------------------------ groups
//
// Several plans (subjects of different node counts) run as one CUDA graph per
// call: each plan's stages on its own stream, forked from and joined to an
// origin stream, with inputs and outputs staged through pinned host buffers
// so the whole generation is one graph launch and one host synchronisation.

static int ensure_pinned(bnm_plan* p) {
    if (p->pinned) return BNM_OK;
    const size_t n = p->cfg.max_sims, N = p->cfg.nodes;
    const size_t doubles = n * 3 * N + n * 5 + n * N, ints = n * 3 + 4;
    BNM_CUDA_TRY(cudaMallocHost((void**)&p->pinned, doubles * 8 + ints * 4));
    double* d = reinterpret_cast<double*>(p->pinned);
    p->io_G = d;
    p->io_wEE = p->io_G + n;
    p->io_wEI = p->io_wEE + n * N;
    p->io_cost = p->io_wEI + n * N;
    p->io_pen = p->io_cost + n;
    p->io_fcc = p->io_pen + n;
    p->io_fcdiff = p->io_fcc + n;
    p->io_ks = p->io_fcdiff + n;
    p->io_wie = p->io_ks + n;
    int* q = reinterpret_cast<int*>(p->io_wie + n * N);
    p->io_failed = q;
    p->io_trials = q + n;
    p->io_unstable = q + 2 * n;
    p->io_status = q + 3 * n;
    return BNM_OK;
}

// One generation of a plan from its pinned inputs to its pinned outputs,
// stream operations only (capturable).  The integrator must be tuned.
static int enqueue_run(bnm_plan* p, int n) {
    const bnm_config& c = p->cfg;
    const bnm_sizes& s = p->sz;
    const int N = c.nodes;
    cudaStream_t st = p->st;
    int rc;
    BNM_CUDA_TRY(cudaMemcpyAsync(p->d_G, p->io_G, n * 8, cudaMemcpyHostToDevice, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->d_wEE, p->io_wEE, (size_t)n * N * 8, cudaMemcpyHostToDevice, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->d_wEI, p->io_wEI, (size_t)n * N * 8, cudaMemcpyHostToDevice, st));
    BNM_CUDA_TRY(rec(p, p->ev[0]));
    p->launches = 2;
    if ((rc = launch_fic(p, n))) return rc;
    BNM_CUDA_TRY(rec(p, p->ev[1]));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, 16, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_status, 0, 16, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_nan, 0, n * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_wsum, 0, (size_t)n * std::max(s.n_windows, 1) * 2 * 8, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_hist, 0, (size_t)n * (p->m + 1) * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->d_eq, 0, (size_t)n * (p->m + 1) * 4, st));
    const SimArgs a = sim_args(p, n);
    if (p->place) {
        BNM_CUDA_TRY(cudaMemcpyAsync(p->d_order, p->io_order, n * 4, cudaMemcpyHostToDevice, st));
        BNM_CUDA_TRY(cudaMemsetAsync(p->d_place_ws, 0, kPlaceWs * 4, st));
    }
    if (c.precision == BNM_PREC_F32)
        BNM_CUDA_TRY(bnm_launch_integrate_shape(a, p->shape, p->num_sms, st));
    else
        BNM_CUDA_TRY(bnm_launch_integrate_exact(a, c.precision == BNM_PREC_F64, p->num_sms, st));
    BNM_CUDA_TRY(rec(p, p->ev[2]));
    if ((rc = launch_analysis(p, n, c.calculate_fic_penalty))) return rc;
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_status, p->d_status, 4, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_cost, p->d_cost, n * 8, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_pen, p->d_pen, n * 8, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_fcc, p->d_fcc, n * 8, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_fcdiff, p->d_fcdiff, n * 8, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_ks, p->d_ks, n * 8, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_wie, p->d_wIE_out, (size_t)n * N * 8, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_failed, p->d_failed, n * 4, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_trials, p->d_trials, n * 4, cudaMemcpyDeviceToHost, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->io_unstable, p->d_unstable, n * 4, cudaMemcpyDeviceToHost, st));
    return BNM_OK;
}

// Stage timings of a finished enqueued run (the events ran on the device).
static int read_timings(bnm_plan* p) {
    float ms;
    for (int i = 0; i < 5; i++) {
        BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->ev[i], p->ev[i + 1]));
        p->timings[i] = ms;
    }
    BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->ev[0], p->ev[5]));
    p->timings[5] = ms;
    p->gram_ms[0] = p->gram_ms[1] = 0;
    for (int g = 0; g < p->n_gram; g++) {
        BNM_CUDA_TRY(cudaEventElapsedTime(&ms, p->gev[2 * g], p->gev[2 * g + 1]));
        p->gram_ms[g == 0 ? 0 : 1] += ms;
    }
    return BNM_OK;
}

struct bnm_group {
    std::vector<bnm_plan*> plans;
    std::vector<int> n;  // batch sizes the graph was captured for
    // plan indices in the order their work is enqueued: largest estimated
    // integration work (N^2 x particles x model time) first
    std::vector<int> order;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double last_ms = 0;
    int graph_launched = 0;
};

extern "C" void bnm_group_destroy(bnm_group* g) {
    if (!g) return;
    if (!g->plans.empty()) cudaSetDevice(g->plans[0]->cfg.device);
    if (g->origin) cudaStreamSynchronize(g->origin);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    for (cudaEvent_t e : g->join)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {g->fork, g->t0, g->t1})
        if (e) cudaEventDestroy(e);
    if (g->origin) cudaStreamDestroy(g->origin);
    delete g;
}

static int group_create(bnm_plan* const* plans, int n_plans, bnm_group* g) {
    for (int i = 0; i < n_plans; i++) {
        if (!plans[i]) return fail(BNM_EINVAL, "plan %d is null", i);
        if (plans[i]->cfg.device != plans[0]->cfg.device) return fail(BNM_EINVAL, "plans of a group share one device");
        if (!plans[i]->cfg.do_fic) return fail(BNM_EINVAL, "group runs use device FIC: plan %d has do_fic = 0", i);
        for (int j = 0; j < i; j++)
            if (plans[j] == plans[i]) return fail(BNM_EINVAL, "plan %d appears twice", i);
        g->plans.push_back(plans[i]);
    }
    BNM_CUDA_TRY(cudaSetDevice(plans[0]->cfg.device));
    BNM_CUDA_TRY(cudaStreamCreateWithFlags(&g->origin, cudaStreamNonBlocking));
    BNM_CUDA_TRY(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
    BNM_CUDA_TRY(cudaEventCreate(&g->t0));
    BNM_CUDA_TRY(cudaEventCreate(&g->t1));
    g->join.assign(n_plans, nullptr);
    for (auto& e : g->join) BNM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (bnm_plan* p : g->plans) {
        int rc = ensure_pinned(p);
        if (rc) return rc;
    }
    return BNM_OK;
}

extern "C" int bnm_group_create(bnm_plan* const* plans, int32_t n_plans, bnm_group** out) {
    if (!plans || !out || n_plans < 1) return fail(BNM_EINVAL, "null argument or empty group");
    *out = nullptr;
    bnm_group* g = new bnm_group();
    int rc = group_create(plans, n_plans, g);
    if (rc) {
        bnm_group_destroy(g);
        return rc;
    }
    *out = g;
    return BNM_OK;
}

// The subjects' kernels share the SMs; whichever is enqueued first gets
// them first.  Starting the largest integrations first and letting the small
// ones fill the SMs they leave measured 12 % shorter generations on eight
// subjects of N = 68..400 than the reverse order.
static void set_order(bnm_group* g) {
    const size_t np = g->plans.size();
    std::vector<double> work(np);
    for (size_t i = 0; i < np; i++) {
        const bnm_plan* p = g->plans[i];
        work[i] = (double)p->cfg.nodes * p->cfg.nodes * g->n[i] * ((double)p->cfg.time_steps + 1.0);
    }
    g->order.resize(np);
    for (size_t i = 0; i < np; i++) g->order[i] = (int)i;
    std::stable_sort(g->order.begin(), g->order.end(), [&](int a, int b) { return work[a] > work[b]; });
}

static int capture(bnm_group* g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    g->exec = nullptr;
    g->graph = nullptr;
    BNM_CUDA_TRY(cudaStreamBeginCapture(g->origin, cudaStreamCaptureModeRelaxed));
    int rc = BNM_OK;
    cudaError_t e = cudaEventRecord(g->fork, g->origin);
    for (size_t k = 0; k < g->plans.size() && e == cudaSuccess && !rc; k++) {
        const int i = g->order[k];
        bnm_plan* p = g->plans[i];
        e = cudaStreamWaitEvent(p->st, g->fork, 0);
        if (e != cudaSuccess) break;
        p->capturing = true;
        rc = enqueue_run(p, g->n[i]);
        p->capturing = false;
        if (!rc) e = cudaEventRecord(g->join[i], p->st);
        if (!rc && e == cudaSuccess) e = cudaStreamWaitEvent(g->origin, g->join[i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e_end = cudaStreamEndCapture(g->origin, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    BNM_CUDA_TRY(e);
    BNM_CUDA_TRY(e_end);
    g->graph = graph;
    BNM_CUDA_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
    return BNM_OK;
}

extern "C" int bnm_group_run(bnm_group* g, const int32_t* n, const double* const* G, const double* const* w_ee,
                             const double* const* w_ei, bnm_batch_out* outs) {
    if (!g || !n || !G || !w_ee || !w_ei || !outs) return fail(BNM_EINVAL, "null argument");
    const size_t np = g->plans.size();
    BNM_CUDA_TRY(cudaSetDevice(g->plans[0]->cfg.device));
    std::vector<int> sizes(np);
    for (size_t i = 0; i < np; i++) {
        bnm_plan* p = g->plans[i];
        const int N = p->cfg.nodes;
        if (n[i] < 1 || n[i] > p->cfg.max_sims) return fail(BNM_EINVAL, "plan %zu: n=%d outside [1, max_sims]", i, n[i]);
        if (!G[i] || !w_ee[i] || !w_ei[i]) return fail(BNM_EINVAL, "plan %zu: null parameters", i);
        const bool rf = p->cfg.precision == BNM_PREC_F32_REF;
        for (int k = 0; k < n[i]; k++) {
            if (!std::isfinite(G[i][k])) return fail(BNM_EINVAL, "plan %zu: G[%d] is not finite", i, k);
            p->io_G[k] = rf ? (double)(float)G[i][k] : G[i][k];
        }
        for (size_t k = 0; k < (size_t)n[i] * N; k++) {
            if (!std::isfinite(w_ee[i][k]) || !std::isfinite(w_ei[i][k]))
                return fail(BNM_EINVAL, "plan %zu: wEE/wEI not finite at %zu", i, k);
            p->io_wEE[k] = rf ? (double)(float)w_ee[i][k] : w_ee[i][k];
            p->io_wEI[k] = rf ? (double)(float)w_ei[i][k] : w_ei[i][k];
        }
        sizes[i] = n[i];
        // the captured graph copies io_order at launch, so it is set for every run
        if (p->place) place_particles(p, n[i], p->io_G, p->io_wEE, p->io_wEI);
    }
    int rc;
    if (!g->exec || sizes != g->n) {
        // first call for these batch sizes: run eagerly (this tunes every
        // plan's integrator, which a capture cannot do), then capture the graph
        g->n = sizes;
        set_order(g);
        for (size_t i = 0; i < np; i++) {
            bnm_plan* p = g->plans[i];
            if (p->cfg.precision == BNM_PREC_F32) {
                BNM_CUDA_TRY(cudaMemcpy(p->d_G, p->io_G, sizes[i] * 8, cudaMemcpyHostToDevice));
                BNM_CUDA_TRY(cudaMemcpy(p->d_wEE, p->io_wEE, (size_t)sizes[i] * p->cfg.nodes * 8, cudaMemcpyHostToDevice));
                BNM_CUDA_TRY(cudaMemcpy(p->d_wEI, p->io_wEI, (size_t)sizes[i] * p->cfg.nodes * 8, cudaMemcpyHostToDevice));
                if ((rc = launch_fic(p, sizes[i]))) return rc;
                if ((rc = tune_integrator(p, sim_args(p, sizes[i]), np > 1))) return rc;
            }
            if ((rc = tune_window(p, sizes[i]))) return rc;
        }
        BNM_CUDA_TRY(cudaEventRecord(g->t0, g->origin));
        BNM_CUDA_TRY(cudaEventRecord(g->fork, g->origin));
        for (size_t k = 0; k < np; k++) {
            const int i = g->order[k];
            bnm_plan* p = g->plans[i];
            BNM_CUDA_TRY(cudaStreamWaitEvent(p->st, g->fork, 0));
            if ((rc = enqueue_run(p, sizes[i]))) return rc;
            BNM_CUDA_TRY(cudaEventRecord(g->join[i], p->st));
            BNM_CUDA_TRY(cudaStreamWaitEvent(g->origin, g->join[i], 0));
        }
        BNM_CUDA_TRY(cudaEventRecord(g->t1, g->origin));
        BNM_CUDA_TRY(cudaStreamSynchronize(g->origin));
        g->graph_launched = 0;
        if ((rc = capture(g))) return rc;
    } else {
        BNM_CUDA_TRY(cudaEventRecord(g->t0, g->origin));
        BNM_CUDA_TRY(cudaGraphLaunch(g->exec, g->origin));
        BNM_CUDA_TRY(cudaEventRecord(g->t1, g->origin));
        BNM_CUDA_TRY(cudaStreamSynchronize(g->origin));
        g->graph_launched = 1;
    }
    float ms;
    BNM_CUDA_TRY(cudaEventElapsedTime(&ms, g->t0, g->t1));
    g->last_ms = ms;
    for (size_t i = 0; i < np; i++) {
        bnm_plan* p = g->plans[i];
        const int k = sizes[i], N = p->cfg.nodes;
        if ((rc = read_timings(p))) return rc;
        const int status = *p->io_status;
        if (status & kStatusTimeout) return fail(BNM_ETIMEOUT, "plan %zu: a device wait gave up (status %d)", i, status);
        if (status) return fail(BNM_ECUDA, "plan %zu: device status %d", i, status);
        bnm_batch_out& o = outs[i];
        auto put = [](auto* dst, const auto* src, size_t cnt) {
            if (dst) std::copy(src, src + cnt, dst);
        };
        put(o.cost, p->io_cost, k);
        put(o.fic_penalty, p->io_pen, k);
        put(o.fc_corr, p->io_fcc, k);
        put(o.fc_diff, p->io_fcdiff, k);
        put(o.fcd_ks, p->io_ks, k);
        put(o.w_ie, p->io_wie, (size_t)k * N);
        put(o.fic_failed, p->io_failed, k);
        put(o.fic_ntrials, p->io_trials, k);
        put(o.fic_unstable, p->io_unstable, k);
        if (p->place) record_particles(p, k, p->io_G, p->io_wEE, p->io_wEI, p->io_trials);
    }
    return BNM_OK;
}

extern "C" int bnm_group_last(bnm_group* g, double* ms, int32_t* graph_launched) {
    if (!g || !ms) return fail(BNM_EINVAL, "null argument");
    *ms = g->last_ms;
    if (graph_launched) *graph_launched = g->graph_launched;
    return BNM_OK;
}

extern "C" int bnm_last_gram(bnm_plan* p, double* ms2, int32_t* launches) {
    if (!p || !ms2) return fail(BNM_EINVAL, "null argument");
    ms2[0] = p->gram_ms[0];
    ms2[1] = p->gram_ms[1];
    if (launches) *launches = p->launches;
    return BNM_OK;
}

extern "C" int bnm_plan_window_tile(bnm_plan* p, int32_t* pairs_per_thread, int32_t* n_tried) {
    if (!p || !pairs_per_thread) return fail(BNM_EINVAL, "null argument");
    *pairs_per_thread = p->win_ppt ? p->win_ppt : 4;
    if (n_tried) *n_tried = p->win_tried;
    return BNM_OK;
}

extern "C" int bnm_plan_graph(bnm_plan* p, int32_t* graph_launched) {
    if (!p || !graph_launched) return fail(BNM_EINVAL, "null argument");
    *graph_launched = p->last_graph;
    return BNM_OK;
}

extern "C" int bnm_plan_placement(bnm_plan* p, int32_t* enabled, int32_t* placed_last) {
    if (!p || !enabled || !placed_last) return fail(BNM_EINVAL, "null argument");
    *enabled = p->place;
    *placed_last = p->place && p->last_placed;
    return BNM_OK;
}

extern "C" int bnm_last_timings(bnm_plan* p, double* ms6) {
    if (!p || !ms6) return fail(BNM_EINVAL, "null argument");
    for (int i = 0; i < 6; i++) ms6[i] = p->timings[i];
    return BNM_OK;
}

extern "C" int bnm_plan_noise(bnm_plan* p, int64_t offset, int64_t n, float* out) {
    if (!p || !out || offset < 0 || n < 0 || offset + n > p->sz.noise_len) return fail(BNM_EINVAL, "bad noise range");
    BNM_CUDA_TRY(cudaSetDevice(p->cfg.device));
    const int N = p->cfg.nodes;
    if (p->d_noise && p->noise_ld == N) {
        BNM_CUDA_TRY(cudaMemcpy(out, p->d_noise + offset, (size_t)n * 4, cudaMemcpyDeviceToHost));
        return BNM_OK;
    }
    // a padded table, or noise drawn in place by the integrator: materialise
    // the values in the unpadded order
    std::vector<float> all;
    const float* src = p->d_noise;
    float* tmp = nullptr;
    if (!src) {
        BNM_CUDA_TRY(cudaMalloc(&tmp, (size_t)p->sz.noise_len * 4));
        cudaError_t e = bnm_launch_philox(tmp, (uint64_t)p->sz.noise_len, N, N, p->cfg.noise_seed, p->num_sms, 0);
        if (e == cudaSuccess) e = cudaMemcpy(out, tmp + offset, (size_t)n * 4, cudaMemcpyDeviceToHost);
        cudaFree(tmp);
        BNM_CUDA_TRY(e);
        return BNM_OK;
    }
    const size_t rows = (size_t)(p->cfg.time_steps + 1) * 10;
    all.resize((size_t)p->sz.noise_len);
    BNM_CUDA_TRY(cudaMemcpy2D(all.data(), (size_t)N * 8, src, (size_t)p->noise_ld * 8, (size_t)N * 8, rows,
                              cudaMemcpyDeviceToHost));
    std::copy(all.begin() + offset, all.begin() + offset + n, out);
    return BNM_OK;
}

extern "C" int bnm_run_simulations(double* corr, double* fic_penalties, const double* G_list, const double* w_EE_list,
                                   const double* w_EI_list, const double* w_IE_list, double* w_IE_fic,
                                   const double* SC, int32_t nodes, int32_t calculate_fic_penalty, int32_t time_steps,
                                   int32_t BOLD_TR, int32_t max_fic_trials, int32_t sim_only,
                                   const double* emp_FC_tril, int32_t n_emp_fc, const double* emp_FCD_tril,
                                   int32_t n_emp_fcd, int32_t window_size, int32_t window_step, int32_t N_SIMS,
                                   const float* noise, int32_t rand_seed, int32_t do_fic, int32_t adjust_fic,
                                   int32_t* FIC_failed, int32_t* fic_n_trials, double* BOLD_ex, double* ext_means) {
    bnm_config cfg;
    bnm_config_default(&cfg);
    bnm_config_from_env(&cfg);
    cfg.nodes = nodes;
    cfg.max_sims = N_SIMS;
    cfg.time_steps = time_steps;
    cfg.bold_tr = BOLD_TR;
    cfg.window_size = window_size;
    cfg.window_step = window_step;
    cfg.max_fic_trials = max_fic_trials;
    cfg.calculate_fic_penalty = calculate_fic_penalty;
    cfg.do_fic = do_fic;
    cfg.numerical_fic = adjust_fic;
    cfg.noise_mode = noise ? BNM_NOISE_HOST : BNM_NOISE_PHILOX;
    cfg.noise_seed = (uint64_t)rand_seed;
    bnm_sizes sz;
    int rc = bnm_config_sizes(&cfg, &sz);
    if (rc) return rc;
    bnm_plan* p = nullptr;
    rc = bnm_plan_create(&cfg, SC, emp_FC_tril, n_emp_fc, emp_FCD_tril, n_emp_fcd, noise, noise ? sz.noise_len : 0, &p);
    if (rc) return rc;
    std::vector<double> cost(N_SIMS), wie_out((size_t)N_SIMS * nodes);
    bnm_batch_out o;
    std::memset(&o, 0, sizeof o);
    o.cost = cost.data();
    o.fic_penalty = fic_penalties;
    o.w_ie = wie_out.data();
    o.fic_failed = FIC_failed;
    o.fic_ntrials = fic_n_trials;
    o.bold = BOLD_ex;
    o.ext_means = ext_means;
    const double* wie_in = do_fic ? w_IE_fic : w_IE_list;
    rc = bnm_run(p, N_SIMS, G_list, w_EE_list, w_EI_list, wie_in, &o);
    bnm_plan_destroy(p);
    if (rc) return rc;
    for (int i = 0; i < N_SIMS; i++) corr[i] = sim_only ? cfg.max_cost : cost[i];
    if (do_fic && w_IE_fic) std::copy(wie_out.begin(), wie_out.end(), w_IE_fic);
    return BNM_OK;
}
