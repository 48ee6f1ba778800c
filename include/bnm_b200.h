/*
 * bnm_b200 -- C ABI of the B200 simulate-and-fit library.
 *
 * Drop-in boundary for the reference's batch entry point and its driver
 * (amnsbr/bnm_cuda):
 *
 *   run_simulations(...)        bnm.cu:594-617   (GPU build; called per CMA-ES
 *                               generation at run_CMAES.cpp:758-780 and for the
 *                               best-particle rerun at run_CMAES.cpp:875-897)
 *                               bnm.cpp:431-439  (CPU build, same meaning)
 *   analytical_fic(...)         fic.cpp:130-207  (per particle, run_CMAES.cpp:144-174)
 *   noise precompute            run_CMAES.cpp:640-657
 *   CMAES_Points()              cmaes.cpp:128-557 (driven at run_CMAES.cpp:714-818)
 *   BNM_* runtime configuration constants.h:93-116
 *
 * All signatures use plain C types.  Every entry point returns a status
 * (BNM_OK or a BNM_E* code) instead of exiting the process; bnm_last_error()
 * gives the message.  Host arrays are flat, particle-major ([n][nodes]).
 */
#ifndef BNM_B200_H
#define BNM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BNM_OK 0
#define BNM_EINVAL 1   /* bad argument or size (the reference exits in these cases) */
#define BNM_ENOMEM 2   /* device allocation failed */
#define BNM_ECUDA 3    /* CUDA runtime error */
#define BNM_ETIMEOUT 4 /* a bounded device wait gave up */

/* Arithmetic of the integrator.  FP32 is the product path (FP32 integration,
 * FP64 FIC solve and FP64 centring of BOLD / window series).  F64 and F32_REF
 * are the reference-order kernels (no FMA contraction): F64 follows the
 * reference's default double build, F32_REF its USE_FLOATS build. */
enum { BNM_PREC_F32 = 0, BNM_PREC_F64 = 1, BNM_PREC_F32_REF = 2 };

/* Noise source.  PHILOX: counter-based Philox4x32-10 + Box-Muller keyed by
 * noise_seed, shared by all particles and FIC trials (the reference's
 * common-random-numbers semantics).  The FP32 cluster kernels (N > 128) draw
 * the values where they use them (no table in HBM); the register kernel
 * (N <= 128) and the reference-order kernels read a table of the same values
 * (BNM_B200_NOISE_SOURCE=inline|table overrides the FP32 default; drawing in
 * place lengthens the register kernel's substep).  HOST: the caller's
 * precomputed table (the
 * reference's mt19937 + normal_distribution<float> stream,
 * run_CMAES.cpp:640-657). */
enum { BNM_NOISE_PHILOX = 0, BNM_NOISE_HOST = 1 };

/* Arithmetic of the FC and FCD Grams (both over rows centred and scaled in
 * FP64).  F32: FCD on the FP32 SIMT pipe, FC from FP64 co-moments.  BF16 and
 * BF16_SPLIT: FC and FCD as tcgen05 tensor-core Grams with FP32 accumulation,
 * operands rounded once to BF16, or split into hi + lo BF16 parts with the
 * hi.hi + hi.lo + lo.hi products accumulated (error near FP32's). */
enum { BNM_GRAM_AUTO = -1, BNM_GRAM_F32 = 0, BNM_GRAM_BF16 = 1, BNM_GRAM_BF16_SPLIT = 2 };

/* Run configuration: the reference's CLI arguments and BNM_* settings. */
typedef struct bnm_config {
    int32_t nodes;             /* argv[6] */
    int32_t max_sims;          /* particles per call (lambda, argv[17]) */
    int32_t time_steps;        /* argv[12], ms; the loop runs 0..time_steps */
    int32_t bold_tr;           /* argv[13], ms */
    int32_t window_step;       /* argv[14] */
    int32_t window_size;       /* argv[15] */
    int32_t bold_remove_s;     /* BNM_BOLD_REMOVE (30) */
    int32_t exc_interhem;      /* BNM_EXC_INTERHEM (1) */
    int32_t do_fic;            /* wIE from FIC (argv[10] == 0) */
    int32_t numerical_fic;     /* BNM_NUMERICAL_FIC (1) */
    int32_t max_fic_trials;    /* BNM_MAX_FIC_TRIALS_CMAES (10) */
    int32_t i_sampling_start;  /* BNM_I_SAMPLING_START (1000) */
    int32_t i_sampling_end;    /* BNM_I_SAMPLING_END (10000) */
    double init_delta;         /* BNM_INIT_DELTA (0.02, rounded to float as the reference does) */
    int32_t use_fc_diff;       /* BNM_USE_FC_DIFF (1) */
    int32_t fic_reject_failed; /* BNM_CMAES_FIC_REJECT_FAILED (0) */
    double fic_penalty_scale;  /* BNM_CMAES_FIC_PENALTY_SCALE (2) */
    double max_cost;           /* BNM_MAX_COST (2) */
    int32_t calculate_fic_penalty; /* on when do_fic (run_CMAES.cpp:389) */
    int32_t no_fcd;            /* fcd path "no_fcd" (run_CMAES.cpp:331) */
    int32_t precision;         /* BNM_PREC_* */
    int32_t noise_mode;        /* BNM_NOISE_* */
    uint64_t noise_seed;       /* argv[16] */
    int32_t device;
    int32_t gram;              /* BNM_GRAM_* (default AUTO: BF16_SPLIT for BNM_PREC_F32, F32 for the
                                  reference-order precisions, whose results are compared with the
                                  reference's own arithmetic; no counterpart in the reference, which
                                  runs FP32/FP64 SIMT) */
} bnm_config;

/* Reference defaults (constants.h:93-116). */
void bnm_config_default(bnm_config *cfg);
/* Overlay the BNM_* environment variables the way the reference reads them
 * (doubles pass through float, helpers.cpp:4-11). */
void bnm_config_from_env(bnm_config *cfg);

const char *bnm_last_error(void);
int bnm_device_count(void);

/* Derived sizes of a configuration (no device work). */
typedef struct bnm_sizes {
    int32_t frames;        /* BOLD frames, time_steps / bold_tr + 1 (run_CMAES.cpp:476-477) */
    int32_t n_vols_remove; /* bold_remove_s * 1000 / bold_tr (run_CMAES.cpp:483) */
    int32_t corr_len;      /* frames - n_vols_remove */
    int32_t n_pairs;       /* FC lower-triangle length (run_CMAES.cpp:494-500) */
    int32_t n_windows;     /* FCD windows (run_CMAES.cpp:531-556) */
    int32_t window_len;    /* frames per window */
    int32_t n_fcd;         /* n_windows * (n_windows - 1) / 2 */
    int64_t noise_len;     /* nodes * (time_steps + 1) * 10 * 2 floats */
} bnm_sizes;
int bnm_config_sizes(const bnm_config *cfg, bnm_sizes *out);

/* ------------------------------------------------------------------ plans
 * A plan owns every device buffer of a configuration (SC, targets, noise
 * table, per-particle work space for max_sims particles) so that one call per
 * CMA-ES generation allocates nothing.  One plan per thread at a time. */
typedef struct bnm_plan bnm_plan;

/* sc: nodes*nodes row-major.  emp_fc: n_pairs values in the reference's pair
 * order.  emp_fcd: any length > 0 (unless no_fcd).  host_noise: required for
 * BNM_NOISE_HOST, noise_len floats. */
int bnm_plan_create(const bnm_config *cfg, const double *sc, const double *emp_fc, int32_t n_emp_fc,
                    const double *emp_fcd, int32_t n_emp_fcd, const float *host_noise, int64_t n_host_noise,
                    bnm_plan **out);
void bnm_plan_destroy(bnm_plan *plan);

/* Per-particle outputs; every pointer except cost may be NULL. */
typedef struct bnm_batch_out {
    double *cost;        /* [n] 1 - r(FC) + KS(FCD) (+ |dmean FC|); max_cost on NaN.  = corr[] of run_simulations */
    double *fic_penalty; /* [n] (0 when not calculated) */
    double *fc_corr;     /* [n] */
    double *fc_diff;     /* [n] */
    double *fcd_ks;      /* [n] */
    double *w_ie;        /* [n][nodes] wIE after FIC (the reference's w_IE_fic out) */
    int32_t *fic_failed; /* [n] */
    int32_t *fic_ntrials;/* [n] */
    int32_t *fic_unstable; /* [n] analytic FIC was unstable (wIE set to 1) */
    double *ext_means;   /* [n][6][nodes] S_E, I_E, r_E, S_I, I_I, r_I means over kept frames */
    double *bold;        /* [n][frames][nodes] */
    double *fc;          /* [n][n_pairs] */
    double *fcd;         /* [n][n_fcd] */
    double *fcd_left;    /* [n][n_fcd] FCD over the first (nodes/2)(nodes/2-1)/2 pairs (left hemisphere) and */
    double *fcd_right;   /* [n][n_fcd] over the last as many (right): the reference's save_hemis outputs,
                            bnm.cu:436-551; computed only when set, not part of the cost */
} bnm_batch_out;

/* One batch (a CMA-ES generation): integrate, BOLD, FC, window FC, FCD, KS,
 * goodness of fit and FIC penalty for n <= max_sims particles.
 * G [n]; w_ee, w_ei [n][nodes].  w_ie [n][nodes]: the fixed wIE when
 * do_fic == 0; with do_fic it is the analytic-FIC starting point (as the
 * reference GPU driver's w_IE_fic), or NULL to compute it on the device.
 * The reference launches seven kernels with a device synchronisation after
 * each (bnm.cu:624-724).  Here the first call for a batch size runs eagerly
 * and tunes the integrator; with the FP32 path and device FIC (w_ie NULL, no
 * hemisphere FCDs) every later call for that batch size is one CUDA graph
 * launch of the whole generation (parameter upload from pinned staging,
 * analytic FIC, integrator, window FC, Grams, KS, fit, result download),
 * captured on its first use; BNM_B200_GRAPH=0 keeps every call eager. */
int bnm_run(bnm_plan *plan, int32_t n, const double *G, const double *w_ee, const double *w_ei, const double *w_ie,
            bnm_batch_out *out);
/* Whether the plan's last bnm_run was a graph launch (1) or eager (0). */
int bnm_plan_graph(bnm_plan *plan, int32_t *graph_launched);

/* Particle placement (FP32, numerical FIC; no counterpart in the reference,
 * whose blocks take particles by index): the plan predicts each particle's FIC
 * restarts from the nearest of the last 4096 particles it simulated.  The
 * register integrator (N <= 128, noise table) gives the heaviest particles to
 * CTAs alone on an SM and the lightest to the second CTA of an SM; the
 * two-particle column-split clusters pair particles of similar predicted work.
 * Results do not depend on it.  enabled: the plan places particles
 * (BNM_B200_PLACE=0 at plan creation turns it off); placed_last: the last
 * run's order came from the history (16 particles or more simulated before). */
int bnm_plan_placement(bnm_plan *plan, int32_t *enabled, int32_t *placed_last);

/* Analytic FIC alone (fic.cpp:130-207) for n particles on the device. */
int bnm_analytic_fic(bnm_plan *plan, int32_t n, const double *G, const double *w_ee, const double *w_ei,
                     double *w_ie_out, int32_t *unstable_out);

/* Time of the last bnm_run on the device, per stage, in ms:
 * [0] analytic FIC, [1] integration, [2] FC + window FC, [3] FCD + KS histogram, [4] GOF, [5] total. */
/* Groups: several plans (e.g. subjects of different node counts, each with
 * its own SC, targets and autotuned integrator) run one generation as one
 * CUDA graph launch: every plan's stages on its own stream, forked from and
 * joined to one origin stream, parameters and results staged through pinned
 * host buffers, one host synchronisation.  No counterpart in the reference,
 * which runs one subject per process.  The first bnm_group_run for a set of
 * batch sizes runs eagerly (and tunes each plan's integrator) and captures
 * the graph; later calls with the same sizes launch it.  Plans must use
 * device FIC (do_fic = 1); outputs per plan: cost, fic_penalty, fc_corr,
 * fc_diff, fcd_ks, w_ie, fic_failed, fic_ntrials, fic_unstable (bold, fc,
 * fcd and ext_means are not filled). */
typedef struct bnm_group bnm_group;
int bnm_group_create(bnm_plan *const *plans, int32_t n_plans, bnm_group **out);
void bnm_group_destroy(bnm_group *group);
int bnm_group_run(bnm_group *group, const int32_t *n, const double *const *G, const double *const *w_ee,
                  const double *const *w_ei, bnm_batch_out *outs);
/* Device time of the last group run (ms, events on the origin stream around
 * the whole generation) and whether it was a graph launch (1) or the eager
 * first run (0). */
int bnm_group_last(bnm_group *group, double *ms, int32_t *graph_launched);

/* Device time of the tensor-core Gram kernels alone in the last bnm_run /
 * bnm_check_fit_bold (ms2[0]: FC Gram, ms2[1]: FCD Gram summed over staged
 * chunks; 0 with BNM_GRAM_F32) and the number of library kernels that call
 * launched (*launches).  No counterpart in the reference. */
int bnm_last_gram(bnm_plan *plan, double *ms2, int32_t *launches);

/* Goodness of fit of given BOLD (check_fit_bold, check_fit.cpp:138-217,
 * batched): bold = n series of corr_len kept frames (those after
 * n_vols_remove) x nodes, particle-major.  Computes FC, window FC, FCD, the
 * KS distance and cost on the device with the plan's configuration, Gram
 * arithmetic and targets, and fills cost, fc_corr, fc_diff, fcd_ks (and fc,
 * fcd when set) of *out; no FIC penalty is added (fic_penalty = 0). */
int bnm_check_fit_bold(bnm_plan *plan, int32_t n, const double *bold, bnm_batch_out *out);

int bnm_last_timings(bnm_plan *plan, double *ms6);

/* FP32 integrator configuration the autotuner picked for the plan's last
 * batch size (no counterpart in the reference, which has one kernel shape).
 * out5: kind (0 register-SC kernel for N <= 128; 1 row-split
 * thread-block-cluster kernel for even 128 < N <= 512; 3 column-split
 * cluster kernel for N > 128 up to about 900 nodes, an odd N with one
 * padding node; 4 the column-split kernel with two particles per cluster; 2 reference-order
 * kernel), then kind 0: particles per CTA; kind 1: -, CTAs per particle,
 * nodes per warp, SC column chunks of 32 in registers; kinds 3 and 4: column
 * pairs per warp, CTAs per cluster, rows per lane, column pairs in
 * registers.  *n_tried: candidate shapes timed.  The tuner runs on the first
 * run of each batch size (by time for bnm_run, by SM time for the plans of a
 * group) and the plan keeps that shape; BNM_B200_SHAPE="k,s,c,r,kr" forces a
 * shape and BNM_B200_TUNE=0 skips the timing. */
int bnm_plan_integrator(bnm_plan *plan, int32_t *out5, int32_t *n_tried);

/* Window-FC tile the tuner picked for the plan's last batch size (no
 * counterpart in the reference, whose fc kernel covers maxThreadsPerBlock
 * pairs per block, bnm.cu:649-708): *pairs_per_thread in {1, 2, 4, 8}, a CTA
 * of 256 threads covering 256 x that many pairs; *n_tried: tiles timed.
 * Tuned with the integrator on the first run of each batch size
 * (BNM_B200_TUNE=0: 4, untimed). */
int bnm_plan_window_tile(bnm_plan *plan, int32_t *pairs_per_thread, int32_t *n_tried);

/* Measured FP32 FMA throughput of a device (packed fma.rn.f32x2 chains), in
 * TFLOP/s: the roofline denominator of the FP32-pipe-bound integrator.  No
 * counterpart in the reference. */
int bnm_measure_fp32_peak(int32_t device, double *tflops);

/* Test support, no counterpart in the reference: for each of the n inputs x,
 * out4 receives the FP32 integrators' Balloon-Windkessel e^x - 1 and
 * ln(1 + x) next to CUDA's expm1f and log1pf ([4 i .. 4 i + 3] = expm1_bw,
 * expm1f, log1p_bw, log1pf). */
int bnm_bw_math_probe(int32_t device, const float *x, int32_t n, float *out4);

/* Test support, no counterpart in the reference: failure detection of the
 * library's bounded device waits without a GPU fault.  One CTA waits, with the
 * integrators' own wait routine, on an mbarrier that nothing arrives on (no
 * copy or MMA in flight) for limit_ns nanoseconds of wall time
 * (0 <= limit_ns <= 1e9, the integrators' limit).  The wait gives up, the
 * kernel records the timeout status and returns normally: the call returns
 * BNM_ETIMEOUT with *status_out = the status word and *elapsed_ms = the
 * measured wait, and the device stays usable. */
int bnm_wait_probe(int32_t device, int64_t limit_ns, int32_t *status_out, double *elapsed_ms);

/* Test support, no counterpart in the reference: the Philox4x32-10 block
 * function (Salmon et al., SC'11) of the noise source, run on the device for
 * n inputs in6[i] = {counter[0..3], key[0..1]}; out4[i] = the four output
 * words.  For a known-answer test against the published vectors. */
int bnm_philox_probe(int32_t device, const uint32_t *in6, int32_t n, uint32_t *out4);

/* The plan's noise in the table's order ([ms][substep][node][E, I]), n floats
 * from offset: the table when the plan holds one, else the Philox values the
 * register integrator draws in place (materialised for the copy). */
int bnm_plan_noise(bnm_plan *plan, int64_t offset, int64_t n, float *out);

/* ------------------------------------------------ allocation-free entry
 * No counterpart in the reference.  Goodness of fit (FC, sliding-window FC,
 * FCD, KS, cost) of n BOLD series that are already on the device, for callers
 * that cannot allocate device memory: hosts that own the allocator (an
 * embedding framework's caching allocator or a fixed memory budget) and
 * real-time or streaming loops that must not call cudaMalloc / cudaFree
 * (cudaFree synchronises the device).  Nothing is allocated: every
 * intermediate lives in one static device array of BNM_NOALLOC_SCRATCH_BYTES
 * per device, resident on every GPU that loads the library until exit.
 *   d_bold          device [n][frames][nodes] float
 *   emp_fc          host [n_pairs], the reference's pair order
 *   emp_fcd_sorted  host [n_emp_fcd], ascending (checked)
 *   d_out           device [5][n] double: cost, fc_corr, fc_diff, fcd_ks, 0
 *   stream          a cudaStream_t (NULL = the default stream); the call is
 *                   asynchronous on it.
 * Calls whose intermediates exceed the scratch array fail with BNM_EINVAL.
 * Calls with fewer than 2 node pairs are rejected with BNM_EINVAL as well.
 * All calls share the array: the call zeroes what it accumulates, but calls
 * that overlap on the GPU race.  The first call on a device looks up the
 * array's address.  emp_fc and emp_fcd_sorted are copied to the device on
 * the stream: from pageable memory the runtime has staged them when the call
 * returns; from page-locked memory the copy runs asynchronously, so keep them
 * unchanged until the stream has passed the call. */
#define BNM_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int bnm_gof_noalloc(const float *d_bold, int32_t n, int32_t frames, int32_t nodes, int32_t n_vols_remove,
                    int32_t window_size, int32_t window_step, int32_t exc_interhem, int32_t use_fc_diff,
                    double max_cost, const double *emp_fc, int32_t n_emp_fc, const double *emp_fcd_sorted,
                    int32_t n_emp_fcd, double *d_out, void *stream);

/* ------------------------------------------------------ one-shot mirror
 * Same argument meaning as the reference's run_simulations (bnm.cu:594-617),
 * flattened: builds a plan, runs one batch, releases it.  corr receives the
 * goodness-of-fit cost, fic_penalties the FIC penalty, w_IE_fic (in/out, may
 * be NULL) the FIC weights, FIC_failed / fic_n_trials the numerical FIC
 * outcome, BOLD_ex the BOLD frames ([N_SIMS][output_ts][nodes], may be NULL),
 * ext_means the extended outputs (may be NULL).  noise may be NULL (Philox,
 * seeded by rand_seed). */
int bnm_run_simulations(double *corr, double *fic_penalties, const double *G_list, const double *w_EE_list,
                        const double *w_EI_list, const double *w_IE_list, double *w_IE_fic, const double *SC,
                        int32_t nodes, int32_t calculate_fic_penalty, int32_t time_steps, int32_t BOLD_TR,
                        int32_t max_fic_trials, int32_t sim_only, const double *emp_FC_tril, int32_t n_emp_fc,
                        const double *emp_FCD_tril, int32_t n_emp_fcd, int32_t window_size, int32_t window_step,
                        int32_t N_SIMS, const float *noise, int32_t rand_seed, int32_t do_fic, int32_t adjust_fic,
                        int32_t *FIC_failed, int32_t *fic_n_trials, double *BOLD_ex, double *ext_means);

/* Parameter expansion of particle values (calculate_params,
 * run_CMAES.cpp:61-143): G_out = G; for each local parameter k in the
 * reference's order (wee, wie, wei; run_CMAES.cpp:252) with bit k of het_mask
 * set, node j gets base_k * (1 + sum_m scales[k][m] * maps[m][j]), and all
 * nodes of that parameter are shifted up so that the smallest is 0.001 when
 * any fell below it; parameters without their bit get the base value on
 * every node.  maps [n_maps][nodes], scales [3][n_maps] (the map coefficients
 * "<param>scale_<m>"); both may be NULL when het_mask == 0.  Outputs [nodes]. */
int bnm_calculate_params(int32_t nodes, int32_t het_mask, int32_t n_maps, const double *maps, double G, double wee,
                         double wie, double wei, const double *scales, double *G_out, double *w_ee, double *w_ei,
                         double *w_ie);

/* ------------------------------------------------------------- CMA-ES
 * Host optimiser with the semantics of the reference's CMAES_Points
 * (cmaes.cpp:128-557): Hansen's CMA-ES (2006 "Variante 6" or 2016 "16"),
 * coordinates in [0,1], boundary penalty (Hansen et al. 2009), early stop on
 * a flat best-cost history.  Random streams as in the reference
 * (std::default_random_engine seeded SeedMW and 11+it). */
typedef struct bnm_cmaes bnm_cmaes;
typedef struct bnm_cmaes_params {
    int32_t lambda, dimension, seed_mw, it_max;
    int32_t variante;       /* BNM_CMAES_VARIANTE (6) */
    double sigma;           /* BNM_CMAES_SIGMA (0.5) */
    double alphacov;        /* BNM_CMAES_ALPHACOV (2) */
    double gamma_scale;     /* BNM_CMAES_GAMMA_SCALE (2) */
    double bound_soft_edge; /* BNM_CMAES_BOUND_SOFT_EDGE (0) */
    int32_t early_stop_gens;/* BNM_CMAES_EARLY_STOP_GENS (30) */
    double early_stop_tol;  /* BNM_CMAES_EARLY_STOP_TOL (1e-3) */
} bnm_cmaes_params;
void bnm_cmaes_params_default(bnm_cmaes_params *p);
void bnm_cmaes_params_from_env(bnm_cmaes_params *p);
/* Creates the optimiser and samples generation 0 (the first CMAES_Points call). */
int bnm_cmaes_create(const bnm_cmaes_params *p, bnm_cmaes **out);
void bnm_cmaes_destroy(bnm_cmaes *c);
/* Iteration counter (the reference's global `it`); >= it_max means stop. */
int32_t bnm_cmaes_iteration(const bnm_cmaes *c);
/* Current sample points: feasible [dim][lambda] (clipped to [0,1]), raw and preferred (may be NULL). */
int bnm_cmaes_samples(const bnm_cmaes *c, double *feasible, double *raw, double *preferred);
/* Report the costs of the current samples (gof cost + FIC penalty, lower is
 * better); computes the boundary penalty (written to penalized, may be NULL)
 * and samples the next generation.  Returns the new iteration counter. */
int32_t bnm_cmaes_tell(bnm_cmaes *c, const double *cost, double *penalized);
/* Replace the current samples (raw [dim][lambda]) before bnm_cmaes_tell, e.g.
 * with surrogate-pre-screened candidates drawn from N(mean, sigma^2 C).  No
 * counterpart in the reference. */
int bnm_cmaes_set_samples(bnm_cmaes *c, const double *raw);
/* Best feasible point [dim] and its value (-cost, the reference's CBVfeas[D]). */
int bnm_cmaes_best(const bnm_cmaes *c, double *x, double *value);
int bnm_cmaes_state(const bnm_cmaes *c, double *mean, double *sigma, double *C);
/* Checkpoint / resume (no counterpart in the reference, whose CMA-ES state is
 * process-global, cmaes.cpp:69-126): bnm_cmaes_save writes the optimiser's
 * whole state (parameters, counters, mean, paths, covariance and its
 * decomposition, current samples, best-so-far and early-stop history; exact
 * doubles) to path, through a temporary file renamed into place, so the file
 * is whole or absent.  bnm_cmaes_load creates an optimiser from such a file;
 * it samples and updates exactly as the one that was saved.  Returns 0, 1
 * (null argument), 2 (file error) or 3 (not a checkpoint of this format). */
int bnm_cmaes_save(const bnm_cmaes *c, const char *path);
int bnm_cmaes_load(const char *path, bnm_cmaes **out);
/* The parameters an optimiser was created (or saved) with. */
int bnm_cmaes_params_of(const bnm_cmaes *c, bnm_cmaes_params *out);

/* ------------------------------------------------------ MLP surrogate
 * No counterpart in the reference.  A ReLU MLP (in -> hidden x layers -> out)
 * trained on the device by the library's own kernels (BF16 tensor-core GEMMs
 * with FP32 accumulation, MSE loss, Adam), used to pre-screen oversampled
 * CMA-ES candidates.  Inputs / targets are float, row-major [n][dim], already
 * normalised by the caller.  Flat parameters: per layer W [out][in] then b. */
typedef struct bnm_mlp bnm_mlp;
int bnm_mlp_create(int32_t in_dim, int32_t hidden, int32_t layers, int32_t out_dim, int32_t max_batch, uint64_t seed,
                   int32_t device, bnm_mlp **out);
void bnm_mlp_destroy(bnm_mlp *mlp);
int64_t bnm_mlp_num_params(const bnm_mlp *mlp);
int bnm_mlp_get_params(bnm_mlp *mlp, float *flat);
/* Sets every parameter; the optimiser state (Adam moments, step count) restarts. */
int bnm_mlp_set_params(bnm_mlp *mlp, const float *flat);
/* epochs of shuffled mini-batches (full batches only); loss_per_epoch may be NULL */
int bnm_mlp_train(bnm_mlp *mlp, const float *X, const float *Y, int32_t n, int32_t epochs, int32_t batch, float lr,
                  uint64_t shuffle_seed, float *loss_per_epoch);
int bnm_mlp_predict(bnm_mlp *mlp, const float *X, int32_t n, float *Y);
/* one batch (n <= max_batch): MSE loss and the gradient of every parameter, no update */
int bnm_mlp_loss_and_grads(bnm_mlp *mlp, const float *X, const float *Y, int32_t n, float *loss, float *grads);

#ifdef __cplusplus
}
#endif
#endif
