/*
 * TEST INFRASTRUCTURE ONLY (oracle).  This project's CPU restatement of the
 * reference's simulate-and-fit path, used by tests/, by smoke() and by the
 * CPU-baseline leg of bench.py to check the device results.  The product never
 * links it.
 *
 * It follows the reference's CPU path (bnm.cpp, check_fit.cpp, fic.cpp):
 *   port_noise            run_CMAES.cpp:643-654 / bnm.cpp:38-43 noise stream
 *   port_analytic_fic     fic.cpp:130-207 (analytical_fic) + run_CMAES.cpp:144-174
 *   port_integrate_*      bnm.cpp:26-290 (rWW Euler-Maruyama, numerical FIC,
 *                         Balloon-Windkessel, BOLD frames) and the extended
 *                         outputs / FIC penalty of bnm.cpp:332-405
 *   port_fc_tril          check_fit.cpp:19-62
 *   port_fcd_tril         check_fit.cpp:64-136
 *   port_gof              check_fit.cpp:138-217 (+ FIC penalty, run_CMAES.cpp:788)
 *
 * The update expressions keep the reference's operand order and operand
 * types (including the double literals that promote float arithmetic in the
 * reference's USE_FLOATS build), so that, compiled with the reference's
 * flags (g++ -O3 -m64), the float and double instantiations reproduce the
 * reference build's results bit for bit.  Statistics primitives come from
 * compat/ (the GSL / libks stand-ins the reference build also uses).
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>
#include <algorithm>
#include <omp.h>
#include "gsl/gsl_compat.h"
#include "ks.h"

namespace {

/* Model constants of constants.h:24-90, instantiated per arithmetic type
 * exactly as the reference declares them (const u_real x = literal). */
template <typename R>
struct K {
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
/* FIC steady-state constants are double in both builds (constants.h:51-64). */
constexpr double tau_I_s = 0.01, gamma_I_s = 1.0;
constexpr double r_I_ss = 3.9218448633, I_I_ss = 0.2528951325, I_E_ss = 0.3773805650;
constexpr double S_I_ss = 0.0392184486, S_E_ss = 0.1647572075;

inline float rexp(float x) { return expf(x); }
inline double rexp(double x) { return exp(x); }
inline float rpow(float a, float b) { return powf(a, b); }
inline double rpow(double a, double b) { return pow(a, b); }
inline float rabs(float x) { return std::abs(x); }
inline double rabs(double x) { return std::abs(x); }

template <typename R>
struct FicParams {
    double I0_I, w_EI, S_E_ss, w_II, gamma_I_s, tau_I_s;
};

/* fic.cpp:58-61 */
template <typename R>
double phi_I(double II) {
    return ((K<R>::a_I * II) - K<R>::b_I) / (1 - exp(-1 * K<R>::d_I * ((K<R>::a_I * II) - K<R>::b_I)));
}
/* fic.cpp:70-74 */
template <typename R>
double inh_curr(double x, void *vp) {
    FicParams<R> *p = (FicParams<R> *)vp;
    return p->I0_I + p->w_EI * p->S_E_ss - p->w_II * p->gamma_I_s * p->tau_I_s * phi_I<R>(x) - x;
}
/* fic.cpp:26-55: Brent on [lo, hi], interval test (0, 0.001), <= 100 iterations. */
double brent_solve(gsl_function F, double lo, double hi) {
    gsl_root_fsolver *s = gsl_root_fsolver_alloc(gsl_root_fsolver_brent);
    gsl_root_fsolver_set(s, &F, lo, hi);
    int status, iter = 0;
    double root = 0;
    do {
        iter++;
        gsl_root_fsolver_iterate(s);
        root = gsl_root_fsolver_root(s);
        lo = gsl_root_fsolver_x_lower(s);
        hi = gsl_root_fsolver_x_upper(s);
        status = gsl_root_test_interval(lo, hi, 0, 0.001);
    } while (status == GSL_CONTINUE && iter < 100);
    gsl_root_fsolver_free(s);
    return status == GSL_SUCCESS ? root : -1;
}

/* fic.cpp:85-160.  SC, wEE and wEI are the double copies the reference builds
 * from u_real values.  Returns 1 when unstable (then wIE is untouched). */
template <typename R>
int analytic_fic(const double *SC, int N, double G, const double *wEE, const double *wEI, double *wIE) {
    const double I0 = (double)K<R>::I_0;
    const double I0_E = I0 * (double)K<R>::w_E, I0_I = I0 * (double)K<R>::w_I;
    const double GJ = G * K<R>::J_NMDA;
    std::vector<double> out(N), krow(N);
    for (int j = 0; j < N; j++) {
        FicParams<R> p = {I0_I, wEI[j], S_E_ss, (double)K<R>::w_II, gamma_I_s, tau_I_s};
        gsl_function F;
        F.function = &inh_curr<R>;
        F.params = &p;
        double II = brent_solve(F, 0.0, 2.0);
        if (II == -1) return 1;
        double rI = phi_I<R>(II);
        double SI = rI * tau_I_s * gamma_I_s;
        /* K_EE row j: SC * (G J_NMDA) + diag(wEE), dotted with S_E_ss */
        double dot = 0.0;
        for (int k = 0; k < N; k++) {
            double kee = SC[(size_t)j * N + k] * GJ;
            if (k == j) kee += wEE[j];
            dot += kee * S_E_ss;
        }
        double J = (-1 / SI) * (I_E_ss - (double)K<R>::I_ext - I0_E - dot);
        if (J < 0) return 1;
        out[j] = J;
    }
    for (int j = 0; j < N; j++) wIE[j] = out[j];
    return 0;
}

struct Noise {
    const float *arr;
    size_t idx;
    int seed;
    std::mt19937 gen;
    std::normal_distribution<float> dist;
    Noise(const float *a, int s) : arr(a), idx(0), seed(s), gen(s), dist(0, 1) {}
    float next() { return arr ? arr[idx++] : dist(gen); }
    void restart() {
        idx = 0;
        gen = std::mt19937(seed);
        dist = std::normal_distribution<float>(0, 1);
    }
};

struct FicConf {
    int sampling_start, sampling_end;
    double init_delta; /* the reference's float-rounded BNM_INIT_DELTA */
};

/* bnm.cpp:26-290 and the r_E mean / FIC penalty of bnm.cpp:338-405. */
template <typename R>
void integrate(const double *SCd, int N, double Gd, const double *wEEd, const double *wEId, const double *wIEd,
               int adjust_fic, int max_trials, int T, int TR, int n_vols_remove, Noise &noise, const FicConf &fc,
               double *bold_out, double *wIE_out, int *trials_out, int *failed_out, double *ext_out) {
    typedef K<R> C;
    const int output_ts = T / TR + 1;
    std::vector<R> SC((size_t)N * N), S_E(N, 0.001), S_I(N, 0.001), S_prev(N), wEE(N), wEI(N), wIE(N);
    std::vector<R> x(N, 0.0), f(N, 1.0), nu(N, 1.0), q(N, 1.0), rE(N, 0), rI(N, 0), IE(N, 0), II(N, 0);
    std::vector<R> mean_IE(N, 0), delta(N, (R)fc.init_delta);
    std::vector<R> bold((size_t)output_ts * N), ext(6 * (size_t)output_ts * N);
    const R G = (R)Gd;
    for (size_t i = 0; i < (size_t)N * N; i++) SC[i] = (R)SCd[i];
    for (int j = 0; j < N; j++) {
        wEE[j] = (R)wEEd[j];
        wEI[j] = (R)wEId[j];
        wIE[j] = (R)wIEd[j];
    }
    const unsigned int duration = fc.sampling_end - fc.sampling_start + 1;
    int trial = 0;
    bool failed = false, adjusting = adjust_fic != 0;
    int ts = 0, frame = 0;
    while (ts <= T) {
        for (int sub = 0; sub < 10; sub++) {
            for (int j = 0; j < N; j++) S_prev[j] = S_E[j];
            for (int j = 0; j < N; j++) {
                R coupling = 0;
                for (int k = 0; k < N; k++) coupling += SC[(size_t)j * N + k] * S_prev[k];
                IE[j] = C::w_E__I_0 + wEE[j] * S_E[j] + coupling * G * C::J_NMDA - wIE[j] * S_I[j];
                II[j] = C::w_I__I_0 + wEI[j] * S_E[j] - S_I[j];
                R eE = rexp(-C::d_E * (C::a_E * IE[j] - C::b_E));
                R eI = rexp(-C::d_I * (C::a_I * II[j] - C::b_I));
                rE[j] = (C::a_E * IE[j] - C::b_E) / (1 - eE);
                rI[j] = (C::a_I * II[j] - C::b_I) / (1 - eI);
                R nE = noise.next();
                R nI = noise.next();
                R dSE = nE * C::sigma_model * C::sqrt_dt + C::dt * ((1 - S_E[j]) * C::gamma_E * rE[j] - (S_E[j] / C::tau_E));
                R dSI = nI * C::sigma_model * C::sqrt_dt + C::dt * (C::gamma_I * rI[j] - (S_I[j] / C::tau_I));
                S_E[j] += dSE;
                S_I[j] += dSI;
                S_E[j] = std::max((R)0.0, std::min(S_E[j], (R)1.0));
                S_I[j] = std::max((R)0.0, std::min(S_I[j], (R)1.0));
            }
        }
        /* Balloon-Windkessel, once per ms (the double literals promote as in the reference) */
        for (int j = 0; j < N; j++) {
            x[j] = x[j] + C::model_dt * (S_E[j] - C::kappa * x[j] - C::y * (f[j] - 1.0));
            R tmp_f = f[j] + C::model_dt * x[j];
            nu[j] = nu[j] + C::model_dt * C::itau * (f[j] - rpow(nu[j], C::ialpha));
            q[j] = q[j] + C::model_dt * C::itau *
                              (f[j] * (1.0 - rpow(C::oneminrho, (R)(1.0 / f[j]))) / C::rho -
                               rpow(nu[j], C::ialpha) * q[j] / nu[j]);
            f[j] = tmp_f;
        }
        if (ts % TR == 0) {
            for (int j = 0; j < N; j++) {
                size_t o = (size_t)frame * N + j;
                bold[o] = C::V_0 * (C::k1 * (1 - q[j]) + C::k2 * (1 - q[j] / nu[j]) + C::k3 * (1 - nu[j]));
                size_t plane = (size_t)output_ts * N;
                ext[0 * plane + o] = S_E[j];
                ext[1 * plane + o] = IE[j];
                ext[2 * plane + o] = rE[j];
                ext[3 * plane + o] = S_I[j];
                ext[4 * plane + o] = II[j];
                ext[5 * plane + o] = rI[j];
            }
            frame++;
        }
        ts++;
        if (adjusting) {
            if (ts >= fc.sampling_start && ts <= fc.sampling_end)
                for (int j = 0; j < N; j++) mean_IE[j] += IE[j];
            if (ts == fc.sampling_end) {
                bool needs = false;
                for (int j = 0; j < N; j++) {
                    mean_IE[j] /= duration;
                    R diff = mean_IE[j] - C::b_a_ratio_E;
                    if (std::abs(diff + 0.026) > 0.005) {
                        needs = true;
                        if (trial < max_trials) {
                            if (diff < -0.026) {
                                wIE[j] -= delta[j];
                                delta[j] -= 0.001;
                                delta[j] = fmaxf(delta[j], 0.001);
                            } else {
                                wIE[j] += delta[j];
                            }
                        }
                    }
                }
                if (needs) {
                    if (trial < max_trials) {
                        for (int j = 0; j < N; j++) {
                            S_E[j] = 0.001;
                            S_I[j] = 0.001;
                            x[j] = 0.0;
                            f[j] = 1.0;
                            nu[j] = 1.0;
                            q[j] = 1.0;
                            mean_IE[j] = 0;
                        }
                        ts = 0;
                        frame = 0;
                        noise.restart();
                        trial++;
                    } else {
                        failed = true;
                        adjusting = false;
                    }
                } else {
                    adjusting = false;
                }
            }
        }
    }
    for (size_t i = 0; i < (size_t)output_ts * N; i++) bold_out[i] = (double)bold[i];
    for (int j = 0; j < N; j++) wIE_out[j] = (double)wIE[j];
    *trials_out = trial;
    *failed_out = failed ? 1 : 0;
    /* means over frames >= n_vols_remove, accumulated in R like bnm.cpp:359-394 */
    if (ext_out) {
        size_t plane = (size_t)output_ts * N;
        for (int v = 0; v < 6; v++)
            for (int j = 0; j < N; j++) {
                R s = 0;
                for (int i = n_vols_remove; i < output_ts; i++) s += ext[v * plane + (size_t)i * N + j];
                s /= (frame - n_vols_remove);
                ext_out[v * N + j] = (double)s;
            }
    }
}

/* bnm.cpp:390-405 from the r_E means. */
template <typename R>
double fic_penalty(const double *mean_rE, int N, double scale, int reject_failed, int failed) {
    R pen = 0;
    for (int j = 0; j < N; j++) {
        R d = rabs((R)mean_rE[j] - 3);
        if (d > 1) pen += 1 - (rexp((R)(-0.05 * (d - 1))));
    }
    pen *= scale;
    pen /= N;
    if (reject_failed & failed) pen += 1;
    return (double)pen;
}

}  // namespace

extern "C" {

/* The reference's noise stream: mt19937(seed) + normal_distribution<float>,
 * drawn in (ms, substep, node, E|I) order. */
void port_noise(int seed, int64_t n, float *out) {
    std::mt19937 gen(seed);
    std::normal_distribution<float> dist(0, 1);
    for (int64_t i = 0; i < n; i++) out[i] = dist(gen);
}

int port_analytic_fic(int fp32, const double *SC, int N, double G, const double *wEE, const double *wEI,
                      double *wIE_out) {
    /* the reference hands analytical_fic double copies of u_real arrays */
    std::vector<double> sc((size_t)N * N), we(N), wi(N);
    for (size_t i = 0; i < (size_t)N * N; i++) sc[i] = fp32 ? (double)(float)SC[i] : SC[i];
    for (int j = 0; j < N; j++) {
        we[j] = fp32 ? (double)(float)wEE[j] : wEE[j];
        wi[j] = fp32 ? (double)(float)wEI[j] : wEI[j];
    }
    /* G reaches analytical_fic as a u_real (bnm.cpp:26-27, run_CMAES.cpp:160) */
    return fp32 ? analytic_fic<float>(sc.data(), N, (double)(float)G, we.data(), wi.data(), wIE_out)
                : analytic_fic<double>(sc.data(), N, G, we.data(), wi.data(), wIE_out);
}

/* One simulation.  noise may be NULL (draw from mt19937(seed) inline, as
 * bnm.cpp does) or the precomputed stream.  ext_out (6*N, optional): means of
 * S_E, I_E, r_E, S_I, I_I, r_I over frames >= n_vols_remove. */
#define PORT_INTEGRATE(NAME, R)                                                                                     \
    void NAME(const double *SC, int N, double G, const double *wEE, const double *wEI, const double *wIE,         \
              int adjust_fic, int max_trials, int T, int TR, int n_vols_remove, int seed, const float *noise,      \
              int sampling_start, int sampling_end, double init_delta, double *bold_out, double *wIE_out,          \
              int *trials_out, int *failed_out, double *ext_out) {                                                 \
        Noise nz(noise, seed);                                                                                     \
        FicConf fc = {sampling_start, sampling_end, init_delta};                                                   \
        integrate<R>(SC, N, G, wEE, wEI, wIE, adjust_fic, max_trials, T, TR, n_vols_remove, nz, fc, bold_out,     \
                     wIE_out, trials_out, failed_out, ext_out);                                                    \
    }
PORT_INTEGRATE(port_integrate_f64, double)
PORT_INTEGRATE(port_integrate_f32, float)

double port_fic_penalty(int fp32, const double *mean_rE, int N, double scale, int reject_failed, int failed) {
    return fp32 ? fic_penalty<float>(mean_rE, N, scale, reject_failed, failed)
                : fic_penalty<double>(mean_rE, N, scale, reject_failed, failed);
}

/* check_fit.cpp:19-62 on a (n_vols x N) row-major BOLD block.  Returns the
 * pair count or -1 on NaN. */
int port_fc_tril(const double *bold, int n_vols, int N, int exc, double *out) {
    int rh = N / 2, idx = 0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            if (!(i > j)) continue;
            if (exc && ((i < rh) ^ (j < rh))) continue;
            double c = gsl_stats_correlation(bold + i, N, bold + j, N, n_vols);
            if (std::isnan(c)) return -1;
            out[idx++] = c;
        }
    return idx;
}

/* Window table of check_fit.cpp:79-106 (drop_edges=true) on a series of
 * n_vols frames: starts/ends inclusive.  Returns the window count. */
int port_windows(int n_vols, int step, int window_size, int *starts, int *ends, int cap) {
    int first = window_size / 2, last = n_vols - 1 - window_size / 2, n = 0;
    for (int c = first; c <= last; c += step) {
        int s = c - window_size / 2, e = c + window_size / 2;
        if (s < 0) s = 0;
        if (e >= n_vols) e = n_vols - 1;
        if (n < cap) {
            starts[n] = s;
            ends[n] = e;
        }
        n++;
    }
    return n;
}

/* check_fit.cpp:64-136.  window_fc_out (optional) gets [n_windows][n_pairs].
 * Returns the FCD length, -1 on NaN. */
int port_fcd_tril(const double *bold, int n_vols, int N, int step, int window_size, int exc, double *fcd_out,
                  double *window_fc_out) {
    std::vector<int> st(n_vols + 1), en(n_vols + 1);
    int W = port_windows(n_vols, step, window_size, st.data(), en.data(), n_vols + 1);
    int P = N * (N - 1) / 2 - (exc ? (N / 2) * (N / 2) : 0);
    std::vector<double> wfc((size_t)W * P);
    for (int w = 0; w < W; w++) {
        int n = port_fc_tril(bold + (size_t)st[w] * N, en[w] - st[w] + 1, N, exc, wfc.data() + (size_t)w * P);
        if (n < 0) return -1;
    }
    if (window_fc_out) std::copy(wfc.begin(), wfc.end(), window_fc_out);
    int idx = 0;
    for (int a = 0; a < W; a++)
        for (int b = 0; b < W; b++) {
            if (!(a > b)) continue;
            double c = gsl_stats_correlation(wfc.data() + (size_t)a * P, 1, wfc.data() + (size_t)b * P, 1, P);
            if (std::isnan(c)) return -1;
            fcd_out[idx++] = c;
        }
    return idx;
}

/* check_fit.cpp:138-217 on the post-removal BOLD block.  out[0..3] =
 * fc_corr, fc_diff, fcd_ks, cost (cost = max_cost when NaN). */
void port_gof(const double *bold, int n_vols, int N, int step, int window_size, int exc, const double *emp_fc,
              int n_fc, const double *emp_fcd, int n_fcd, int use_fc_diff, double max_cost, double *out) {
    int P = N * (N - 1) / 2 - (exc ? (N / 2) * (N / 2) : 0);
    std::vector<double> fc(P);
    out[0] = out[1] = out[2] = NAN;
    if (port_fc_tril(bold, n_vols, N, exc, fc.data()) < 0) {
        out[3] = max_cost;
        return;
    }
    double r = gsl_stats_correlation(emp_fc, 1, fc.data(), 1, n_fc);
    double cost = 1 - r;
    out[0] = r;
    if (use_fc_diff) {
        double d = std::abs(gsl_stats_mean(emp_fc, 1, n_fc) - gsl_stats_mean(fc.data(), 1, P));
        cost += d;
        out[1] = d;
    }
    std::vector<double> fcd((size_t)n_vols * n_vols / 2 + 1);
    int nf = port_fcd_tril(bold, n_vols, N, step, window_size, exc, fcd.data(), NULL);
    if (nf < 0) {
        out[3] = max_cost;
        return;
    }
    std::vector<double> e(emp_fcd, emp_fcd + n_fcd);
    double ks = ks_stat(e.data(), fcd.data(), n_fcd, nf, NULL);
    out[2] = ks;
    out[3] = cost + ks;
}

/* Two-sample KS statistic (compat/ks.h) on copies. */
double port_ks(const double *x, int n, const double *y, int m) {
    std::vector<double> a(x, x + n), b(y, y + m);
    return ks_stat(a.data(), b.data(), n, m, NULL);
}

/* A batch of independent simulations over OpenMP threads (the shape of
 * bnm.cpp:431-466): integration + GOF + FIC penalty per particle.  Analytic
 * FIC runs when do_fic.  cost_out[i] is the GOF cost (no FIC penalty added);
 * pen_out[i] the FIC penalty. */
void port_run_batch(int fp32, int n_sims, const double *SC, int N, const double *G, const double *wEE,
                    const double *wEI, const double *wIE, int do_fic, int adjust_fic, int max_trials, int T, int TR,
                    int n_vols_remove, int seed, const float *noise, int sampling_start, int sampling_end,
                    double init_delta, int step, int window_size, int exc, const double *emp_fc, int n_fc,
                    const double *emp_fcd, int n_fcd, int use_fc_diff, double max_cost, double pen_scale,
                    int reject_failed, int n_threads, double *cost_out, double *pen_out, double *wIE_out,
                    int *trials_out, int *failed_out) {
    const int output_ts = T / TR + 1, n_vols = output_ts - n_vols_remove;
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < n_sims; p++) {
        std::vector<double> bold((size_t)output_ts * N), ext(6 * (size_t)N), w0(N);
        const double *we = wEE + (size_t)p * N, *wi = wEI + (size_t)p * N;
        for (int j = 0; j < N; j++) w0[j] = wIE[(size_t)p * N + j];
        if (do_fic) {
            if (port_analytic_fic(fp32, SC, N, G[p], we, wi, w0.data()))
                for (int j = 0; j < N; j++) w0[j] = 1.0;
        }
        int tr = 0, fl = 0;
        if (fp32)
            port_integrate_f32(SC, N, G[p], we, wi, w0.data(), do_fic && adjust_fic, max_trials, T, TR,
                               n_vols_remove, seed, noise, sampling_start, sampling_end, init_delta, bold.data(),
                               wIE_out + (size_t)p * N, &tr, &fl, ext.data());
        else
            port_integrate_f64(SC, N, G[p], we, wi, w0.data(), do_fic && adjust_fic, max_trials, T, TR,
                               n_vols_remove, seed, noise, sampling_start, sampling_end, init_delta, bold.data(),
                               wIE_out + (size_t)p * N, &tr, &fl, ext.data());
        trials_out[p] = tr;
        failed_out[p] = fl;
        double g[4];
        port_gof(bold.data() + (size_t)n_vols_remove * N, n_vols, N, step, window_size, exc, emp_fc, n_fc, emp_fcd,
                 n_fcd, use_fc_diff, max_cost, g);
        cost_out[p] = g[3];
        pen_out[p] = do_fic ? port_fic_penalty(fp32, ext.data() + 2 * N, N, pen_scale, reject_failed, fl) : 0.0;
    }
}

}  // extern "C"
