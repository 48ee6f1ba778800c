/*
 * TEST INFRASTRUCTURE ONLY (oracle).  Built into oracle/_ref/ by
 * oracle/Makefile; never linked by the product.
 *
 * Compiles the reference's own, unmodified CPU sources in one translation
 * unit, through run_CMAES.cpp (which includes cmaes.cpp, helpers.cpp and
 * bnm.cpp, and bnm.cpp fic.cpp, constants.h and check_fit.cpp), against the GSL/libks
 * stand-ins in oracle/compat, and exposes plain C entry points so the tests
 * can call the reference directly:
 *
 *   ref_run_simulations   -> run_simulations   bnm.cpp:431-466 (OpenMP CPU path)
 *   ref_fc_tril           -> fc_tril           check_fit.cpp:19-62
 *   ref_fcd_tril          -> fcd_tril          check_fit.cpp:64-136
 *   ref_check_fit_bold    -> check_fit_bold    check_fit.cpp:138-217
 *   ref_analytical_fic    -> analytical_fic    fic.cpp:130-207
 *   ref_cmaes_*           -> CMAES_Points      cmaes.cpp:128-557, driven the
 *                            way main() drives it (run_CMAES.cpp:667-818)
 *   ref_calculate_params  -> calculate_params  run_CMAES.cpp:61-143
 *   ref_run_cmaes_cpu     -> main()            run_CMAES.cpp:177-951 (the CPU
 *                            driver, argv as on its command line)
 *
 * u_real is double by default and float with -DUSE_FLOATS (constants.h:8-22);
 * the entry points take and return double and convert at the boundary.
 * Runtime configuration (BNM_* environment variables) is read by the
 * reference at load time (constants.h:93-116), so set it before loading.
 */
#include <chrono>
#include <ctime>
#include <map>
#include <vector>
#include <string>
/* run_CMAES.cpp itself (CPU build: it includes cmaes.cpp, helpers.cpp and
 * bnm.cpp, run_CMAES.cpp:47-59), with its main() renamed so that this
 * library can expose calculate_params and the whole CPU driver. */
#define main ref_run_cmaes_main
#include "run_CMAES.cpp"
#undef main

extern "C" {

int ref_u_real_size(void) { return (int)sizeof(u_real); }

/* Runtime constants as the reference resolved them at load time. */
void ref_constants(double *out) {
    out[0] = bold_remove_s;
    out[1] = MAX_COST;
    out[2] = I_SAMPLING_START;
    out[3] = I_SAMPLING_END;
    out[4] = I_SAMPLING_DURATION;
    out[5] = numerical_fic;
    out[6] = max_fic_trials_cmaes;
    out[7] = init_delta;
    out[8] = use_fc_diff;
    out[9] = exc_interhemispheric;
    out[10] = fic_penalty_scale;
    out[11] = fic_reject_failed;
    out[12] = sigma;
    out[13] = early_stop_gens;
    out[14] = early_stop_tol;
}

static gsl_matrix *to_gsl(const double *a, int rows, int cols) {
    gsl_matrix *m = gsl_matrix_alloc(rows, cols);
    for (int i = 0; i < rows; i++)
        for (int j = 0; j < cols; j++) gsl_matrix_set(m, i, j, a[(size_t)i * cols + j]);
    return m;
}
static gsl_vector *to_gslv(const double *a, int n) {
    gsl_vector *v = gsl_vector_alloc(n);
    for (int i = 0; i < n; i++) gsl_vector_set(v, i, a[i]);
    return v;
}

void ref_run_simulations(double *corr, double *fic_penalties, const double *G_list, const double *w_EE_list,
                         const double *w_EI_list, const double *w_IE_list, const double *SC, int nodes, int N_SIMS,
                         int calculate_fic_penalty, int time_steps, int BOLD_TR, int rand_seed, int max_fic_trials,
                         const double *emp_fc, int n_emp_fc, const double *emp_fcd, int n_emp_fcd, int sim_only,
                         int no_fcd, int window_step, int window_size, const char *out_prefix, int verbose,
                         int save_output, int extended_output) {
    std::vector<u_real> G(N_SIMS), wee((size_t)N_SIMS * nodes), wei((size_t)N_SIMS * nodes),
        wie((size_t)N_SIMS * nodes), sc((size_t)nodes * nodes), pen(N_SIMS, 0);
    for (int i = 0; i < N_SIMS; i++) G[i] = (u_real)G_list[i];
    for (size_t i = 0; i < (size_t)N_SIMS * nodes; i++) {
        wee[i] = (u_real)w_EE_list[i];
        wei[i] = (u_real)w_EI_list[i];
        wie[i] = (u_real)w_IE_list[i];
    }
    for (size_t i = 0; i < (size_t)nodes * nodes; i++) sc[i] = (u_real)SC[i];
    /* run_CMAES.cpp:363-374 fills SC_gsl from the u_real SC */
    gsl_matrix *sc_gsl = gsl_matrix_alloc(nodes, nodes);
    for (int i = 0; i < nodes; i++)
        for (int j = 0; j < nodes; j++) gsl_matrix_set(sc_gsl, i, j, sc[(size_t)i * nodes + j]);
    gsl_vector *efc = to_gslv(emp_fc, n_emp_fc);
    gsl_vector *efcd = to_gslv(emp_fcd, n_emp_fcd > 0 ? n_emp_fcd : 1);
    if (n_emp_fcd <= 0) efcd->size = 0;
    run_simulations(corr, pen.data(), G.data(), wee.data(), wei.data(), wie.data(), sc.data(), sc_gsl, nodes, N_SIMS,
                    calculate_fic_penalty != 0, time_steps, BOLD_TR, rand_seed, max_fic_trials, efc, efcd,
                    sim_only != 0, no_fcd != 0, window_step, window_size, std::string(out_prefix ? out_prefix : ""),
                    verbose != 0, save_output != 0, extended_output != 0);
    for (int i = 0; i < N_SIMS; i++) fic_penalties[i] = (double)pen[i];
    gsl_vector_free(efc);
    gsl_vector_free(efcd);
    gsl_matrix_free(sc_gsl);
}

/* Returns the number of pairs written, or -1 when the reference reports NaN. */
int ref_fc_tril(const double *bold, int n_vols, int nodes, int exc, double *out) {
    gsl_matrix *b = to_gsl(bold, n_vols, nodes);
    gsl_vector *v = fc_tril(b, exc != 0);
    gsl_matrix_free(b);
    if (!v) return -1;
    int n = (int)v->size;
    for (int i = 0; i < n; i++) out[i] = gsl_vector_get(v, i);
    gsl_vector_free(v);
    return n;
}

int ref_fcd_tril(const double *bold, int n_vols, int nodes, int step, int window_size, int drop_edges, int exc,
                 double *out, int cap) {
    gsl_matrix *b = to_gsl(bold, n_vols, nodes);
    gsl_vector *v = fcd_tril(b, step, window_size, drop_edges != 0, exc != 0);
    gsl_matrix_free(b);
    if (!v) return -1;
    int n = (int)v->size;
    for (int i = 0; i < n && i < cap; i++) out[i] = gsl_vector_get(v, i);
    gsl_vector_free(v);
    return n;
}

double ref_check_fit_bold(const double *bold, int n_vols, int nodes, int step, int window_size, int drop_edges,
                          const double *emp_fc, int n_emp_fc, const double *emp_fcd, int n_emp_fcd, int no_fcd,
                          int exc) {
    gsl_matrix *b = to_gsl(bold, n_vols, nodes);
    gsl_vector *efc = to_gslv(emp_fc, n_emp_fc);
    gsl_vector *efcd = to_gslv(emp_fcd, n_emp_fcd > 0 ? n_emp_fcd : 1);
    double cost = check_fit_bold(b, step, window_size, drop_edges != 0, efc, efcd, no_fcd != 0, false, exc != 0);
    gsl_matrix_free(b);
    gsl_vector_free(efc);
    gsl_vector_free(efcd);
    return cost;
}

double ref_ks_stat(const double *x, int n, const double *y, int m) {
    std::vector<double> a(x, x + n), b(y, y + m);
    return ks_stat(a.data(), b.data(), n, m, NULL);
}

/* Returns the reference's "unstable" flag; wIE_out is written when stable. */
int ref_analytical_fic(const double *SC, int nodes, double G, const double *wEE, const double *wEI, double *wIE_out) {
    gsl_matrix *sc = to_gsl(SC, nodes, nodes);
    gsl_vector *out = gsl_vector_alloc(nodes);
    std::vector<double> we(wEE, wEE + nodes), wi(wEI, wEI + nodes);
    bool unstable = false;
    analytical_fic(sc, G, we.data(), wi.data(), out, &unstable);
    if (!unstable)
        for (int j = 0; j < nodes; j++) wIE_out[j] = gsl_vector_get(out, j);
    gsl_vector_free(out);
    gsl_matrix_free(sc);
    return unstable ? 1 : 0;
}

/* ---- CMA-ES, driven like run_CMAES.cpp main() ---------------------------- */
void ref_cmaes_setup(int lam, int dim, int seed_mw, int it_max) {
    lambda = lam;
    Dimension = dim;
    SeedMW = seed_mw;
    itMax = it_max;
    /* run_CMAES.cpp:668-712 */
    int hist = (int)(20 + std::ceil((float)(3 * Dimension) / (float)lambda));
    weights = new double[lambda];
    Gamma = new double[Dimension];
    lb = new double[Dimension];
    ub = new double[Dimension];
    ksi = new double[Dimension];
    psigma = new double[Dimension];
    pc = new double[Dimension];
    m = new double[Dimension];
    mpref = new double[Dimension];
    malt = new double[Dimension];
    IQAhist = new double[hist];
    IQAhistsort = new double[hist];
    CBVfeas = new double[Dimension + 1];
    CBGVariables = new double[Dimension + 1];
    ww = new double[lambda];
    kk = new double[lambda];
    BDz = new double[Dimension];
    Temporaer = new double[Dimension];
    corr = new double[lambda];
    corrraw = new double[lambda];
    Helper = new double[Dimension];
    C1d = new double[Dimension * Dimension];
    indexx = new int[lambda];
    C = new double *[Dimension];
    B = new double *[Dimension];
    D = new double *[Dimension];
    Variables = new double *[Dimension];
    Variablesfeas = new double *[Dimension];
    Variablespref = new double *[Dimension];
    for (int i = 0; i < Dimension; i++) {
        C[i] = new double[Dimension];
        B[i] = new double[Dimension];
        D[i] = new double[Dimension];
        Variables[i] = new double[lambda];
        Variablesfeas[i] = new double[lambda];
        Variablespref[i] = new double[lambda];
        lb[i] = 0;
        ub[i] = 1;
    }
    mue = std::floor(lambda / 2);
    it = CMAES_Points();
}

int ref_cmaes_it(void) { return it; }

/* Feasible sample points, layout [dim][lambda]. */
void ref_cmaes_get(double *feas, double *vars, double *pref) {
    for (int i = 0; i < Dimension; i++)
        for (int j = 0; j < lambda; j++) {
            if (feas) feas[i * lambda + j] = Variablesfeas[i][j];
            if (vars) vars[i * lambda + j] = Variables[i][j];
            if (pref) pref[i * lambda + j] = Variablespref[i][j];
        }
}

/* One generation's bookkeeping after the simulations, run_CMAES.cpp:787-816:
 * cost[] already holds gof cost (+ FIC penalty).  Writes the boundary-
 * penalised cost per particle and returns the new iteration counter. */
int ref_cmaes_tell(const double *cost, double *penalized) {
    for (int i = 0; i < lambda; i++) {
        corr[i] = cost[i];
        corrraw[i] = corr[i];
        kk[i] = -corr[i];
    }
    penalty = 1;
    it = CMAES_Points();
    for (int i = 0; i < lambda; i++)
        for (int j = 0; j < Dimension; j++)
            corr[i] += Gamma[j] / ksi[j] / Dimension * (Variablespref[j][i] - Variables[j][i]) *
                       (Variablespref[j][i] - Variables[j][i]);
    if (penalized)
        for (int i = 0; i < lambda; i++) penalized[i] = corr[i];
    it = CMAES_Points();
    return it;
}

/* Best feasible point so far (CBVfeas[0..D-1]) and its gof (CBVfeas[D]). */
void ref_cmaes_best(double *out) {
    for (int i = 0; i <= Dimension; i++) out[i] = CBVfeas[i];
}
void ref_cmaes_state(double *mean_out, double *sigma_out, double *C_out) {
    for (int i = 0; i < Dimension; i++) {
        mean_out[i] = m[i];
        for (int j = 0; j < Dimension; j++) C_out[i * Dimension + j] = C[i][j];
    }
    *sigma_out = sigma;
}

/* calculate_params (run_CMAES.cpp:61-143, CPU signature) for one particle.
 * het_mask bit k marks local parameter k of {wee, wie, wei} (run_CMAES.cpp:252)
 * as regional; scales [3][n_maps] are the map coefficients "<param>scale_<m>". */
void ref_calculate_params(int nodes, int het_mask, int n_maps, const double *maps, double G, double wee, double wie,
                          double wei, const double *scales, double *G_out, double *w_ee, double *w_ei,
                          double *w_ie) {
    static const char *local[3] = {"wee", "wie", "wei"};
    std::map<std::string, u_real> cp;
    cp["G"] = (u_real)G;
    cp["wee"] = (u_real)wee;
    cp["wie"] = (u_real)wie;
    cp["wei"] = (u_real)wei;
    std::vector<std::string> het, homo;
    for (int k = 0; k < 3; k++) {
        if (het_mask >> k & 1) {
            het.push_back(local[k]);
            for (int m = 0; m < n_maps; m++)
                cp[std::string(local[k]) + "scale_" + std::to_string(m)] = (u_real)scales[k * n_maps + m];
        } else {
            homo.push_back(local[k]);
        }
    }
    std::vector<std::vector<u_real>> mp(n_maps, std::vector<u_real>(nodes));
    for (int m = 0; m < n_maps; m++)
        for (int j = 0; j < nodes; j++) mp[m][j] = (u_real)maps[(size_t)m * nodes + j];
    std::vector<u_real> g(1), ee(nodes), ei(nodes), ie(nodes);
    calculate_params(g.data(), ee.data(), ei.data(), ie.data(), cp, 0, nodes, het, homo, mp, false);
    *G_out = (double)g[0];
    for (int j = 0; j < nodes; j++) {
        w_ee[j] = (double)ee[j];
        w_ei[j] = (double)ei[j];
        w_ie[j] = (double)ie[j];
    }
}

/* The body of run_simulations' OpenMP loop (bnm.cpp:441-465: one bnm() call
 * per particle, same arguments), with each particle's wall time recorded and,
 * when out_dir is given, each particle's save_output files written under its
 * own prefix <out_dir>/p<i> (run_simulations gives every particle the same
 * prefix), so that the reference's own FIC trial counts can be read back
 * (<prefix>_fic_ntrials.txt, bnm.cpp:301-309).  Used to time full-length
 * simulations of the reference's CPU path. */
void ref_run_particles_timed(double *corr, double *fic_penalties, const double *G_list, const double *w_EE_list,
                             const double *w_EI_list, const double *w_IE_list, const double *SC, int nodes,
                             int N_SIMS, int time_steps, int BOLD_TR, int rand_seed, int max_fic_trials,
                             const double *emp_fc, int n_emp_fc, const double *emp_fcd, int n_emp_fcd,
                             int window_step, int window_size, int sim_only, const char *out_dir, double *seconds) {
    std::vector<u_real> G(N_SIMS), wee((size_t)N_SIMS * nodes), wei((size_t)N_SIMS * nodes),
        wie((size_t)N_SIMS * nodes), sc((size_t)nodes * nodes), pen(N_SIMS, 0);
    for (int i = 0; i < N_SIMS; i++) G[i] = (u_real)G_list[i];
    for (size_t i = 0; i < (size_t)N_SIMS * nodes; i++) {
        wee[i] = (u_real)w_EE_list[i];
        wei[i] = (u_real)w_EI_list[i];
        wie[i] = (u_real)w_IE_list[i];
    }
    for (size_t i = 0; i < (size_t)nodes * nodes; i++) sc[i] = (u_real)SC[i];
    gsl_matrix *sc_gsl = gsl_matrix_alloc(nodes, nodes);
    for (int i = 0; i < nodes; i++)
        for (int j = 0; j < nodes; j++) gsl_matrix_set(sc_gsl, i, j, sc[(size_t)i * nodes + j]);
    gsl_vector *efc = to_gslv(emp_fc, n_emp_fc);
    gsl_vector *efcd = to_gslv(emp_fcd, n_emp_fcd);
    const bool save = out_dir && *out_dir;
#pragma omp parallel for
    for (int i = 0; i < N_SIMS; i++) {
        const std::string prefix = save ? std::string(out_dir) + "/p" + std::to_string(i) : std::string("");
        const double t0 = omp_get_wtime();
        corr[i] = bnm(nodes, sc.data(), sc_gsl, G[i], wee.data() + (size_t)i * nodes, wei.data() + (size_t)i * nodes,
                      wie.data() + (size_t)i * nodes, pen.data() + i, true, time_steps, BOLD_TR, rand_seed,
                      max_fic_trials, efc, efcd, sim_only != 0, false, window_step, window_size, prefix, false, save,
                      false);
        seconds[i] = omp_get_wtime() - t0;
    }
    for (int i = 0; i < N_SIMS; i++) fic_penalties[i] = (double)pen[i];
    gsl_vector_free(efc);
    gsl_vector_free(efcd);
    gsl_matrix_free(sc_gsl);
}

/* The reference's CPU driver (run_CMAES.cpp main()). */
int ref_run_cmaes_cpu(int argc, char **argv) { return ref_run_cmaes_main(argc, argv); }

} /* extern "C" */
