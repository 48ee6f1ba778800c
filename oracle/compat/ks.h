/*
 * TEST INFRASTRUCTURE ONLY (oracle).  Stand-in for libks (agentlans/libks,
 * no version pinned by the reference: README.md:31-35 clones its HEAD),
 * which is not installed here.  Called at check_fit.cpp:204-209 and
 * bnm.cu:736-741 as ks_stat(x, y, n, m, NULL); the reference copies the
 * empirical vector first because the call sorts its inputs in place.
 *
 * Restated from the definition of the two-sample Kolmogorov-Smirnov
 * statistic: D = sup_v |F_x(v) - F_y(v)| with right-continuous empirical
 * CDFs, evaluated at every distinct value of the pooled sample (ties
 * between and within samples are stepped over together).  This equals
 * scipy.stats.ks_2samp(...).statistic.  libks' own tie handling is not
 * visible here, so parity at this boundary is unpinned.
 */
#ifndef BNM_ORACLE_KS_H
#define BNM_ORACLE_KS_H
#include <stdlib.h>
#include <math.h>

static int bnm_ks_cmp(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

static double ks_stat(double *x, double *y, size_t n, size_t m, void *unused) {
    (void)unused;
    if (n == 0 || m == 0) return NAN;
    qsort(x, n, sizeof(double), bnm_ks_cmp);
    qsort(y, m, sizeof(double), bnm_ks_cmp);
    size_t i = 0, j = 0;
    double d = 0.0;
    while (i < n && j < m) {
        double v = (x[i] < y[j]) ? x[i] : y[j];
        while (i < n && x[i] <= v) i++;
        while (j < m && y[j] <= v) j++;
        double diff = fabs((double)i / (double)n - (double)j / (double)m);
        if (diff > d) d = diff;
    }
    return d;
}
#endif
