/*
 * TEST INFRASTRUCTURE ONLY (oracle).  Nothing in the product links this file.
 *
 * A project-written stand-in for the handful of GNU Scientific Library 2.7
 * entry points that the reference's CPU sources call.  GSL itself is not
 * installed here and there is no network, so the reference (check_fit.cpp,
 * fic.cpp, cmaes.cpp, bnm.cpp, run_CMAES.cpp) is compiled against these
 * declarations instead.  Every routine is written from the documented
 * behaviour in the GSL reference manual or from the published numerical
 * method it names; no GSL source is used.
 *
 * Call sites in the reference that these stand in for:
 *   gsl_stats_correlation  check_fit.cpp:48,122,172  bnm.cu:730
 *   gsl_stats_mean         check_fit.cpp:182-183     bnm.cu:746-747
 *   gsl_blas_ddot          fic.cpp:193
 *   Brent root solver      fic.cpp:71-100 (gsl_fsolve)
 *   gsl_eigen_symmv(+sort) cmaes.cpp:392-400
 *   gsl_stats_{max,min}    cmaes.cpp:484-485
 *   gsl_stats_quantile_from_sorted_data  cmaes.cpp:502-503
 *   gsl_stats_median       cmaes.cpp:527,533
 *
 * Known, documented differences from the real library (parity at this
 * boundary is unpinned: there is no GSL here to compare with):
 *   - correlation uses two passes (mean, then centred sums); GSL uses a
 *     one-pass recurrence.  Results agree to round-off.
 *   - the eigen-solver is cyclic Jacobi; eigenvector signs follow a fixed
 *     convention (largest-magnitude component positive), which GSL does not
 *     promise.  CMA-ES samples depend on those signs.
 *   - Brent's method follows Brent (1973), "Algorithms for Minimization
 *     without Derivatives", ch. 4 (zeroin), exposed through GSL's documented
 *     iterate / root / x_lower / x_upper interface.
 */
#ifndef BNM_ORACLE_GSL_COMPAT_H
#define BNM_ORACLE_GSL_COMPAT_H

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>

#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_CONTINUE (-2)
#define GSL_EINVAL 4
#define GSL_EBADFUNC 9
#define GSL_DBL_EPSILON DBL_EPSILON

/* ---------------------------------------------------------------- vectors */
typedef struct {
    size_t size;
    size_t stride;
    double *data;
    void *block;
    int owner;
} gsl_vector;

typedef struct {
    gsl_vector vector;
} gsl_vector_view;

static inline gsl_vector *gsl_vector_alloc(size_t n) {
    gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
    v->size = n;
    v->stride = 1;
    v->data = (double *)malloc((n ? n : 1) * sizeof(double));
    v->block = NULL;
    v->owner = 1;
    return v;
}
static inline gsl_vector *gsl_vector_calloc(size_t n) {
    gsl_vector *v = gsl_vector_alloc(n);
    memset(v->data, 0, (n ? n : 1) * sizeof(double));
    return v;
}
static inline void gsl_vector_free(gsl_vector *v) {
    if (!v) return;
    if (v->owner) free(v->data);
    free(v);
}
static inline double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
static inline void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }
static inline void gsl_vector_set_all(gsl_vector *v, double x) {
    for (size_t i = 0; i < v->size; i++) v->data[i * v->stride] = x;
}
static inline void gsl_vector_set_zero(gsl_vector *v) { gsl_vector_set_all(v, 0.0); }
static inline int gsl_vector_memcpy(gsl_vector *dst, const gsl_vector *src) {
    for (size_t i = 0; i < src->size; i++) dst->data[i * dst->stride] = src->data[i * src->stride];
    return GSL_SUCCESS;
}
static inline int gsl_vector_scale(gsl_vector *v, double a) {
    for (size_t i = 0; i < v->size; i++) v->data[i * v->stride] *= a;
    return GSL_SUCCESS;
}
static inline int gsl_vector_fprintf(FILE *f, const gsl_vector *v, const char *fmt) {
    for (size_t i = 0; i < v->size; i++) {
        fprintf(f, fmt, v->data[i * v->stride]);
        fputc('\n', f);
    }
    return GSL_SUCCESS;
}
static inline gsl_vector_view gsl_vector_view_array(double *base, size_t n) {
    gsl_vector_view w;
    w.vector.size = n;
    w.vector.stride = 1;
    w.vector.data = base;
    w.vector.block = NULL;
    w.vector.owner = 0;
    return w;
}

/* --------------------------------------------------------------- matrices */
typedef struct {
    size_t size1;  /* rows */
    size_t size2;  /* columns */
    size_t tda;    /* row stride in elements */
    double *data;
    void *block;
    int owner;
} gsl_matrix;

typedef struct {
    gsl_matrix matrix;
} gsl_matrix_view;

static inline gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
    gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = (double *)malloc((n1 * n2 ? n1 * n2 : 1) * sizeof(double));
    m->block = NULL;
    m->owner = 1;
    return m;
}
static inline gsl_matrix *gsl_matrix_calloc(size_t n1, size_t n2) {
    gsl_matrix *m = gsl_matrix_alloc(n1, n2);
    memset(m->data, 0, (n1 * n2 ? n1 * n2 : 1) * sizeof(double));
    return m;
}
static inline void gsl_matrix_free(gsl_matrix *m) {
    if (!m) return;
    if (m->owner) free(m->data);
    free(m);
}
static inline double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
static inline void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
static inline void gsl_matrix_set_all(gsl_matrix *m, double x) {
    for (size_t i = 0; i < m->size1; i++)
        for (size_t j = 0; j < m->size2; j++) m->data[i * m->tda + j] = x;
}
static inline void gsl_matrix_set_zero(gsl_matrix *m) { gsl_matrix_set_all(m, 0.0); }
static inline void gsl_matrix_set_identity(gsl_matrix *m) {
    for (size_t i = 0; i < m->size1; i++)
        for (size_t j = 0; j < m->size2; j++) m->data[i * m->tda + j] = (i == j) ? 1.0 : 0.0;
}
static inline int gsl_matrix_scale(gsl_matrix *m, double a) {
    for (size_t i = 0; i < m->size1; i++)
        for (size_t j = 0; j < m->size2; j++) m->data[i * m->tda + j] *= a;
    return GSL_SUCCESS;
}
static inline int gsl_matrix_memcpy(gsl_matrix *dst, const gsl_matrix *src) {
    for (size_t i = 0; i < src->size1; i++)
        for (size_t j = 0; j < src->size2; j++) dst->data[i * dst->tda + j] = src->data[i * src->tda + j];
    return GSL_SUCCESS;
}
static inline int gsl_matrix_add(gsl_matrix *a, const gsl_matrix *b) {
    for (size_t i = 0; i < a->size1; i++)
        for (size_t j = 0; j < a->size2; j++) a->data[i * a->tda + j] += b->data[i * b->tda + j];
    return GSL_SUCCESS;
}
static inline gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j) {
    gsl_vector_view w;
    w.vector.size = m->size1;
    w.vector.stride = m->tda;
    w.vector.data = m->data + j;
    w.vector.block = NULL;
    w.vector.owner = 0;
    return w;
}
static inline gsl_vector_view gsl_matrix_row(gsl_matrix *m, size_t i) {
    gsl_vector_view w;
    w.vector.size = m->size2;
    w.vector.stride = 1;
    w.vector.data = m->data + i * m->tda;
    w.vector.block = NULL;
    w.vector.owner = 0;
    return w;
}
static inline gsl_matrix_view gsl_matrix_submatrix(gsl_matrix *m, size_t k1, size_t k2, size_t n1, size_t n2) {
    gsl_matrix_view w;
    w.matrix.size1 = n1;
    w.matrix.size2 = n2;
    w.matrix.tda = m->tda;
    w.matrix.data = m->data + k1 * m->tda + k2;
    w.matrix.block = NULL;
    w.matrix.owner = 0;
    return w;
}
static inline gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2) {
    gsl_matrix_view w;
    w.matrix.size1 = n1;
    w.matrix.size2 = n2;
    w.matrix.tda = n2;
    w.matrix.data = base;
    w.matrix.block = NULL;
    w.matrix.owner = 0;
    return w;
}
static inline int gsl_matrix_set_col(gsl_matrix *m, size_t j, const gsl_vector *v) {
    for (size_t i = 0; i < m->size1; i++) m->data[i * m->tda + j] = v->data[i * v->stride];
    return GSL_SUCCESS;
}
static inline int gsl_matrix_get_row(gsl_vector *v, const gsl_matrix *m, size_t i) {
    for (size_t j = 0; j < m->size2; j++) v->data[j * v->stride] = m->data[i * m->tda + j];
    return GSL_SUCCESS;
}

/* ------------------------------------------------------------- statistics */
/* Arithmetic mean, plain sum divided by n. */
static inline double gsl_stats_mean(const double data[], size_t stride, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += data[i * stride];
    return s / (double)n;
}
/* Pearson correlation: two passes (means, then centred co-moments). */
static inline double gsl_stats_correlation(const double x[], size_t sx, const double y[], size_t sy, size_t n) {
    double mx = gsl_stats_mean(x, sx, n), my = gsl_stats_mean(y, sy, n);
    double sxx = 0.0, syy = 0.0, sxy = 0.0;
    for (size_t i = 0; i < n; i++) {
        double dx = x[i * sx] - mx, dy = y[i * sy] - my;
        sxx += dx * dx;
        syy += dy * dy;
        sxy += dx * dy;
    }
    return sxy / (sqrt(sxx) * sqrt(syy));
}
static inline double gsl_stats_max(const double data[], size_t stride, size_t n) {
    double m = data[0];
    for (size_t i = 1; i < n; i++)
        if (data[i * stride] > m || isnan(data[i * stride])) m = data[i * stride];
    return m;
}
static inline double gsl_stats_min(const double data[], size_t stride, size_t n) {
    double m = data[0];
    for (size_t i = 1; i < n; i++)
        if (data[i * stride] < m || isnan(data[i * stride])) m = data[i * stride];
    return m;
}
/* Manual: delta = (n-1) f, i = floor(delta); linear interpolation between
 * sorted_data[i] and sorted_data[i+1]. */
static inline double gsl_stats_quantile_from_sorted_data(const double s[], size_t stride, size_t n, double f) {
    double delta = (n - 1) * f;
    size_t i = (size_t)floor(delta);
    delta = delta - (double)i;
    if (n == 0) return 0.0;
    if (i == n - 1) return s[i * stride];
    return (1 - delta) * s[i * stride] + delta * s[(i + 1) * stride];
}
static inline int bnm_compat_cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}
/* Median of unsorted data (even n: mean of the two middle values). */
static inline double gsl_stats_median(double data[], size_t stride, size_t n) {
    if (n == 0) return 0.0;
    double *tmp = (double *)malloc(n * sizeof(double));
    for (size_t i = 0; i < n; i++) tmp[i] = data[i * stride];
    qsort(tmp, n, sizeof(double), bnm_compat_cmp_double);
    double med = (n % 2) ? tmp[n / 2] : 0.5 * (tmp[n / 2 - 1] + tmp[n / 2]);
    free(tmp);
    return med;
}

/* ------------------------------------------------------------------- BLAS */
static inline int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result) {
    double s = 0.0;
    for (size_t i = 0; i < x->size; i++) s += x->data[i * x->stride] * y->data[i * y->stride];
    *result = s;
    return GSL_SUCCESS;
}

/* ------------------------------------------------------------ root finding */
typedef struct {
    double (*function)(double x, void *params);
    void *params;
} gsl_function;
#define GSL_FN_EVAL(F, x) (*((F)->function))(x, (F)->params)

typedef struct {
    const char *name;
} gsl_root_fsolver_type;

typedef struct {
    const gsl_root_fsolver_type *type;
    gsl_function *function;
    double root, x_lower, x_upper;
    /* Brent state: b best estimate, c contrapoint (f(b), f(c) of opposite
     * sign), a previous b; d last step, e step before that. */
    double a, b, c, fa, fb, fc, d, e;
} gsl_root_fsolver;

static const gsl_root_fsolver_type bnm_compat_brent_type = {"brent"};
static const gsl_root_fsolver_type *gsl_root_fsolver_brent = &bnm_compat_brent_type;

static inline gsl_root_fsolver *gsl_root_fsolver_alloc(const gsl_root_fsolver_type *T) {
    gsl_root_fsolver *s = (gsl_root_fsolver *)calloc(1, sizeof(gsl_root_fsolver));
    s->type = T;
    return s;
}
static inline void gsl_root_fsolver_free(gsl_root_fsolver *s) { free(s); }

static inline int gsl_root_fsolver_set(gsl_root_fsolver *s, gsl_function *f, double lo, double hi) {
    s->function = f;
    s->x_lower = lo;
    s->x_upper = hi;
    s->root = 0.5 * (lo + hi);
    s->a = lo;
    s->fa = GSL_FN_EVAL(f, lo);
    s->b = hi;
    s->fb = GSL_FN_EVAL(f, hi);
    s->c = s->a;
    s->fc = s->fa;
    s->d = s->e = hi - lo;
    if ((s->fa < 0.0 && s->fb < 0.0) || (s->fa > 0.0 && s->fb > 0.0)) return GSL_EINVAL;
    return GSL_SUCCESS;
}

/* One step of Brent's zeroin (Brent 1973, ch. 4): keep a bracket [b, c],
 * try inverse quadratic / secant interpolation, fall back to bisection when
 * the interpolated step is not safely inside the bracket or does not shrink
 * fast enough. */
static inline int gsl_root_fsolver_iterate(gsl_root_fsolver *s) {
    gsl_function *f = s->function;
    double a = s->a, b = s->b, c = s->c, fa = s->fa, fb = s->fb, fc = s->fc, d = s->d, e = s->e;
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) {
        c = a;
        fc = fa;
        d = e = b - a;
    }
    if (fabs(fc) < fabs(fb)) {
        a = b; fa = fb;
        b = c; fb = fc;
        c = a; fc = fa;
    }
    double tol = 2.0 * DBL_EPSILON * fabs(b);
    double m = 0.5 * (c - b);
    if (fb == 0.0 || fabs(m) <= tol) {
        s->a = a; s->b = b; s->c = c; s->fa = fa; s->fb = fb; s->fc = fc; s->d = d; s->e = e;
        s->root = b;
        s->x_lower = (b < c) ? b : c;
        s->x_upper = (b < c) ? c : b;
        if (fb == 0.0) s->x_lower = s->x_upper = b;
        return GSL_SUCCESS;
    }
    if (fabs(e) >= tol && fabs(fa) > fabs(fb)) {
        double p, q, r, sr = fb / fa;
        if (a == c) { /* secant */
            p = 2.0 * m * sr;
            q = 1.0 - sr;
        } else { /* inverse quadratic interpolation */
            q = fa / fc;
            r = fb / fc;
            p = sr * (2.0 * m * q * (q - r) - (b - a) * (r - 1.0));
            q = (q - 1.0) * (r - 1.0) * (sr - 1.0);
        }
        if (p > 0.0) q = -q; else p = -p;
        double lim1 = 3.0 * m * q - fabs(tol * q), lim2 = fabs(e * q);
        if (2.0 * p < (lim1 < lim2 ? lim1 : lim2)) {
            e = d;
            d = p / q;
        } else {
            d = m;
            e = m;
        }
    } else {
        d = m;
        e = m;
    }
    a = b;
    fa = fb;
    b += (fabs(d) > tol) ? d : (m > 0.0 ? tol : -tol);
    fb = GSL_FN_EVAL(f, b);
    if (!isfinite(fb)) return GSL_EBADFUNC;
    s->a = a; s->b = b; s->c = c; s->fa = fa; s->fb = fb; s->fc = fc; s->d = d; s->e = e;
    s->root = b;
    /* keep the reported bracket consistent with the sign change */
    double cc = c;
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) cc = a;
    s->x_lower = (b < cc) ? b : cc;
    s->x_upper = (b < cc) ? cc : b;
    return GSL_SUCCESS;
}
static inline double gsl_root_fsolver_root(const gsl_root_fsolver *s) { return s->root; }
static inline double gsl_root_fsolver_x_lower(const gsl_root_fsolver *s) { return s->x_lower; }
static inline double gsl_root_fsolver_x_upper(const gsl_root_fsolver *s) { return s->x_upper; }

/* Manual: success when |a - b| < epsabs + epsrel * min(|a|,|b|), with the
 * min replaced by 0 when the interval contains the origin. */
static inline int gsl_root_test_interval(double lo, double hi, double epsabs, double epsrel) {
    double abs_lo = fabs(lo), abs_hi = fabs(hi);
    if (epsrel < 0.0 || epsabs < 0.0 || lo > hi) return GSL_EINVAL;
    double min_abs = ((lo > 0.0 && hi > 0.0) || (lo < 0.0 && hi < 0.0)) ? (abs_lo < abs_hi ? abs_lo : abs_hi) : 0.0;
    double tolerance = epsabs + epsrel * min_abs;
    if (fabs(hi - lo) < tolerance) return GSL_SUCCESS;
    return GSL_CONTINUE;
}

/* ----------------------------------------------------- symmetric eigen */
typedef struct {
    size_t size;
} gsl_eigen_symmv_workspace;

typedef enum {
    GSL_EIGEN_SORT_VAL_ASC,
    GSL_EIGEN_SORT_VAL_DESC,
    GSL_EIGEN_SORT_ABS_ASC,
    GSL_EIGEN_SORT_ABS_DESC
} gsl_eigen_sort_t;

static inline gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n) {
    gsl_eigen_symmv_workspace *w = (gsl_eigen_symmv_workspace *)malloc(sizeof(gsl_eigen_symmv_workspace));
    w->size = n;
    return w;
}
static inline void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { free(w); }

/* Cyclic Jacobi rotations (Golub & Van Loan, "Matrix Computations", 8.5).
 * Like GSL, the lower triangle of A is destroyed. Eigenvectors are the
 * columns of evec; each is scaled so its largest-magnitude component is
 * positive. */
static inline int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w) {
    size_t n = A->size1;
    (void)w;
    double *a = (double *)malloc(n * n * sizeof(double));
    double *v = (double *)malloc(n * n * sizeof(double));
    for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < n; j++) {
            /* symmetric input: use the lower triangle as the source */
            a[i * n + j] = (i >= j) ? gsl_matrix_get(A, i, j) : gsl_matrix_get(A, j, i);
            v[i * n + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (size_t p = 0; p < n; p++)
            for (size_t q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
        if (off == 0.0) break;
        for (size_t p = 0; p < n; p++) {
            for (size_t q = p + 1; q < n; q++) {
                double apq = a[p * n + q];
                if (apq == 0.0) continue;
                double app = a[p * n + p], aqq = a[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (size_t k = 0; k < n; k++) {
                    double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = cs * akp - sn * akq;
                    a[k * n + q] = sn * akp + cs * akq;
                }
                for (size_t k = 0; k < n; k++) {
                    double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = cs * apk - sn * aqk;
                    a[q * n + k] = sn * apk + cs * aqk;
                }
                for (size_t k = 0; k < n; k++) {
                    double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = cs * vkp - sn * vkq;
                    v[k * n + q] = sn * vkp + cs * vkq;
                }
            }
        }
    }
    for (size_t j = 0; j < n; j++) {
        gsl_vector_set(eval, j, a[j * n + j]);
        size_t imax = 0;
        for (size_t i = 1; i < n; i++)
            if (fabs(v[i * n + j]) > fabs(v[imax * n + j])) imax = i;
        double sgn = (v[imax * n + j] < 0) ? -1.0 : 1.0;
        for (size_t i = 0; i < n; i++) gsl_matrix_set(evec, i, j, sgn * v[i * n + j]);
    }
    for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < i; j++) gsl_matrix_set(A, i, j, 0.0);
    free(a);
    free(v);
    return GSL_SUCCESS;
}

/* Stable selection sort of (eval, evec column) pairs by the chosen key. */
static inline int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, gsl_eigen_sort_t type) {
    size_t n = eval->size;
    for (size_t i = 0; i + 1 < n; i++) {
        size_t k = i;
        double ek = gsl_vector_get(eval, i);
        for (size_t j = i + 1; j < n; j++) {
            double ej = gsl_vector_get(eval, j);
            int better = 0;
            switch (type) {
                case GSL_EIGEN_SORT_VAL_ASC: better = ej < ek; break;
                case GSL_EIGEN_SORT_VAL_DESC: better = ej > ek; break;
                case GSL_EIGEN_SORT_ABS_ASC: better = fabs(ej) < fabs(ek); break;
                case GSL_EIGEN_SORT_ABS_DESC: better = fabs(ej) > fabs(ek); break;
            }
            if (better) { k = j; ek = ej; }
        }
        if (k != i) {
            double tmp = gsl_vector_get(eval, i);
            gsl_vector_set(eval, i, gsl_vector_get(eval, k));
            gsl_vector_set(eval, k, tmp);
            for (size_t r = 0; r < evec->size1; r++) {
                double t2 = gsl_matrix_get(evec, r, i);
                gsl_matrix_set(evec, r, i, gsl_matrix_get(evec, r, k));
                gsl_matrix_set(evec, r, k, t2);
            }
        }
    }
    return GSL_SUCCESS;
}

#endif
