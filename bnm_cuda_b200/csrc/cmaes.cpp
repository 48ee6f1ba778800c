// Host CMA-ES with the semantics of the reference's CMAES_Points
// (cmaes.cpp:128-557), as a re-entrant object instead of process globals.
//
// It follows Hansen's CMA-ES (2006 review, "Variante 6"; 2016 tutorial,
// "Variante 16") with the reference's boundary handling (Hansen et al. 2009:
// feasible points clipped to [lb, ub], quadratic penalty weighted by
// Gamma/ksi from the inter-quartile range of the costs), the reference's
// early stop (range of the best value over `early_stop_gens` generations
// below `early_stop_tol`), and the reference's random streams:
// std::default_random_engine seeded SeedMW for the first mean and 11+it for
// the samples of generation it, each created afresh on every call.
// The eigen-decomposition C = B D^2 B^T uses cyclic Jacobi rotations with
// eigenvalues sorted by ascending magnitude and each eigenvector's
// largest-magnitude component made positive.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include "../../include/bnm_b200.h"

namespace {

// Symmetric eigen-decomposition (Golub & Van Loan 8.5, cyclic Jacobi).
// a: n x n row-major (lower triangle used), eval[n], evec n x n (columns).
void jacobi_eigen(int n, const std::vector<double>& A, std::vector<double>& eval, std::vector<double>& evec) {
    std::vector<double> a((size_t)n * n), v((size_t)n * n);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            a[i * n + j] = (i >= j) ? A[i * n + j] : A[j * n + i];
            v[i * n + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
        if (off == 0.0) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = a[p * n + q];
                if (apq == 0.0) continue;
                double app = a[p * n + p], aqq = a[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < n; k++) {
                    double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = cs * akp - sn * akq;
                    a[k * n + q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = cs * apk - sn * aqk;
                    a[q * n + k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = cs * vkp - sn * vkq;
                    v[k * n + q] = sn * vkp + cs * vkq;
                }
            }
    }
    eval.assign(n, 0.0);
    evec.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; j++) {
        eval[j] = a[j * n + j];
        int imax = 0;
        for (int i = 1; i < n; i++)
            if (std::fabs(v[i * n + j]) > std::fabs(v[imax * n + j])) imax = i;
        double sgn = (v[imax * n + j] < 0) ? -1.0 : 1.0;
        for (int i = 0; i < n; i++) evec[i * n + j] = sgn * v[i * n + j];
    }
    // selection sort by |eigenvalue| ascending, swapping columns
    for (int i = 0; i + 1 < n; i++) {
        int k = i;
        double ek = eval[i];
        for (int j = i + 1; j < n; j++)
            if (std::fabs(eval[j]) < std::fabs(ek)) {
                k = j;
                ek = eval[j];
            }
        if (k != i) {
            std::swap(eval[i], eval[k]);
            for (int r = 0; r < n; r++) std::swap(evec[r * n + i], evec[r * n + k]);
        }
    }
}

double median_of(std::vector<double> v) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    size_t n = v.size();
    return (n % 2) ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
}

// quantile of sorted data: delta = (n-1) f, linear interpolation.
double quantile_sorted(const std::vector<double>& s, double f) {
    size_t n = s.size();
    double delta = (n - 1) * f;
    size_t i = (size_t)std::floor(delta);
    delta -= (double)i;
    if (i == n - 1) return s[i];
    return (1 - delta) * s[i] + delta * s[i + 1];
}

}  // namespace

struct bnm_cmaes {
    bnm_cmaes_params P;
    int lambda, mue, D, H;
    double sigma;
    double cc = 0, ccov = 0, csigma = 0, dsigma = 0, chiN = 0, muecov = 0, mueeff = 0, c1 = 0, cmue = 0;
    std::vector<double> weights, Gamma, lb, ub, ksi, psigma, pc, m, mpref, malt, IQAhist, CBVfeas, CBGVariables, ww,
        kk, BDz, Temp, corr, corrraw, Helper, tVektor;
    std::vector<int> indexx;
    std::vector<double> C, B, Dm;                 // D x D row-major
    std::vector<double> Vars, Feas, Pref;         // [D][lambda]
    int it = 0, penalty = 0, cancel = 0, hsigma = 0;

    double& c_(int i, int j) { return C[i * D + j]; }
    double& b_(int i, int j) { return B[i * D + j]; }
    double& d_(int i, int j) { return Dm[i * D + j]; }
    double& var(int i, int j) { return Vars[(size_t)i * lambda + j]; }

    int points();
    void make_feasible();
};

// One call of CMAES_Points (cmaes.cpp:128-557).
int bnm_cmaes::points() {
    std::default_random_engine genMW;
    genMW.seed(P.seed_mw);
    std::uniform_real_distribution<double> uni(0, 1.0);
    std::default_random_engine genADr;
    genADr.seed(11 + it);
    std::normal_distribution<double> nrm(0, 1.0);
    const int V = P.variante;

    if (penalty == 0) {
        if (it == 0) {
            double s1 = 0, s2 = 0;
            for (int i = 0; i < mue; i++) {
                if (V == 6) weights[i] = std::log(mue + 1) - std::log(i + 1);
                else if (V == 16) weights[i] = std::log((lambda + 1) / 2.) - std::log(i + 1);
                s1 += weights[i];
                s2 += weights[i] * weights[i];
            }
            for (int i = 0; i < mue; i++) weights[i] /= s1;
            mueeff = (s1 * s1) / s2;
            muecov = mueeff;
            if (V == 16) {
                s1 = 0;
                s2 = 0;
                for (int i = mue; i < lambda; i++) {
                    weights[i] = std::log((lambda + 1) / 2.) - std::log(i + 1);
                    s1 += weights[i];
                    s2 += weights[i] * weights[i];
                }
                double mueeffminus = (s1 * s1) / s2;
                c1 = P.alphacov / (((D + 1.3) * (D + 1.3)) + mueeff);
                double t1 = P.alphacov * (mueeff - 2 + (1 / mueeff)) / (((D + 2) * (D + 2)) + (P.alphacov * mueeff / 2));
                cmue = ((1 - c1) < t1) ? (1 - c1) : t1;
                double amin = 1 + (c1 / cmue);
                double aeff = 1 + ((2 * mueeffminus) / (mueeff + 2));
                double apos = (1 - c1 - cmue) / (D * cmue);
                double t2 = std::min(std::min(amin, aeff), apos);
                for (int i = mue; i < lambda; i++) {
                    weights[i] /= (-1 * s1);
                    weights[i] *= t2;
                }
                cc = (4 + (mueeff / D)) / (D + 4 + (2 * mueeff / D));
                csigma = (mueeff + 2) / (D + mueeff + 5);
            }
            if (V == 6) {
                cc = 4. / (D + 4);
                csigma = (mueeff + 2) / (D + mueeff + 3);
            }
            double t1 = 2. / ((D + std::sqrt(2)) * (D + std::sqrt(2)));
            double t2 = ((2 * mueeff) - 1) / ((D + 2) * (D + 2) + mueeff);
            t2 = (t2 > 1) ? 1 : t2;
            ccov = (1 / muecov) * t1 + (1 - (1 / muecov)) * t2;
            dsigma = 1 + 2 * std::max(0., std::sqrt((mueeff - 1) / (D + 1.)) - 1) + csigma;
            chiN = std::sqrt(D) * (1 - 1. / (4 * D) + 1. / (21 * D * D));
            CBVfeas[D] = 0;
            CBGVariables[D] = -HUGE_VAL;
            for (int i = 0; i < D; i++) {
                CBVfeas[i] = 0;
                CBGVariables[i] = 0;
                psigma[i] = 0;
                pc[i] = 0;
                malt[i] = 0;
                Gamma[i] = 0;
                m[i] = uni(genMW);
                for (int j = 0; j < D; j++) {
                    c_(i, j) = d_(i, j) = b_(i, j) = (i == j) ? 1 : 0;
                }
            }
            for (int i = 0; i < D; i++)
                for (int j = 0; j < lambda; j++) var(i, j) = m[i] + sigma * nrm(genADr);
            for (int i = 0; i < H; i++) IQAhist[i] = 0;
        } else {
            for (int i = 0; i < lambda; i++) ww[i] = corr[i];
            std::sort(corr.begin(), corr.end());
            // map sorted values back to indices; ties keep the original order
            int W1 = 0, W2 = 0;
            for (int i = 0; i < lambda; i++) {
                if (W2 > 1) {
                    W2 -= 1;
                    continue;
                }
                W2 = 0;
                for (int j = 0; j < lambda; j++)
                    if (corr[i] == ww[j]) {
                        indexx[W1] = j;
                        W1 += 1;
                        W2 += 1;
                    }
            }
            if (-corr[0] > CBGVariables[D]) {
                CBVfeas[D] = kk[indexx[0]];
                CBGVariables[D] = -corr[0];
                for (int i = 0; i < D; i++) {
                    CBGVariables[i] = var(i, indexx[0]);
                    CBVfeas[i] = Feas[(size_t)i * lambda + indexx[0]];
                }
            }
            for (int i = 0; i < D; i++) {
                malt[i] = m[i];
                m[i] = 0;
                for (int j = 0; j < mue; j++) m[i] += weights[j] * var(i, indexx[j]);
                BDz[i] = std::sqrt(mueeff) * (m[i] - malt[i]) / sigma;
            }
            for (int i = 0; i < D; i++) {
                double s = 0;
                for (int j = 0; j < D; j++) s += b_(j, i) * BDz[j];
                Temp[i] = s / d_(i, i);
            }
            for (int i = 0; i < D; i++) {
                double s = 0;
                for (int j = 0; j < D; j++) s += b_(i, j) * Temp[j];
                psigma[i] = (1 - csigma) * psigma[i] + std::sqrt(csigma * (2 - csigma)) * s;
            }
            double np2 = 0;
            for (int i = 0; i < D; i++) np2 += psigma[i] * psigma[i];
            if (V == 16)
                hsigma = ((std::sqrt(np2) / std::sqrt(1 - std::pow((1 - csigma), 2 * it))) / chiN < 1.4 + (2. / (D + 1))) ? 1 : 0;
            else if (V == 6)
                hsigma = ((std::sqrt(np2) / std::sqrt(1 - std::pow((1 - csigma), 2 * it))) / chiN < 1.5 + (1. / (D - 0.5))) ? 1 : 0;
            for (int i = 0; i < D; i++) pc[i] = (1 - cc) * pc[i] + hsigma * std::sqrt(cc * (2 - cc)) * BDz[i];
            sigma *= std::exp(((std::sqrt(np2) / chiN) - 1) * csigma / dsigma);
            if (V == 6) {
                for (int i = 0; i < D; i++)
                    for (int j = 0; j <= i; j++) {
                        c_(i, j) = (1 - ccov) * c_(i, j) + (ccov / muecov) * (pc[i] * pc[j] + (1 - hsigma) * cc * (2 - cc) * c_(i, j));
                        for (int k = 0; k < mue; k++)
                            c_(i, j) += ccov * (1 - (1 / muecov)) * weights[k] * (var(i, indexx[k]) - malt[i]) *
                                        (var(j, indexx[k]) - malt[j]) / (sigma * sigma);
                        c_(j, i) = c_(i, j);
                    }
            } else if (V == 16) {
                double wsum = 0;
                for (int i = 0; i < lambda; i++) wsum += weights[i];
                for (int i = 0; i < D; i++)
                    for (int j = 0; j <= i; j++) {
                        c_(i, j) = (1 - c1 - (cmue * wsum)) * c_(i, j) + c1 * (pc[i] * pc[j] + (1 - hsigma) * cc * (2 - cc) * c_(i, j));
                        for (int k = 0; k < mue; k++)
                            c_(i, j) += cmue * weights[k] * (var(i, indexx[k]) - malt[i]) * (var(j, indexx[k]) - malt[j]) /
                                        (sigma * sigma);
                        for (int k = mue; k < lambda; k++) {
                            for (int z = 0; z < D; z++) BDz[z] = (var(z, indexx[k]) - m[z]) / sigma;
                            for (int z = 0; z < D; z++) {
                                double s = 0;
                                for (int zz = 0; zz < D; zz++) s += b_(zz, z) * BDz[zz];
                                Temp[z] = s / d_(z, z);
                            }
                            for (int z = 0; z < D; z++) {
                                double s = 0;
                                for (int zz = 0; zz < D; zz++) s += b_(z, zz) * Temp[zz];
                                Helper[z] = s;
                            }
                            double nh2 = 0;
                            for (int z = 0; z < D; z++) nh2 += Helper[z] * Helper[z];
                            c_(i, j) += cmue * weights[k] * (D / nh2) * (var(i, indexx[k]) - malt[i]) *
                                        (var(j, indexx[k]) - malt[j]) / (sigma * sigma);
                        }
                        c_(j, i) = c_(i, j);
                    }
            }
            std::vector<double> eval, evec;
            jacobi_eigen(D, C, eval, evec);
            for (int i = 0; i < D; i++) {
                if (eval[i] <= 0) cancel = 1;
                d_(i, i) = std::sqrt(eval[i]);
                for (int j = 0; j < D; j++) b_(i, j) = evec[i * D + j];
            }
            if (cancel == 1) {
                std::fprintf(stderr, "C no longer positive definite\n");
                return P.it_max;
            }
            for (int k = 0; k < lambda; k++) {
                for (int i = 0; i < D; i++) Temp[i] = d_(i, i) * nrm(genADr);
                for (int i = 0; i < D; i++) {
                    double s = 0;
                    for (int j = 0; j < D; j++) s += b_(i, j) * Temp[j];
                    var(i, k) = m[i] + sigma * s;
                }
            }
        }
        make_feasible();
        tVektor[it % P.early_stop_gens] = CBGVariables[D];
        if (it > P.early_stop_gens) {
            double mx = tVektor[0], mn = tVektor[0];
            for (double v : tVektor) {
                mx = std::max(mx, v);
                mn = std::min(mn, v);
            }
            if (mx - mn < P.early_stop_tol) return P.it_max;
        }
        it += 1;
    } else if (penalty == 1) {
        penalty = 0;
        std::vector<double> sorted(corrraw.begin(), corrraw.end());
        std::sort(sorted.begin(), sorted.end());
        std::copy(sorted.begin(), sorted.end(), corrraw.begin());
        double IQA = quantile_sorted(sorted, 0.75) - quantile_sorted(sorted, 0.25);
        double diag = 0;
        for (int i = 0; i < D; i++) diag += c_(i, i);
        IQA /= (sigma * sigma * diag);
        IQAhist[(it - 1) % H] = IQA;
        diag = 0;
        for (int i = 0; i < D; i++) {
            if (c_(i, i) <= 0) {
                cancel = 1;
                break;
            }
            diag += std::log(c_(i, i));
            if (m[i] < (lb[i] + P.bound_soft_edge) || m[i] > (ub[i] - P.bound_soft_edge) || it == 1) {
                const int cnt = (it < H) ? it + 1 : H;
                Gamma[i] = 5.0001 * D * median_of(std::vector<double>(IQAhist.begin(), IQAhist.begin() + cnt));
                double thr = 3 * sigma * std::sqrt(c_(i, i)) * std::max(1.0, std::sqrt((double)D) / mueeff);
                int s1 = (m[i] - mpref[i]) < 0.0 ? -1 : 1, s2 = (m[i] - malt[i]) < 0.0 ? -1 : 1;
                if (std::fabs(m[i] - mpref[i]) > thr && s1 == s2) Gamma[i] *= 1.1;
                Gamma[i] *= P.gamma_scale;
            }
        }
        if (cancel == 1) {
            std::fprintf(stderr, "Diagonal of C no longer positive\n");
            return P.it_max;
        }
        for (int i = 0; i < D; i++) ksi[i] = std::exp(0.9 * (std::log(c_(i, i)) - (diag / D)));
    }
    return it;
}

void bnm_cmaes::make_feasible() {
    const double e = P.bound_soft_edge;
    for (int i = 0; i < D; i++) {
        for (int j = 0; j < lambda; j++) {
            const double v = var(i, j);
            const size_t o = (size_t)i * lambda + j;
            Feas[o] = v < lb[i] ? lb[i] : (v > ub[i] ? ub[i] : v);
            Pref[o] = v < (lb[i] + e) ? lb[i] + e : (v > (ub[i] - e) ? ub[i] - e : v);
        }
        mpref[i] = m[i] < (lb[i] + e) ? lb[i] + e : (m[i] > (ub[i] - e) ? ub[i] - e : m[i]);
    }
}

extern "C" void bnm_cmaes_params_default(bnm_cmaes_params* p) {
    std::memset(p, 0, sizeof *p);
    p->lambda = 10;
    p->dimension = 3;
    p->seed_mw = 1;
    p->it_max = 4;
    p->variante = 6;
    p->sigma = 0.5;
    p->alphacov = 2;
    p->gamma_scale = 2.0;
    p->bound_soft_edge = 0.0;
    p->early_stop_gens = 30;
    p->early_stop_tol = (double)(float)1e-3;
}

static double envf(const char* k, double d) {
    const char* v = std::getenv(k);
    return v ? (double)(float)std::atof(v) : d;
}
static int envi(const char* k, int d) {
    const char* v = std::getenv(k);
    return v ? std::atoi(v) : d;
}

// constants.h:106-113 (doubles read through float, helpers.cpp:4-11).
extern "C" void bnm_cmaes_params_from_env(bnm_cmaes_params* p) {
    p->sigma = envf("BNM_CMAES_SIGMA", p->sigma);
    p->alphacov = (double)envi("BNM_CMAES_ALPHACOV", (int)p->alphacov);
    p->variante = envi("BNM_CMAES_VARIANTE", p->variante);
    p->gamma_scale = envf("BNM_CMAES_GAMMA_SCALE", p->gamma_scale);
    p->bound_soft_edge = envf("BNM_CMAES_BOUND_SOFT_EDGE", p->bound_soft_edge);
    p->early_stop_gens = envi("BNM_CMAES_EARLY_STOP_GENS", p->early_stop_gens);
    p->early_stop_tol = envf("BNM_CMAES_EARLY_STOP_TOL", p->early_stop_tol);
}

extern "C" int bnm_cmaes_create(const bnm_cmaes_params* p, bnm_cmaes** out) {
    if (!p || !out || p->lambda < 2 || p->dimension < 1 || p->early_stop_gens < 1 ||
        (p->variante != 6 && p->variante != 16))
        return 1;
    bnm_cmaes* c = new bnm_cmaes();
    c->P = *p;
    c->lambda = p->lambda;
    c->D = p->dimension;
    c->mue = (int)std::floor(p->lambda / 2);
    c->H = (int)(20 + std::ceil((float)(3 * c->D) / (float)c->lambda));
    c->sigma = p->sigma;
    const int L = c->lambda, D = c->D;
    for (auto* v : {&c->weights, &c->ww, &c->kk, &c->corr, &c->corrraw}) v->assign(L, 0.0);
    for (auto* v : {&c->Gamma, &c->ksi, &c->psigma, &c->pc, &c->m, &c->mpref, &c->malt, &c->BDz, &c->Temp, &c->Helper})
        v->assign(D, 0.0);
    c->lb.assign(D, 0.0);
    c->ub.assign(D, 1.0);
    c->IQAhist.assign(c->H, 0.0);
    c->CBVfeas.assign(D + 1, 0.0);
    c->CBGVariables.assign(D + 1, 0.0);
    c->tVektor.assign(p->early_stop_gens, 0.0);
    c->indexx.assign(L, 0);
    c->C.assign((size_t)D * D, 0.0);
    c->B.assign((size_t)D * D, 0.0);
    c->Dm.assign((size_t)D * D, 0.0);
    c->Vars.assign((size_t)D * L, 0.0);
    c->Feas.assign((size_t)D * L, 0.0);
    c->Pref.assign((size_t)D * L, 0.0);
    c->it = c->points();
    *out = c;
    return 0;
}

extern "C" void bnm_cmaes_destroy(bnm_cmaes* c) { delete c; }
extern "C" int32_t bnm_cmaes_iteration(const bnm_cmaes* c) { return c->it; }

extern "C" int bnm_cmaes_samples(const bnm_cmaes* c, double* feas, double* raw, double* pref) {
    const size_t n = (size_t)c->D * c->lambda;
    if (feas) std::copy(c->Feas.begin(), c->Feas.begin() + n, feas);
    if (raw) std::copy(c->Vars.begin(), c->Vars.begin() + n, raw);
    if (pref) std::copy(c->Pref.begin(), c->Pref.begin() + n, pref);
    return 0;
}

// run_CMAES.cpp:787-816: costs in, boundary penalty, next generation.
extern "C" int32_t bnm_cmaes_tell(bnm_cmaes* c, const double* cost, double* penalized) {
    const int L = c->lambda, D = c->D;
    for (int i = 0; i < L; i++) {
        c->corr[i] = cost[i];
        c->corrraw[i] = cost[i];
        c->kk[i] = -cost[i];
    }
    // as in the reference driver, both calls always run and the iteration
    // counter takes each return value (it_max after an early stop or cancel)
    c->penalty = 1;
    c->it = c->points();
    for (int i = 0; i < L; i++)
        for (int j = 0; j < D; j++) {
            const size_t o = (size_t)j * L + i;
            const double d = c->Pref[o] - c->Vars[o];
            c->corr[i] += c->Gamma[j] / c->ksi[j] / D * d * d;
        }
    if (penalized) std::copy(c->corr.begin(), c->corr.end(), penalized);
    c->it = c->points();
    return c->it;
}

// Replace the current generation's sample points (raw, [dim][lambda]) before
// tell(): pre-screened candidates drawn by the caller from N(m, sigma^2 C).
// No counterpart in the reference.
extern "C" int bnm_cmaes_set_samples(bnm_cmaes* c, const double* raw) {
    if (!c || !raw) return 1;
    std::copy(raw, raw + (size_t)c->D * c->lambda, c->Vars.begin());
    c->make_feasible();
    return 0;
}

extern "C" int bnm_cmaes_best(const bnm_cmaes* c, double* x, double* value) {
    if (x) std::copy(c->CBVfeas.begin(), c->CBVfeas.begin() + c->D, x);
    if (value) *value = c->CBVfeas[c->D];
    return 0;
}

extern "C" int bnm_cmaes_params_of(const bnm_cmaes* c, bnm_cmaes_params* out) {
    if (!c || !out) return 1;
    *out = c->P;
    return 0;
}

extern "C" int bnm_cmaes_state(const bnm_cmaes* c, double* mean, double* sigma, double* C) {
    if (mean) std::copy(c->m.begin(), c->m.end(), mean);
    if (sigma) *sigma = c->sigma;
    if (C) std::copy(c->C.begin(), c->C.end(), C);
    return 0;
}

// ------------------------------------------------------------ checkpoint
// The optimiser's whole state in one file: a magic word and format version,
// the parameters, the scalars and every vector with its length, doubles as
// their exact bytes.  The random engines are seeded afresh inside each
// sampling call (SeedMW and 11 + it), so they hold no state of their own.
// No counterpart in the reference (its state is process-global).
namespace {

constexpr uint64_t kCkptMagic = 0x544b50434d424e42ull;  // "BNBMCPKT"
constexpr uint32_t kCkptVersion = 1;

struct Writer {
    std::FILE* f;
    bool ok = true;
    void raw(const void* p, size_t n) { ok = ok && std::fwrite(p, 1, n, f) == n; }
    template <typename T> void put(const T& v) { raw(&v, sizeof v); }
    template <typename T> void vec(const std::vector<T>& v) {
        put((uint64_t)v.size());
        if (!v.empty()) raw(v.data(), v.size() * sizeof(T));
    }
};

struct Reader {
    std::FILE* f;
    bool ok = true;
    void raw(void* p, size_t n) { ok = ok && std::fread(p, 1, n, f) == n; }
    template <typename T> void get(T& v) { raw(&v, sizeof v); }
    template <typename T> void vec(std::vector<T>& v, size_t expect) {
        uint64_t n = 0;
        get(n);
        ok = ok && n == expect;
        if (!ok) return;
        v.assign(n, T());
        if (n) raw(v.data(), n * sizeof(T));
    }
};

template <typename IO, typename S>
void scalars(IO& io, S& c) {
    auto f = [&](auto& x) {
        if constexpr (std::is_same_v<IO, Writer>)
            io.put(x);
        else
            io.get(x);
    };
    f(c.lambda), f(c.mue), f(c.D), f(c.H), f(c.sigma), f(c.cc), f(c.ccov), f(c.csigma), f(c.dsigma), f(c.chiN),
        f(c.muecov), f(c.mueeff), f(c.c1), f(c.cmue), f(c.it), f(c.penalty), f(c.cancel), f(c.hsigma);
}

}  // namespace

extern "C" int bnm_cmaes_save(const bnm_cmaes* c, const char* path) {
    if (!c || !path) return 1;
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return 2;
    Writer w{f};
    w.put(kCkptMagic);
    w.put(kCkptVersion);
    w.put(c->P);
    scalars(w, *c);
    for (const auto* v : {&c->weights, &c->Gamma, &c->lb, &c->ub, &c->ksi, &c->psigma, &c->pc, &c->m, &c->mpref,
                          &c->malt, &c->IQAhist, &c->CBVfeas, &c->CBGVariables, &c->ww, &c->kk, &c->BDz, &c->Temp,
                          &c->corr, &c->corrraw, &c->Helper, &c->tVektor, &c->C, &c->B, &c->Dm, &c->Vars, &c->Feas,
                          &c->Pref})
        w.vec(*v);
    w.vec(c->indexx);
    const bool ok = w.ok && std::fflush(f) == 0;
    if (std::fclose(f) != 0 || !ok) {
        std::remove(tmp.c_str());
        return 2;
    }
    // the file appears whole or not at all
    return std::rename(tmp.c_str(), path) == 0 ? 0 : 2;
}

extern "C" int bnm_cmaes_load(const char* path, bnm_cmaes** out) {
    if (!path || !out) return 1;
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return 2;
    Reader r{f};
    uint64_t magic = 0;
    uint32_t version = 0;
    r.get(magic);
    r.get(version);
    bnm_cmaes* c = new bnm_cmaes();
    r.get(c->P);
    r.ok = r.ok && magic == kCkptMagic && version == kCkptVersion;
    if (r.ok) scalars(r, *c);
    const size_t L = r.ok ? (size_t)std::max(c->lambda, 0) : 0, D = r.ok ? (size_t)std::max(c->D, 0) : 0;
    r.ok = r.ok && L >= 2 && D >= 1 && c->lambda == c->P.lambda && c->D == c->P.dimension && c->H >= 1 &&
           c->P.early_stop_gens >= 1;
    const size_t H = r.ok ? (size_t)c->H : 0, E = r.ok ? (size_t)c->P.early_stop_gens : 0;
    const std::pair<std::vector<double>*, size_t> vs[] = {
        {&c->weights, L}, {&c->Gamma, D},  {&c->lb, D},       {&c->ub, D},           {&c->ksi, D},
        {&c->psigma, D},  {&c->pc, D},     {&c->m, D},        {&c->mpref, D},        {&c->malt, D},
        {&c->IQAhist, H}, {&c->CBVfeas, D + 1}, {&c->CBGVariables, D + 1}, {&c->ww, L}, {&c->kk, L},
        {&c->BDz, D},     {&c->Temp, D},   {&c->corr, L},     {&c->corrraw, L},      {&c->Helper, D},
        {&c->tVektor, E}, {&c->C, D * D},  {&c->B, D * D},    {&c->Dm, D * D},       {&c->Vars, D * L},
        {&c->Feas, D * L}, {&c->Pref, D * L}};
    for (const auto& v : vs)
        if (r.ok) r.vec(*v.first, v.second);
    if (r.ok) r.vec(c->indexx, L);
    char extra;
    r.ok = r.ok && std::fread(&extra, 1, 1, f) == 0;  // nothing after the state
    std::fclose(f);
    if (!r.ok) {
        delete c;
        return 3;
    }
    *out = c;
    return 0;
}
