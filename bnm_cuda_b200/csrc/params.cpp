// Parameter expansion of one CMA-ES particle (the reference's
// calculate_params, run_CMAES.cpp:61-143): G, and per-node wEE / wEI / wIE
// from base values, optionally scaled per node by regional maps
// (base * (1 + sum_m coef_m * map_m[j])) and shifted so that the smallest
// node value of a heterogeneous parameter is 0.001.  Same operation order and
// double arithmetic as the reference's default build, so the values agree
// bit for bit.
#include <cstdint>
#include <cstring>

#include "../../include/bnm_b200.h"

int bnm_fail_msg(int code, const char* msg);

extern "C" int bnm_calculate_params(int32_t nodes, int32_t het_mask, int32_t n_maps, const double* maps, double G,
                                    double wee, double wie, double wei, const double* scales, double* G_out,
                                    double* w_ee, double* w_ei, double* w_ie) {
    if (nodes < 1 || n_maps < 0 || (het_mask & ~7) || !G_out || !w_ee || !w_ei || !w_ie)
        return bnm_fail_msg(BNM_EINVAL, "calculate_params: bad arguments");
    if (het_mask && (n_maps < 1 || !maps || !scales))
        return bnm_fail_msg(BNM_EINVAL, "calculate_params: heterogeneous parameters need maps and scales");
    // the reference's local parameter order (run_CMAES.cpp:252): wee, wie, wei
    const double base[3] = {wee, wie, wei};
    double* out[3] = {w_ee, w_ie, w_ei};
    *G_out = G;
    double mn[3] = {1000, 1000, 1000}, mx[3] = {-1000, -1000, -1000};
    for (int j = 0; j < nodes; j++) {
        for (int k = 0; k < 3; k++) {
            if (!(het_mask >> k & 1)) continue;
            double scaler = 1;
            for (int m = 0; m < n_maps; m++) scaler += scales[k * n_maps + m] * maps[(size_t)m * nodes + j];
            const double v = base[k] * scaler;
            if (v < mn[k]) mn[k] = v;
            if (v > mx[k]) mx[k] = v;
            out[k][j] = v;
        }
        for (int k = 0; k < 3; k++)
            if (!(het_mask >> k & 1)) out[k][j] = base[k];
    }
    for (int k = 0; k < 3; k++) {
        if (!(het_mask >> k & 1) || !(mn[k] < 0.001)) continue;
        for (int j = 0; j < nodes; j++) out[k][j] -= mn[k] - 0.001;
    }
    return BNM_OK;
}
