// A fake of the engine calls that gb_modelopt.cpp makes, for testing the
// model optimiser's host logic without a GPU.  It keeps the model slots it is
// given and scores a "tree" as a smooth function of each slot's model (its
// rate matrix, discrete-gamma rates, category weights, frequencies and pinv),
// so the optimiser sees a likelihood surface with an interior optimum in every
// parameter.  Test infrastructure only (tests/test_modelopt_host.py).
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/garli_b200.h"

namespace {

const int kS = 4, kR = 4, kSlots = 9, kTax = 11, kPat = 845;

struct Slot {
    double Q[kS * kS] = {0};
    double bm = 1.0;
    double freqs[kS] = {0.25, 0.25, 0.25, 0.25};
    double rates[kR] = {1, 1, 1, 1};
    double weights[kR] = {0.25, 0.25, 0.25, 0.25};
    double pinv = 0.0;
};
Slot g_slot[kSlots];
long long g_models = 0, g_calls = 0;

// a smooth surface with its optimum at Q_ij = Q*_ij (rates 1.5, 3.9, 1.6,
// 1.3, 4.7, 1 under the frequencies below), rates[0] of the gamma at
// alpha = 1.25, pinv = 0.3, frequencies (0.244, 0.243, 0.25, 0.263)
double surface(const Slot &s) {
    static const double pis[kS] = {0.244, 0.243, 0.25, 0.263};
    static const double rel[6] = {1.5, 3.9, 1.6, 1.3, 4.7, 1.0};
    double Qs[kS * kS] = {0};
    double bm = 1.0;
    gbm_gtr_qmat(rel, pis, Qs, &bm);
    double r0[kR];
    gbm_discrete_gamma(1.25, kR, r0);
    double f = -13930.5;
    for (int i = 0; i < kS; i++)
        for (int j = 0; j < kS; j++)
            if (i != j) f -= 40.0 * (s.Q[i * kS + j] - Qs[i * kS + j]) * (s.Q[i * kS + j] - Qs[i * kS + j]);
    f -= 300.0 * (s.rates[0] - r0[0]) * (s.rates[0] - r0[0]);
    f -= 900.0 * (s.pinv - 0.3) * (s.pinv - 0.3) + 50.0 * (s.weights[0] - 0.175) * (s.weights[0] - 0.175);
    for (int i = 0; i < kS; i++) f -= 3000.0 * (s.freqs[i] - pis[i]) * (s.freqs[i] - pis[i]);
    return f;
}

}  // namespace

extern "C" {

int gbt_get_instance(int tree) { return tree == 0 ? 0 : GB_ERROR_UNINITIALIZED_INSTANCE; }

int gb_get_instance_shape(int instance, int *out) {
    if (instance != 0) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out[0] = kTax;
    out[1] = (3 + kSlots - 1) * (kTax - 2);
    out[2] = kS;
    out[3] = kR;
    out[4] = kPat;
    return GB_SUCCESS;
}

int gb_get_instance_capacity(int instance, int *out) {
    if (instance != 0) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out[0] = (3 + kSlots - 1) * (kTax - 2);
    out[1] = kSlots * (2 * kTax - 2);
    out[2] = kSlots;
    return GB_SUCCESS;
}

int gb_set_eigen_from_rate_matrices(int, int count, const int *idx, const double *Q, const double *, const double *bm,
                                    int *) {
    for (int c = 0; c < count; c++) {
        if (idx[c] < 0 || idx[c] >= kSlots) return GB_ERROR_OUT_OF_RANGE;
        std::memcpy(g_slot[idx[c]].Q, Q + (size_t)c * kS * kS, sizeof(double) * kS * kS);
        g_slot[idx[c]].bm = bm[c];
    }
    return GB_SUCCESS;
}

int gb_set_model_slot(int, int e, const double *freqs, const double *rates, const double *weights, double pinv, int) {
    if (e < 0 || e >= kSlots) return GB_ERROR_OUT_OF_RANGE;
    std::memcpy(g_slot[e].freqs, freqs, sizeof(double) * kS);
    std::memcpy(g_slot[e].rates, rates, sizeof(double) * kR);
    std::memcpy(g_slot[e].weights, weights, sizeof(double) * kR);
    g_slot[e].pinv = pinv;
    return GB_SUCCESS;
}

int gbt_make_all_dirty(int) { return GB_SUCCESS; }

int gbt_score(int, int, double *out) {
    out[0] = surface(g_slot[0]);
    return GB_SUCCESS;
}

int gbt_score_models(int, int count, const int *slots, double *lnl) {
    for (int k = 0; k < count; k++) lnl[k] = surface(g_slot[slots[k]]);
    g_models += count;
    g_calls++;
    return GB_SUCCESS;
}

int gbt_optimize_all_branches(int, double, double *out) {
    out[0] = 0.0;
    out[1] = surface(g_slot[0]);
    return GB_SUCCESS;
}

int gbt_get_branch_lengths(int, double *dlen) {
    for (int i = 0; i < 2 * kTax - 2; i++) dlen[i] = 0.1;
    return GB_SUCCESS;
}

int gbt_set_branch_length(int, int, double) { return GB_SUCCESS; }

// calls of gbt_score_models and the models they scored (fake-only)
void fake_counters(long long *out2) {
    out2[0] = g_calls;
    out2[1] = g_models;
}

}  // extern "C"
