// Host-side lookup tables and derived parameters of the time-driven models.
//
// These are computed on the CPU with the same C library calls and the same
// float/double promotions the reference uses, so the device sees bit-identical
// values (compiled with -ffp-contract=off):
//   ExponentialTable        include/simulation/ExponentialTable.h:76-83 (double exp)
//   HH channel-rate table   include/neuron_model/HHTimeDrivenModel.h:372-421 (float expf)
//   NMDA gating table       src/neuron_model/LIFTimeDrivenModel.cpp:26-36 (float expf)
//   conductance decay       e.g. LIFTimeDrivenModel::Calculate_conductance_exp_values,
//                           src/neuron_model/LIFTimeDrivenModel.cpp:244-252 (float expf)
#include <cmath>
#include <cstdint>
#include <vector>
#include "eb_tables.h"

namespace eb {

std::vector<float> make_exp_table() {
    std::vector<float> t(kExptTable);
    const float mn = -20.0f, mx = 20.0f;
    for (int i = 0; i < kExptTable; ++i) {
        float e = mn + ((mx - mn) * i) / (kExptTable - 1);
        t[i] = (float)::exp((double)e);
    }
    return t;
}

float exp_table_aux() { return (kExptTable - 1) / (20.0f - (-20.0f)); }
float hh_table_aux() { return (kHHTable - 1) / (50.0f - (-90.0f)); }

std::vector<float> make_hh_table(float vt) {
    std::vector<float> t((size_t)kHHTable * 6);
    const float mn = -90.0f, mx = 50.0f;
    for (int i = 0; i < kHHTable; ++i) {
        float V = mn + ((mx - mn) * i) / (kHHTable - 1);
        float *o = t.data() + (size_t)i * 6;
        float x = 13.0f - V + vt;
        o[0] = (x == 0.0) ? 1.279999894092334f : 0.32f * x / (::expf(x * 0.25f) - 1.0f);
        x = V - vt - 40.0f;
        o[1] = (x == 0.0) ? 1.400030971093304f : 0.28f * x / (::expf(x * 0.2f) - 1.0f);
        o[2] = 0.128f * ::expf((17.0f - V + vt) * 0.05555555f);
        o[3] = 4.0f / (1.0f + ::expf((40.0f - V + vt) * 0.2f));
        x = 15.0f - V + vt;
        o[4] = (x == 0.0) ? 0.1599999867615418f : 0.032f * x / (::expf(x * 0.2f) - 1.0f);
        o[5] = 0.5f * ::expf((10.0f - V + vt) * 0.025f);
    }
    return t;
}

std::vector<float> make_nmda_table(float e_exc, float e_inh, float *aux) {
    std::vector<float> t(kNmdaTable);
    *aux = (kNmdaTable - 1) / (e_exc - e_inh);
    for (int i = 0; i < kNmdaTable; ++i) {
        float V = e_inh + ((e_exc - e_inh) * i) / (kNmdaTable - 1);
        t[i] = 1.0f / (1.0f + ::expf(-0.062f * V) * (1.2f / 3.57f));
    }
    return t;
}

float decay_factor(float elapsed_ms, float tau_ms) {
    float inv = (float)(1.0 / (double)tau_ms);  // inv_tau_* = 1.0 / tau (double division)
    return ::expf(-elapsed_ms * inv);
}

float inv_double(float x) { return (float)(1. / (double)x); }

void bdf_coefficients(float c[7][7]) {
    static const float num[7][7] = {{1, 1, 0, 0, 0, 0, 0}, {1, 1, 0, 0, 0, 0, 0}, {2, 4, -1, 0, 0, 0, 0},
                                    {6, 18, -9, 2, 0, 0, 0}, {12, 48, -36, 16, -3, 0, 0},
                                    {60, 300, -300, 200, -75, 12, 0},
                                    {60, 360, -450, 400, -225, 72, -10}};
    static const float den[7] = {1, 1, 3, 11, 25, 137, 147};
    for (int r = 0; r < 7; ++r)
        for (int k = 0; k < 7; ++k) c[r][k] = num[r][k] / den[r];
}

double round_propagation_delay(float d) {
    const double minpd = 0.0001, invminpd = 1.0 / 0.0001;
    double r = std::floor((double)d * invminpd + minpd * 0.5) * minpd;
    return r <= 0 ? minpd : r;
}

int64_t delay_units(float d) {
    const double minpd = 0.0001, invminpd = 1.0 / 0.0001;
    double f = std::floor((double)d * invminpd + minpd * 0.5);
    return f <= 0 ? 1 : (int64_t)f;
}

}  // namespace eb
