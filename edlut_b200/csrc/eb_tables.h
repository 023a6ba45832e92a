// Host-side lookup tables and derived parameters (eb_tables.cpp).
#pragma once
#include <cstdint>
#include <vector>
#include "eb_types.h"

namespace eb {
std::vector<float> make_exp_table();
float exp_table_aux();
float hh_table_aux();
std::vector<float> make_hh_table(float v_thr);
std::vector<float> make_nmda_table(float e_exc, float e_inh, float *aux);
float decay_factor(float elapsed_ms, float tau_ms);
float inv_double(float x);
void bdf_coefficients(float c[7][7]);
double round_propagation_delay(float d);
int64_t delay_units(float d);  // round_propagation_delay(d) / 1e-4 as an integer
}  // namespace eb
