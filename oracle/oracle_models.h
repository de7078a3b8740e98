// oracle_models.h - entry points of the gauge-sector oracles (test infrastructure; see oracle.cpp).
#pragma once

#include "../include/clb200.h"

#include <string>

namespace oracle_models {

// complex scalar + U(1) links (lphi4U1), oracle_u1.cpp
void *u1_create(const clb_config *cfg, const clb_model_desc *md, std::string &err);
void u1_destroy(void *h);
std::string &u1_err(void *h);
int u1_set_state(void *h, const double *fields, const double *momenta, const clb_scalefactor *sf);
int u1_get_state(void *h, double *fields, double *momenta, clb_scalefactor *sf);
int u1_initialize(void *h, int32_t correct_adot);
int u1_evolve(void *h, int64_t n);
int u1_sync(void *h);
int u1_measure(void *h, double e0, clb_measurement *m);

} // namespace oracle_models
