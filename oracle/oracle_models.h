// oracle_models.h - entry points of the gauge-sector oracles (test infrastructure; see oracle.cpp).
#pragma once

#include "../include/clb200.h"

#include <string>
#include <vector>

namespace oracle_models {

// VelocityVerletParameters::getCoeffs (evolvers/velocityverletparameters.h:23-46)
inline std::vector<double> oracle_vv_weights(int ev)
{
  switch (ev) {
  case CLB_VV2: return {1.0};
  case CLB_VV4: return {1.351207191959657771818, -1.702414403875838200264};
  case CLB_VV6: return {0.78451361047755726382, 0.23557321335935813368, -1.1776799841788710069, 1.3151863206839112189};
  case CLB_VV6_2:
    return {0.39216144400731413928, 0.33259913678935943860, -0.70624617255763935981, 0.082213596293550800230,
            0.79854399093482996340};
  case CLB_VV8:
    return {0.74167036435061295345, -0.40910082580003159400, 0.19075471029623837995, -0.57386247111608226666,
            0.29906418130365592384, 0.33462491824529818378,  0.31529309239676659663, -0.79688793935291635402};
  case CLB_VV10:
    return {-0.48159895600253002870, 0.0036303931544595926879, 0.50180317558723140279,  0.28298402624506254868,
            0.80702967895372223806,  -0.026090580538592205447, -0.87286590146318071547, -0.52373568062510581643,
            0.44521844299952789252,  0.18612289547097907887,   0.23137327866438360633,  -0.52191036590418628905,
            0.74866113714499296793,  0.066736511890604057532,  -0.80360324375670830316, 0.91249037635867994571};
  default: return {};
  }
}

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

namespace oracle_models {

// real scalar + complex scalar + SU(2) doublet + U(1) + SU(2) (lphi4SU2U1), oracle_su2.cpp
void *su2_create(const clb_config *cfg, const clb_model_desc *md, std::string &err);
void su2_destroy(void *h);
std::string &su2_err(void *h);
int su2_set_state(void *h, const double *fields, const double *momenta, const clb_scalefactor *sf);
int su2_get_state(void *h, double *fields, double *momenta, clb_scalefactor *sf);
int su2_initialize(void *h, int32_t correct_adot);
int su2_evolve(void *h, int64_t n);
int su2_sync(void *h);
int su2_measure(void *h, double e0, clb_measurement *m);

} // namespace oracle_models
