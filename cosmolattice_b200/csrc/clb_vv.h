// clb_vv.h - velocity-Verlet composition weights (VelocityVerletParameters::getCoeffs,
// evolvers/velocityverletparameters.h:23-46), as the reference quotes them.  A VVn step runs
// 2|w| - 1 stages with weight w[i < P ? i : S - i - 1] (velocityverlet.h:67-71).
#pragma once

#include "../../include/clb200.h"

#include <vector>

namespace clb {

inline std::vector<double> vv_coefficients(int ev)
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

// Position-Verlet weights (PositionVerletParameters::getCoeffs, positionverletparameters.h:23-46):
// the reference quotes the same numbers as for the velocity-Verlet scheme of the same order.
inline bool is_pv(int ev) { return ev >= CLB_PV2 && ev <= CLB_PV6_2; }
inline std::vector<double> pv_coefficients(int ev)
{
  return is_pv(ev) ? vv_coefficients(CLB_VV2 + (ev - CLB_PV2)) : std::vector<double>{};
}

} // namespace clb
