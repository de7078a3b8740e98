// oracle_models.h - entry points of the gauge-sector oracles (test infrastructure; see oracle.cpp).
#pragma once

#include "../include/clb200.h"

#include <cmath>
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

// The GW sector of a gauge-model oracle: the reference's default GW leapfrog staggered over the
// matter evolver (evolver.h:102-138), u_ij as five components (11, 12, 13, 22, 23) of N^3 sites,
// zero at the start (gwsinitializer.h).  Kick (leapfrog.h:136-139, gwskernels.h:27-33):
// pi_u += h [a^(1+alpha) lapl u + a^(1+alpha) 2 Pi], Pi the traceless part of the anisotropic
// tensor P(x, y, z, out[6]) (00, 01, 02, 11, 12, 22) that the model gives (PITensor.h:52-111), lapl
// as gaugederivatives.h:42-46.  Drift (leapfrog.h:198-201): u += pow(aSI, alpha-3) (dt pi_u).
struct GWs {
  bool on = false, synced = true;
  std::vector<double> u, pi;
  void enable(size_t n3)
  {
    on = true;
    synced = true;
    u.assign(5 * n3, 0.0);
    pi.assign(5 * n3, 0.0);
  }
  template <class Tensor> void kick(int N, double dx, double aI, double alpha, double h, Tensor P)
  {
    const size_t n3 = (size_t)N * N * N;
    const double A = std::pow(aI, 1 + alpha), inv_dx2 = 1.0 / (dx * dx);
    auto at = [N](int x, int y, int z) { return ((size_t)x * N + y) * N + z; };
#pragma omp parallel for schedule(static)
    for (int x = 0; x < N; ++x)
      for (int y = 0; y < N; ++y)
        for (int z = 0; z < N; ++z) {
          const int xp = (x + 1) % N, xm = (x + N - 1) % N, yp = (y + 1) % N, ym = (y + N - 1) % N;
          const int zp = (z + 1) % N, zm = (z + N - 1) % N;
          const size_t s = at(x, y, z);
          double T[6];
          P(x, y, z, T);
          const double third = ((T[0] + T[3]) + T[5]) * (1.0 / 3.0);
          const double S[5] = {T[0] - third, T[1], T[2], T[3] - third, T[4]};
          for (int c = 0; c < 5; ++c) {
            const double *U = u.data() + (size_t)c * n3;
            const double uc = U[s];
            const double tx = (U[at(xp, y, z)] + U[at(xm, y, z)]) - 2 * uc;
            const double ty = (U[at(x, yp, z)] + U[at(x, ym, z)]) - 2 * uc;
            const double tz = (U[at(x, y, zp)] + U[at(x, y, zm)]) - 2 * uc;
            const double K = A * (inv_dx2 * ((tx + ty) + tz)) + (A * 2) * S[c];
            pi[c * n3 + s] = pi[c * n3 + s] + h * K;
          }
        }
  }
  void drift(double p, double dt)
  {
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < u.size(); ++s) u[s] = u[s] + p * (dt * pi[s]);
  }
};

// The gauge part of PITensor.h (:58-111) at one site, added to T in the reference's order:
// 2 Re[D_i phi conj(D_j phi)] (D_i phi = (U_i(x) phi(x+i) - phi(x)) / dx, U_i = complexPhase(
// -dx g A_i)), then -1/a^2/(fStar/omegaStar)^2 pi_A,i pi_A,j and the same of B_i B_j, B = (F_23,
// F_31, F_12), F(A, i, j) = forwDiff(A_j, i) - forwDiff(A_i, j).  ph0/ph1: Re and Im phi; A, pA:
// the three components of A and of its momentum; nb[i]: the site x + i; first: T holds no
// singlet part yet.
inline void gw_gauge_tensor(const double *ph0, const double *ph1, const double *const (&A)[3],
                            const double *const (&pA)[3], const size_t (&nb)[3], size_t s, double dx, double g,
                            double aI, double rfo2, bool first, double (&T)[6])
{
  double dr[3], di[3], B[3], E[3];
  for (int i = 0; i < 3; ++i) {
    const double th = (-dx * g) * A[i][s];
    const double ur = std::cos(th), ui = std::sin(th);
    const double pr = ph0[nb[i]], pm = ph1[nb[i]];
    const double wr = ur * pr - ui * pm, wi = ur * pm + ui * pr;
    dr[i] = (wr - ph0[s]) / dx;
    di[i] = (wi - ph1[s]) / dx;
    E[i] = pA[i][s];
  }
  auto fdA = [&](int j, int i) { return (A[j][nb[i]] - A[j][s]) / dx; };
  B[0] = fdA(2, 1) - fdA(1, 2);
  B[1] = fdA(0, 2) - fdA(2, 0);
  B[2] = fdA(1, 0) - fdA(0, 1);
  const double pref = (-1.0 / (aI * aI)) / rfo2;
  const int I[6] = {0, 0, 0, 1, 1, 2}, J[6] = {0, 1, 2, 1, 2, 2};
  for (int k = 0; k < 6; ++k) {
    const int i = I[k], j = J[k];
    const double c = 2 * (dr[i] * dr[j] + di[i] * di[j]);
    const double e = (pref * E[i]) * E[j];
    const double m = (pref * B[i]) * B[j];
    T[k] = ((first ? c : T[k] + c) + e) + m;
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
int u1_gws_enable(void *h);
GWs *u1_gws(void *h);

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
int su2_gws_enable(void *h);
GWs *su2_gws(void *h);

} // namespace oracle_models
