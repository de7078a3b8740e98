// oracle.cpp - FP64 CPU restatement of CosmoLattice's lattice time evolution.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is loaded by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the product path.
//
// It restates, in the reference's own operation order, the arithmetic of
//   evolvers/velocityverlet.h:51-266, evolvers/velocityverletparameters.h:23-46,
//   evolvers/leapfrog.h:29-277, evolvers/positionverlet.h:45-276,
//   evolvers/positionverletparameters.h:23-46, evolvers/kernels/scalarsingletkernels.h:30-40,
//   evolvers/kernels/scalefactorkernels.h:27-80, definitions/energies.h:37-239,
//   definitions/averages.h:27-129, definitions/fieldfunctionals.h:52-67,
//   definitions/gaugederivatives.h:36-73, definitions/hubbleconstraint.h:27-36,
//   measurements/energiesmeasurer.h:45-122, measurements/meansmeasurer.h:28-48,
//   initializers/modelinitializer.h:73-80 and models/lphi4.h:154-226
// (paths relative to the reference's include/CosmoInterface or the reference root).
//
// Parity status: the operators that live in the un-vendored TempLat runtime (LatLapl, Grad2,
// average, pow<N>) are restated from their in-tree definitions where one exists
// (gaugederivatives.h:36-40 Laplacian, :70-73 forward gradient) and otherwise by a stated choice;
// the reference's tests hold no golden vectors for this path, so the oracle is pinned only by
// physics known-answer tests (see tests/test_oracle_*.py): parity unpinned against TempLat itself.
//
// Deterministic: every volume sum is formed per x-plane (fixed z, then y order), and the planes
// are added in x order, independent of the OpenMP thread count.

#include "../include/clb200.h"
#include "oracle_models.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Integer power by repeated multiplication; negative exponents invert the positive power.
// (TempLat pow<N>; restated choice.)
inline double ipow(double x, int n)
{
  if (n == 0) return 1.0;
  if (n < 0) return 1.0 / ipow(x, -n);
  double r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return r;
}

// Composition coefficients, velocityverletparameters.h:23-46.
std::vector<double> vvCoeffs(int ev)
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

// Position-Verlet composition coefficients, positionverletparameters.h:23-46 (the same numbers).
bool isPV(int ev) { return ev >= CLB_PV2 && ev <= CLB_PV6_2; }
std::vector<double> pvCoeffs(int ev) { return isPV(ev) ? vvCoeffs(CLB_VV2 + (ev - CLB_PV2)) : std::vector<double>{}; }

struct Oracle {
  clb_config cfg;
  clb_model_desc md;
  int N;
  size_t n3;
  int Ns;
  std::vector<double> fld, pi; // Ns x N^3 each

  // ScaleFactorBase (scalefactorbase.h:20-21) and cached averages (scalarbase.h, abstractmodel.h:142)
  double aI = 1, aSI = 1, aIM = 1, aDotI = 0, aDotSI = 0, aDotSIM = 0;
  double pi2AvI = 0, pi2AvSI = 0, pi2AvSIM = 0, grad2AvI = 0, potAvI = 0, potAvSI = 0;
  double pi2AvIM = 0, grad2AvSI = 0; // position Verlet (positionverlet.h:238-276)
  // fixed background (fixedbackgroundexpansion.h:21-45): pEoS, H0 and the main loop's time t
  bool fb = false;
  double pEoS = 0, H0fb = 0, t = 0;
  double aBg(double dtm) const { return std::pow(1 + H0fb / pEoS * dtm, pEoS); }
  double aBgDot(double dtm) const { return H0fb * std::pow(1 + H0fb / pEoS * dtm, pEoS - 1); }
  bool synced = true;   // LeapFrog::synced (leapfrog.h:31)
  bool initialized = false;
  std::vector<double> ws;
  std::string err;

  size_t at(int x, int y, int z) const { return ((size_t)x * N + y) * N + z; }
  int up(int i) const { return i + 1 == N ? 0 : i + 1; }
  int dn(int i) const { return i == 0 ? N - 1 : i - 1; }

  double *F(int f) { return fld.data() + (size_t)f * n3; }
  double *P(int f) { return pi.data() + (size_t)f * n3; }

  // ---- model: lphi4 (models/lphi4.h:154-226), c0 = couplings[0] (1 in the reference), q = couplings[1]
  double c0() const { return md.couplings[0]; }
  double q() const { return md.couplings[1]; }

  // The scalar-singlet model: 0 lphi4 (above), 1 tanh2 (models/tanh2.h), set by orc_set_scalar_model.
  // tanh2 couplings: mu = M / phi_i = couplings[0], q = couplings[1]; x = phi / mu.
  int scalar_model = 0;
  double mu() const { return md.couplings[0]; }

  // lphi4 potentialTerms(Tag<0>) = 0.25 * pow<4>(phi);  Tag<1> = 0.5 * q * pow<2>(phi * chi)
  // tanh2 potentialTerms(Tag<0>) = pow<2>(M/phi_i) pow<2>(tanh(phi phi_i/M)) / 2 (tanh2.h)
  double potTerm(int k, size_t s) const
  {
    const double p = fld[s];
    if (k == 0 && scalar_model == 1) {
      const double t = std::tanh(p * (1.0 / mu()));
      return ((mu() * mu()) * (t * t)) * 0.5;
    }
    if (k == 0) return (0.25 * c0()) * ipow(p, 4);
    const double c = fld[n3 + s];
    return (0.5 * q()) * ipow(p * c, 2);
  }
  double potential(size_t s) const
  {
    double v = potTerm(0, s);
    if (Ns > 1) v = v + potTerm(1, s);
    return v;
  }
  // potDeriv(Tag<0>) = pow<3>(phi) + q * phi * pow<2>(chi);  Tag<1> = q * chi * pow<2>(phi)
  // tanh2 potDeriv(Tag<0>) = 2 (M/phi_i) pow<2>(tanh(x)) / sinh(2 x) + q phi chi^2 (tanh2.h)
  double potDeriv(int f, size_t s) const
  {
    const double p = fld[s];
    double d0;
    if (scalar_model == 1) {
      const double x = p * (1.0 / mu()), t = std::tanh(x);
      d0 = ((2 * mu()) * (t * t)) / std::sinh(2 * x);
    } else {
      d0 = c0() * ipow(p, 3);
    }
    if (Ns == 1) return d0;
    const double c = fld[n3 + s];
    if (f == 0) return d0 + (q() * p) * ipow(c, 2);
    return (q() * c) * ipow(p, 2);
  }

  // Lattice Laplacian: (1/dx^2) * sum_i [f(x+i) + f(x-i) - 2 f(x)]  (gaugederivatives.h:36-40)
  double lapl(const double *f, int x, int y, int z) const
  {
    const double c = f[at(x, y, z)];
    const double tx = (f[at(up(x), y, z)] + f[at(dn(x), y, z)]) - 2 * c;
    const double ty = (f[at(x, up(y), z)] + f[at(x, dn(y), z)]) - 2 * c;
    const double tz = (f[at(x, y, up(z))] + f[at(x, y, dn(z))]) - 2 * c;
    return (1.0 / (md_dx() * md_dx())) * ((tx + ty) + tz);
  }
  double md_dx() const { return cfg.dx; }

  // Sum over the forward-difference gradient squared, sum_i (f(x+i)-f(x))^2 / dx^2
  // (Grad2 of fieldfunctionals.h:52-56 with the forward derivative of gaugederivatives.h:70-73).
  double grad2(const double *f, int x, int y, int z) const
  {
    const double c = f[at(x, y, z)];
    const double gx = f[at(up(x), y, z)] - c;
    const double gy = f[at(x, up(y), z)] - c;
    const double gz = f[at(x, y, up(z))] - c;
    return ((gx * gx + gy * gy) + gz * gz) * (1.0 / (cfg.dx * cfg.dx));
  }

  // Deterministic volume average of a per-site functional g(x,y,z).
  template <class G> double average(G g) const
  {
    std::vector<double> planes(N, 0.0);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < N; ++x) {
      double sx = 0;
      for (int y = 0; y < N; ++y) {
        double sy = 0;
        for (int z = 0; z < N; ++z) sy += g(x, y, z);
        sx += sy;
      }
      planes[x] = sx;
    }
    double s = 0;
    for (int x = 0; x < N; ++x) s += planes[x];
    return s / (double)n3;
  }

  // ---- Averages (averages.h:290-298, velocityverlet.h:249-266)
  double avPi2()
  {
    return average([&](int x, int y, int z) {
      const size_t s = at(x, y, z);
      double v = pi[s] * pi[s];
      for (int f = 1; f < Ns; ++f) v = v + pi[f * n3 + s] * pi[f * n3 + s];
      return v;
    });
  }
  double avGrad2()
  {
    return average([&](int x, int y, int z) {
      double v = grad2(F(0), x, y, z);
      for (int f = 1; f < Ns; ++f) v = v + grad2(F(f), x, y, z);
      return v;
    });
  }
  double avPot()
  {
    return average([&](int x, int y, int z) { return potential(at(x, y, z)); });
  }

  // ---- Energies (energies.h:37-45): kineticS = 0.5 * <pi^2> * a^-6, gradientS = 0.5 * <grad^2> * a^-2
  double kineticS(double fldf) const { return (0.5 * fldf) * ipow(aI, -6); }
  double gradientS(double fldf) const { return (0.5 * fldf) * ipow(aI, -2); }

  // ScaleFactorKernels::get (scalefactorkernels.h:73-77), scalar singlets only.
  double sfKernel() const
  {
    const double al = md.alpha;
    const double Eks = kineticS(pi2AvI);
    const double Egs = gradientS(grad2AvI);
    const double fm = md.fStar / md.MPl;
    return std::pow(aI, 2 * al + 1) / 3.0 * (fm * fm) *
           ((((al - 2) * Eks + al * Egs) + (al - 1) * 0.0) + (al + 1) * potAvI);
  }

  // ScaleFactorKernels::getSI (scalefactorkernels.h:83-119): the half-step averages at aI.
  double sfKernelSI() const
  {
    const double al = md.alpha;
    const double Eks = kineticS(pi2AvSI);
    const double Egs = gradientS(grad2AvSI);
    const double fm = md.fStar / md.MPl;
    return std::pow(aI, 2 * al + 1) / 3.0 * (fm * fm) *
           ((((al - 2) * Eks + al * Egs) + (al - 1) * 0.0) + (al + 1) * potAvSI);
  }

  // ---- Sweeps
  // Kick: pi += h * [a^(1+alpha) lapl(phi) - a^(3+alpha) dV/dphi]  (scalarsingletkernels.h:30-40)
  void kick(double h)
  {
    // In place: the kick reads phi (stencil) and pi only at the site it writes.
    const double A = std::pow(aI, 1 + md.alpha);
    const double B = std::pow(aI, 3 + md.alpha);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < N; ++x)
      for (int y = 0; y < N; ++y)
        for (int z = 0; z < N; ++z) {
          const size_t s = at(x, y, z);
          for (int f = 0; f < Ns; ++f) {
            const double K = A * lapl(F(f), x, y, z) - B * potDeriv(f, s);
            pi[f * n3 + s] = pi[f * n3 + s] + h * K;
          }
        }
  }
  // Drift: phi += pow(aSI, alpha-3) * (c * pi)  (velocityverlet.h:181-184, leapfrog.h:185-190)
  void drift(double c)
  {
    const double p = std::pow(aSI, md.alpha - 3);
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < (size_t)Ns * n3; ++s) fld[s] = fld[s] + p * (c * pi[s]);
  }

  // Position-Verlet drift: phi += pow(aI, alpha-3) * (c * pi)  (positionverlet.h:170-173)
  void driftPV(double c)
  {
    const double p = std::pow(aI, md.alpha - 3);
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < (size_t)Ns * n3; ++s) fld[s] = fld[s] + p * (c * pi[s]);
  }

  // ---- gravitational waves (evolver.h:102-138 with the default doLFforGWs: a leapfrog staggered
  // over the matter evolver).  Five components of the traceless symmetric u_ij (11, 12, 13, 22,
  // 23; u_33 = -u_11 - u_22, as gwsprojector.h reads them), zero at the start (gwsinitializer.h).
  // Kick (leapfrog.h:136-139, gwskernels.h:27-33): pi_u += (w dt) [a^(1+alpha) lapl u
  // + a^(1+alpha) 2 Pi], Pi the traceless part of sum_a forwDiff_i phi_a forwDiff_j phi_a
  // (PITensor.h scalar-singlet source; forwDiff (f(x+i) - f(x)) / dx, gaugederivatives.h:70-73;
  // lapl as gaugederivatives.h:42-46).  Drift (leapfrog.h:198-201): u += pow(aSI, alpha-3) (dt pi_u).
  bool gws = false, gwSynced = true;
  std::vector<double> gu, gpi;
  void gwKick(double w)
  {
    const double A = std::pow(aI, 1 + md.alpha);
    const double h = w * cfg.dt;
    const double dx = cfg.dx;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < N; ++x)
      for (int y = 0; y < N; ++y)
        for (int z = 0; z < N; ++z) {
          const size_t s = at(x, y, z);
          const size_t nb[3] = {at(up(x), y, z), at(x, up(y), z), at(x, y, up(z))};
          double P[6] = {0, 0, 0, 0, 0, 0}; // 00, 01, 02, 11, 12, 22
          for (int f = 0; f < Ns; ++f) {
            const double *F0 = fld.data() + (size_t)f * n3;
            double g[3];
            for (int i = 0; i < 3; ++i) g[i] = (F0[nb[i]] - F0[s]) / dx;
            const double t[6] = {g[0] * g[0], g[0] * g[1], g[0] * g[2], g[1] * g[1], g[1] * g[2], g[2] * g[2]};
            for (int k = 0; k < 6; ++k) P[k] = f == 0 ? t[k] : P[k] + t[k];
          }
          const double third = ((P[0] + P[3]) + P[5]) * (1.0 / 3.0);
          const double S[5] = {P[0] - third, P[1], P[2], P[3] - third, P[4]};
          for (int c = 0; c < 5; ++c) {
            const double K = A * lapl(gu.data() + (size_t)c * n3, x, y, z) + (A * 2) * S[c];
            gpi[c * n3 + s] = gpi[c * n3 + s] + h * K;
          }
        }
  }
  void gwDrift()
  {
    const double p = std::pow(aSI, md.alpha - 3);
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < 5 * n3; ++s) gu[s] = gu[s] + p * (cfg.dt * gpi[s]);
  }

  // ---- Averages::setAllAverages (averages.h:349-358)
  void setAllAverages()
  {
    potAvI = avPot();
    potAvSI = potAvI;
    pi2AvI = avPi2();
    pi2AvSI = pi2AvI;
    grad2AvI = avGrad2();
  }

  // Energies::rho (energies.h:217-239) and HubbleConstraint::get (hubbleconstraint.h:27-36)
  void hubble(double out[3])
  {
    setAllAverages();
    const double rho = (kineticS(pi2AvI) + gradientS(grad2AvI)) + potAvI;
    const double LHS = aDotI * aDotI;
    const double fm = md.fStar / md.MPl;
    const double RHS = std::pow(aI, 2 * md.alpha + 2) / 3. * (fm * fm) * rho;
    out[0] = (LHS - RHS) / (LHS + RHS);
    out[1] = LHS;
    out[2] = RHS;
  }

  // ---- VelocityVerlet::evolve (velocityverlet.h:51-114), self-consistent or no expansion
  void evolveVV()
  {
    const double dt = cfg.dt;
    const size_t P = ws.size();
    const size_t stages = (P - 1) * 2 + 1;
    const bool ex = cfg.expansion != 0;
    if (fb) { // velocityverlet.h:74-118 with driftScaleFactor's fixed branch (:225-231)
      double tcurrent = t - cfg.t0;
      for (size_t i = 0; i < stages; ++i) {
        const double w = ws[i < P ? i : stages - i - 1];
        kick(w * dt / 2);
        aIM = aI;
        aI = aBg(tcurrent + w * dt);
        drift(dt * w);
        kick(w * dt / 2);
        tcurrent += dt * w;
      }
      return;
    }
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < P ? i : stages - i - 1];
      if (ex) aDotSI = aDotI + (dt / 2) * sfKernel() * w;   // kickScaleFactorHalf (:165-169)
      kick(w * dt / 2);                                      // kickScalar (:129-132)
      if (ex) {
        pi2AvI = avPi2();                                    // storeMomentaAverages (:249-256)
        aIM = aI;                                            // driftScaleFactor (:225-243)
        aI += dt * aDotSI * w;
        aSI = (aIM + aI) / 2.0;
      }
      drift(dt * w);                                         // driftScalar (:181-184)
      if (ex) {                                              // storeFieldsAverages (:258-266)
        grad2AvI = avGrad2();
        potAvI = avPot();
      }
      kick(w * dt / 2);
      if (ex) {
        pi2AvI = avPi2();
        aDotI = aDotSI + (dt / 2) * sfKernel() * w;          // kickScaleFactorOne (:171-174)
      }
    }
  }

  // ---- PositionVerlet::evolve (positionverlet.h:45-99), self-consistent or no expansion
  void evolvePV()
  {
    const double dt = cfg.dt;
    const size_t P = ws.size();
    const size_t stages = (P - 1) * 2 + 1;
    const bool ex = cfg.expansion != 0;
    if (fb) { // positionverlet.h:45-99 with the fixed branches of :207-235
      double tcurrent = t - cfg.t0;
      for (size_t i = 0; i < stages; ++i) {
        const double w = ws[i < P ? i : stages - i - 1];
        driftPV(dt / 2 * w);
        aIM = aI;
        aI = aBg(tcurrent + w * dt / 2.0);
        aSI = aI;
        kick(w * dt);
        aI = aBg(tcurrent + w * dt);
        driftPV(dt / 2 * w);
        tcurrent += dt * w;
      }
      return;
    }
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < P ? i : stages - i - 1];
      driftPV(dt / 2 * w);                                   // driftScalar (:170-173)
      if (ex) {
        aIM = aI;                                            // driftScaleFactorFirstHalf (:209-222)
        aI += dt / 2.0 * aDotI * w;
        aSI = aI;
        grad2AvSI = avGrad2();                               // storeFieldsAveragesHalf (:258-266)
        potAvSI = avPot();
      }
      kick(w * dt);                                          // kickScalar (:132-135)
      if (ex) {
        pi2AvIM = pi2AvI;                                    // storeMomentaAverages (:238-256)
        pi2AvI = avPi2();
        pi2AvSI = 0.5 * (pi2AvI + pi2AvIM);
        aDotI += dt * sfKernelSI() * w;                      // kickScaleFactor (:160-163)
        aI += dt / 2.0 * aDotI * w;                          // driftScaleFactorSecondHalf (:225-234)
        aSI = (aIM + aI) / 2.0;
      }
      driftPV(dt / 2 * w);
      if (ex) {                                              // storeFieldsAveragesInt (:268-276)
        grad2AvI = avGrad2();
        potAvI = avPot();
      }
    }
  }

  // ---- LeapFrog::evolve (leapfrog.h:42-89)
  void evolveLF()
  {
    const double dt = cfg.dt;
    const bool ex = cfg.expansion != 0;
    const double weight = synced ? 0.5 : 1.0;
    if (fb) { // leapfrog.h:55-89 with driftScaleFactor's fixed branch (:168-175)
      kick(weight * dt);
      aIM = aI;
      aI = aBg(t - cfg.t0 + dt);
      aSI = aBg(t - cfg.t0 + dt / 2.0);
      drift(dt);
      synced = false;
      return;
    }
    kick(weight * dt);                                      // kickScalar (:131-134)
    if (ex) {
      pi2AvSIM = pi2AvSI;                                   // storeMomentaAverages (:239-245)
      pi2AvSI = avPi2();
      pi2AvI = 0.5 * (pi2AvSIM + pi2AvSI);
      aDotSIM = aDotSI;                                     // kickScaleFactor (:124-129)
      aDotSI += dt * sfKernel();
      aDotI = (aDotSIM + aDotSI) / 2.0;
      aIM = aI;                                             // driftScaleFactor (:168-184)
      aI += dt * aDotSI;
      aSI = (aIM + aI) / 2.0;
    }
    drift(dt);                                              // driftScalar (:185-190)
    if (ex) {                                               // storeFieldsAverages (:269-277)
      grad2AvI = avGrad2();
      potAvI = avPot();
    }
    synced = false;
  }

  // ---- LeapFrog::sync (leapfrog.h:96-116)
  void syncLF()
  {
    if (!synced && fb) {
      kick(0.5 * cfg.dt);
    } else if (!synced) {
      kick(0.5 * cfg.dt);
      if (cfg.expansion) {
        pi2AvI = avPi2();
        aDotI = aDotSI + cfg.dt / 2.0 * sfKernel();
      }
    }
    synced = true;
  }
};

thread_local std::string g_err;

// Every orc_handle is a Handle: the scalar oracle above or a gauge-sector oracle (oracle_models.h).
struct Handle {
  int kind;
  void *impl;
};
inline Handle *H(void *h) { return reinterpret_cast<Handle *>(h); }
inline bool isU1(void *h) { return H(h)->kind == CLB_MODEL_LPHI4U1; }
inline bool isSU2(void *h) { return H(h)->kind == CLB_MODEL_LPHI4SU2U1; }
inline Oracle *S(void *h) { return reinterpret_cast<Oracle *>(H(h)->impl); }

} // namespace

extern "C" {

typedef struct orc_handle orc_handle;

const char *orc_last_error(orc_handle *h)
{
  if (!h) return g_err.c_str();
  if (isSU2(h)) return oracle_models::su2_err(H(h)->impl).c_str();
  return isU1(h) ? oracle_models::u1_err(H(h)->impl).c_str() : S(h)->err.c_str();
}

int orc_create(const clb_config *cfg, const clb_model_desc *md, orc_handle **out)
{
  if (!cfg || !md || !out) { g_err = "null argument"; return CLB_EINVAL; }
  if (md->kind == CLB_MODEL_LPHI4SU2U1) {
    void *u = oracle_models::su2_create(cfg, md, g_err);
    if (!u) return CLB_EINVAL;
    *out = reinterpret_cast<orc_handle *>(new Handle{CLB_MODEL_LPHI4SU2U1, u});
    return CLB_OK;
  }
  if (md->kind == CLB_MODEL_LPHI4U1) {
    void *u = oracle_models::u1_create(cfg, md, g_err);
    if (!u) return CLB_EINVAL;
    *out = reinterpret_cast<orc_handle *>(new Handle{CLB_MODEL_LPHI4U1, u});
    return CLB_OK;
  }
  if (md->kind != CLB_MODEL_LPHI4 || md->n_scalars < 1 || md->n_scalars > 2) {
    g_err = "oracle: only lphi4 with 1 or 2 scalar singlets";
    return CLB_EUNSUPPORTED;
  }
  if (cfg->N < 2) { g_err = "N must be >= 2"; return CLB_EINVAL; }
  Oracle *o = new Oracle();
  o->cfg = *cfg;
  o->md = *md;
  o->N = cfg->N;
  o->n3 = (size_t)cfg->N * cfg->N * cfg->N;
  o->Ns = md->n_scalars;
  o->fld.assign((size_t)o->Ns * o->n3, 0.0);
  o->pi.assign((size_t)o->Ns * o->n3, 0.0);
  o->fb = cfg->expansion && cfg->fixed_background;
  if (o->fb) {
    o->pEoS = 2.0 / (3.0 * (1.0 + cfg->omega_eos) - 2.0 * md->alpha);
    o->H0fb = cfg->H0;
  }
  o->t = cfg->t0;
  if (cfg->evolver != CLB_LF) {
    o->ws = isPV(cfg->evolver) ? pvCoeffs(cfg->evolver) : vvCoeffs(cfg->evolver);
    if (o->ws.empty()) { delete o; g_err = "unsupported evolver"; return CLB_EUNSUPPORTED; }
  }
  *out = reinterpret_cast<orc_handle *>(new Handle{CLB_MODEL_LPHI4, o});
  return CLB_OK;
}

void orc_destroy(orc_handle *h)
{
  if (!h) return;
  if (isSU2(h))
    oracle_models::su2_destroy(H(h)->impl);
  else if (isU1(h))
    oracle_models::u1_destroy(H(h)->impl);
  else
    delete S(h);
  delete H(h);
}

// Selects the scalar-singlet potential restated above: 0 lphi4, 1 tanh2 (scalar-singlet handles).
int orc_set_scalar_model(orc_handle *h, int32_t id)
{
  if (!h || (id != 0 && id != 1)) return CLB_EINVAL;
  if (isU1(h) || isSU2(h)) return CLB_EUNSUPPORTED;
  S(h)->scalar_model = id;
  return CLB_OK;
}

// Gravitational waves of a scalar-singlet handle: enable (zero u and pi_u), set and get the five
// components of each (5 x N^3 doubles, the order of u_11, u_12, u_13, u_22, u_23).
int orc_gws_enable(orc_handle *h)
{
  if (!h) return CLB_EINVAL;
  if (isSU2(h)) return oracle_models::su2_gws_enable(H(h)->impl);
  if (isU1(h)) return oracle_models::u1_gws_enable(H(h)->impl);
  Oracle *o = S(h);
  o->gws = true;
  o->gwSynced = true;
  o->gu.assign(5 * o->n3, 0.0);
  o->gpi.assign(5 * o->n3, 0.0);
  return CLB_OK;
}
// the GW sector of a gauge handle (null for a scalar-singlet handle)
static oracle_models::GWs *gauge_gws(orc_handle *h)
{
  if (isSU2(h)) return oracle_models::su2_gws(H(h)->impl);
  if (isU1(h)) return oracle_models::u1_gws(H(h)->impl);
  return nullptr;
}

int orc_gws_set_state(orc_handle *h, const double *u, const double *pi)
{
  if (!h) return CLB_EINVAL;
  if (oracle_models::GWs *g = gauge_gws(h)) {
    if (!g->on) return CLB_ESTATE;
    if (u) std::memcpy(g->u.data(), u, g->u.size() * sizeof(double));
    if (pi) std::memcpy(g->pi.data(), pi, g->pi.size() * sizeof(double));
    return CLB_OK;
  }
  if (!S(h)->gws) return CLB_ESTATE;
  Oracle *o = S(h);
  if (u) std::memcpy(o->gu.data(), u, o->gu.size() * sizeof(double));
  if (pi) std::memcpy(o->gpi.data(), pi, o->gpi.size() * sizeof(double));
  return CLB_OK;
}
int orc_gws_get_state(orc_handle *h, double *u, double *pi)
{
  if (!h) return CLB_EINVAL;
  if (oracle_models::GWs *g = gauge_gws(h)) {
    if (!g->on) return CLB_ESTATE;
    if (u) std::memcpy(u, g->u.data(), g->u.size() * sizeof(double));
    if (pi) std::memcpy(pi, g->pi.data(), g->pi.size() * sizeof(double));
    return CLB_OK;
  }
  if (!S(h)->gws) return CLB_ESTATE;
  Oracle *o = S(h);
  if (u) std::memcpy(u, o->gu.data(), o->gu.size() * sizeof(double));
  if (pi) std::memcpy(pi, o->gpi.data(), o->gpi.size() * sizeof(double));
  return CLB_OK;
}

int orc_set_state(orc_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf)
{
  if (isSU2(h)) return oracle_models::su2_set_state(H(h)->impl, fields, momenta, sf);
  if (isU1(h)) return oracle_models::u1_set_state(H(h)->impl, fields, momenta, sf);
  Oracle *o = S(h);
  std::memcpy(o->fld.data(), fields, o->fld.size() * sizeof(double));
  std::memcpy(o->pi.data(), momenta, o->pi.size() * sizeof(double));
  if (sf) {
    o->aI = sf->aI; o->aSI = sf->aSI; o->aIM = sf->aIM;
    o->aDotI = sf->aDotI; o->aDotSI = sf->aDotSI; o->aDotSIM = sf->aDotSIM;
  }
  o->initialized = false;
  return CLB_OK;
}

int orc_get_state(orc_handle *h, double *fields, double *momenta, clb_scalefactor *sf)
{
  if (isSU2(h)) return oracle_models::su2_get_state(H(h)->impl, fields, momenta, sf);
  if (isU1(h)) return oracle_models::u1_get_state(H(h)->impl, fields, momenta, sf);
  Oracle *o = S(h);
  if (fields) std::memcpy(fields, o->fld.data(), o->fld.size() * sizeof(double));
  if (momenta) std::memcpy(momenta, o->pi.data(), o->pi.size() * sizeof(double));
  if (sf) {
    sf->aI = o->aI; sf->aSI = o->aSI; sf->aIM = o->aIM;
    sf->aDotI = o->aDotI; sf->aDotSI = o->aDotSI; sf->aDotSIM = o->aDotSIM;
  }
  return CLB_OK;
}

// ModelInitializer tail (modelinitializer.h:74-80) then the evolver constructor (leapfrog.h:35).
int orc_initialize(orc_handle *h, int32_t correct_adot)
{
  if (isSU2(h)) return oracle_models::su2_initialize(H(h)->impl, correct_adot);
  if (isU1(h)) return oracle_models::u1_initialize(H(h)->impl, correct_adot);
  Oracle *o = S(h);
  o->setAllAverages();
  if (o->cfg.expansion && correct_adot == 1 && !o->fb) { // modelinitializer.h:74-80
    double hl[3];
    o->hubble(hl);
    o->aDotI = std::sqrt(hl[2]);
  }
  o->synced = true;
  o->gwSynced = correct_adot != CLB_INIT_RESTART; // Evolver's GWsynced(!doWeRestart), evolver.h:52
  o->t = o->cfg.t0;
  if (o->cfg.evolver == CLB_LF && o->cfg.expansion) o->aDotSI = o->aDotI - o->cfg.dt / 2.0 * o->sfKernel();
  o->initialized = true;
  return CLB_OK;
}

int orc_evolve(orc_handle *h, int64_t n)
{
  if (isSU2(h)) return oracle_models::su2_evolve(H(h)->impl, n);
  if (isU1(h)) return oracle_models::u1_evolve(H(h)->impl, n);
  Oracle *o = S(h);
  if (!o->initialized) { o->err = "evolve before initialize"; return CLB_ESTATE; }
  for (int64_t s = 0; s < n; ++s) {
    if (o->gws) { // evolver.h:104-107
      o->gwKick(o->gwSynced ? 0.5 : 1.0);
      o->gwSynced = false;
    }
    if (o->cfg.evolver == CLB_LF)
      o->evolveLF();
    else if (isPV(o->cfg.evolver))
      o->evolvePV();
    else
      o->evolveVV();
    if (o->gws) o->gwDrift(); // evolver.h:123
    o->t += o->cfg.dt; // the main loop's t (cosmolattice.cpp:186-188)
  }
  return CLB_OK;
}

int orc_sync(orc_handle *h)
{
  if (isSU2(h)) return oracle_models::su2_sync(H(h)->impl);
  if (isU1(h)) return oracle_models::u1_sync(H(h)->impl);
  Oracle *o = S(h);
  if (o->gws && !o->gwSynced) { // evolver.h:134-137
    o->gwKick(0.5);
    o->gwSynced = true;
  }
  if (o->cfg.evolver == CLB_LF) o->syncLF();
  if (o->fb) o->aDotI = o->aBgDot(o->t - o->cfg.t0); // velocityverlet.h:121, leapfrog.h:114, positionverlet.h:106
  return CLB_OK;
}

// Measurer::measure frequent output: EnergiesMeasurer (energiesmeasurer.h:45-122), MeansMeasurer
// (meansmeasurer.h:28-48), ScaleFactorMeasurer (scalefactormeasurer.h:37-48).
int orc_measure(orc_handle *h, double e0, clb_measurement *m)
{
  if (isSU2(h)) return oracle_models::su2_measure(H(h)->impl, e0, m);
  if (isU1(h)) return oracle_models::u1_measure(H(h)->impl, e0, m);
  Oracle *o = S(h);
  std::memset(m, 0, sizeof(*m));
  if (!o->cfg.expansion) o->potAvI = o->avPot();               // measurer.h:274-276
  const double am6 = ipow(o->aI, -6), am2 = ipow(o->aI, -2);
  double Etot = 0;
  int k = 0;
  for (int f = 0; f < o->Ns; ++f) {
    const double *pf = o->P(f);
    const double *ff = o->F(f);
    const double Ekin = o->average([&](int x, int y, int z) {
      const double p = pf[o->at(x, y, z)];
      return (0.5 * (p * p)) * am6;
    });
    const double Egrad = o->average([&](int x, int y, int z) { return (0.5 * o->grad2(ff, x, y, z)) * am2; });
    Etot += Ekin + Egrad;
    m->energies[k++] = Ekin;
    m->energies[k++] = Egrad;
  }
  const int nPot = o->Ns > 1 ? 2 : 1;
  for (int t = 0; t < nPot; ++t) {
    const double v = o->average([&](int x, int y, int z) { return o->potTerm(t, o->at(x, y, z)); });
    m->energies[k++] = v;
    Etot += v;
  }
  m->energies[k++] = Etot;
  m->n_energies = k;
  if (o->cfg.expansion) {
    o->hubble(m->friedmann);
  } else {
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  }
  const double am = std::pow(o->aI, o->md.alpha - 3);
  for (int f = 0; f < o->Ns; ++f) {
    const double *pf = o->P(f);
    const double *ff = o->F(f);
    const double phi = o->average([&](int x, int y, int z) { return ff[o->at(x, y, z)]; });
    const double phi2 = o->average([&](int x, int y, int z) { const double v = ff[o->at(x, y, z)]; return v * v; });
    const double mom = o->average([&](int x, int y, int z) { return pf[o->at(x, y, z)] * am; });
    const double mom2 = o->average([&](int x, int y, int z) { const double v = pf[o->at(x, y, z)] * am; return v * v; });
    const double r1 = phi2 - phi * phi, r2 = mom2 - mom * mom;
    m->means[f][0] = phi;
    m->means[f][1] = mom;
    m->means[f][2] = phi2;
    m->means[f][3] = mom2;
    m->means[f][4] = r1 > 0 ? std::sqrt(r1) : 0;
    m->means[f][5] = r2 > 0 ? std::sqrt(r2) : 0;
  }
  m->n_means = o->Ns;
  m->aI = o->aI;
  m->aDotI = o->aDotI;
  m->hubble = o->aDotI / o->aI;
  return CLB_OK;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

} // extern "C"
