// oracle_u1.cpp - FP64 CPU restatement of the complex scalar + U(1) gauge sector (lphi4U1).
//
// TEST INFRASTRUCTURE ONLY (see oracle.cpp).  Restates, in the reference's operation order:
//   evolvers/velocityverlet.h:51-266 and evolvers/leapfrog.h:29-277 (the CS / U1 kicks and drifts),
//   evolvers/kernels/complexscalarkernels.h:28-35, evolvers/kernels/u1kernels.h:31-52,
//   evolvers/kernels/scalefactorkernels.h:27-80, definitions/gaugederivatives.h:36-102,
//   definitions/mattercurrents.h:27-76, definitions/fieldfunctionals.h:80-153,
//   definitions/energies.h:47-97, 217-239, definitions/gausslaws.h:34-53, definitions/potential.h:30-79,
//   measurements/energiesmeasurer.h:45-122, measurements/complexscalarmeasurer.h:61-72,
//   measurements/u1measurer.h:78-87 and models/lphi4U1.h:117-140.
// TempLat operators without an in-tree definition are restated by a stated choice (parity
// unpinned against TempLat): complexPhase(t) = cos t + i sin t; forwDiff(f, i) = (f(x+i) - f(x))/dx;
// backDiff(f, j) = (f(x) - f(x-j))/dx; fieldStrength(A, i, j) = forwDiff(A_j, i) - forwDiff(A_i, j);
// magneticField(A)_1 = forwDiff(A_2, 3) - forwDiff(A_3, 2) and cyclic (u1measurer.h:98-100).
// Components: 0 Re phi, 1 Im phi, 2..4 A_1..A_3 (directions x, y, z).

#include "../include/clb200.h"
#include "oracle_models.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

inline double ipow(double x, int n)
{
  if (n == 0) return 1.0;
  if (n < 0) return 1.0 / ipow(x, -n);
  double r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return r;
}

struct U1Oracle {
  clb_config cfg;
  clb_model_desc md;
  int N;
  size_t n3;
  std::vector<double> F, P; // 5 components each
  double aI = 1, aSI = 1, aIM = 1, aDotI = 0, aDotSI = 0, aDotSIM = 0;
  double csPi2I = 0, csPi2SI = 0, csPi2SIM = 0, csGrad2I = 0;
  double u1Pi2I = 0, u1Pi2SI = 0, u1Pi2SIM = 0, u1Mag2I = 0;
  double csPi2IM = 0, u1Pi2IM = 0, csGrad2SI = 0, u1Mag2SI = 0; // position Verlet (positionverlet.h:238-276)
  // fixed background (fixedbackgroundexpansion.h:21-45): pEoS, H0, the main loop's time t
  bool fb = false;
  double pEoS = 0, H0fb = 0, t = 0;
  double aBg(double d) const { return std::pow(1 + H0fb / pEoS * d, pEoS); }
  double aBgDot(double d) const { return H0fb * std::pow(1 + H0fb / pEoS * d, pEoS - 1); }

  double potI = 0, potSI = 0;
  bool synced = true, initialized = false;
  oracle_models::GWs gw; // the GW sector (PITensor.h source: phi and A)
  std::vector<double> ws;
  std::string err;

  double *f(int c) { return F.data() + (size_t)c * n3; }
  double *p(int c) { return P.data() + (size_t)c * n3; }
  const double *f(int c) const { return F.data() + (size_t)c * n3; }
  double c4() const { return md.couplings[0]; }
  double gQ() const { return md.couplings[1]; }
  double rfo2() const { const double r = md.fStar / md.omegaStar; return r * r; } // pow<2>(fStar / omegaStar)
  double rof2() const { const double r = md.omegaStar / md.fStar; return r * r; } // pow<2>(omegaStar / fStar)

  size_t at(int x, int y, int z) const { return ((size_t)x * N + y) * N + z; }
  int wrap(int i) const { return i < 0 ? i + N : (i >= N ? i - N : i); }
  // site (x,y,z) shifted by s1 along d1 and s2 along d2
  size_t nb(int x, int y, int z, int d1, int s1, int d2 = 0, int s2 = 0) const
  {
    int c[3] = {x, y, z};
    c[d1] += s1;
    c[d2] += s2;
    return at(wrap(c[0]), wrap(c[1]), wrap(c[2]));
  }

  // U_d(s) = complexPhase(-dx gQ A_d(s))  (gaugederivatives.h:96-101)
  void link(size_t s, int d, double &ur, double &ui) const
  {
    const double th = (-cfg.dx * gQ()) * f(2 + d)[s];
    ur = std::cos(th);
    ui = std::sin(th);
  }
  double norm(size_t s) const
  {
    const double a = f(0)[s], b = f(1)[s];
    return std::sqrt(a * a + b * b);
  }
  double pot(size_t s) const { return c4() * ipow(norm(s), 4); } // lphi4U1.h:117-120
  double fd(int comp, size_t s, size_t sp) const { return (f(comp)[sp] - f(comp)[s]) / cfg.dx; }

  // covariant Laplacian of phi (gaugederivatives.h:48-53), component c
  void covLap(int x, int y, int z, double out[2]) const
  {
    const size_t s = at(x, y, z);
    double pr = 0, pim = 0, mr = 0, mim = 0;
    for (int d = 0; d < 3; ++d) {
      const size_t sp = nb(x, y, z, d, +1), sm = nb(x, y, z, d, -1);
      double ur, ui;
      link(s, d, ur, ui);
      const double wr = ur * f(0)[sp] - ui * f(1)[sp], wi = ur * f(1)[sp] + ui * f(0)[sp];
      double vr, vi;
      link(sm, d, vr, vi);
      const double cr = vr * f(0)[sm] - (-vi) * f(1)[sm], ci = vr * f(1)[sm] + (-vi) * f(0)[sm];
      if (d == 0) {
        pr = wr;
        pim = wi;
        mr = cr;
        mim = ci;
      } else {
        pr = pr + wr;
        pim = pim + wi;
        mr = mr + cr;
        mim = mim + ci;
      }
    }
    const double dx2 = cfg.dx * cfg.dx;
    out[0] = ((pr + mr) - 6 * f(0)[s]) / dx2;
    out[1] = ((pim + mim) - 6 * f(1)[s]) / dx2;
  }

  // ComplexScalarKernels::get (complexscalarkernels.h:28-35)
  void csKernel(int x, int y, int z, double K[2]) const
  {
    const size_t s = at(x, y, z);
    double cl[2];
    covLap(x, y, z, cl);
    const double A = std::pow(aI, 1 + md.alpha), B2 = std::pow(aI, 3 + md.alpha) / 2;
    const double n = norm(s);
    const double nd = c4() * (4 * ipow(n, 3)); // potDerivNormCS (lphi4U1.h:126-129)
    for (int c = 0; c < 2; ++c) {
      const double dV = nd / n * f(c)[s]; // derivComponentFromNorm (potential.h:30-34)
      K[c] = A * cl[c] - B2 * dV;
    }
  }

  // lattice Laplacian of component comp (gaugederivatives.h:36-40)
  double lapl(int comp, int x, int y, int z) const
  {
    const double *a = f(comp);
    const double c = a[at(x, y, z)];
    double t[3];
    for (int d = 0; d < 3; ++d) t[d] = (a[nb(x, y, z, d, +1)] + a[nb(x, y, z, d, -1)]) - 2 * c;
    return (1.0 / (cfg.dx * cfg.dx)) * ((t[0] + t[1]) + t[2]);
  }

  // U1Kernels::get (u1kernels.h:31-52), direction i, with MatterCurrents::U1Current (mattercurrents.h:52-76)
  double u1Kernel(int i, int x, int y, int z) const
  {
    const size_t s = at(x, y, z);
    const double lap = lapl(2 + i, x, y, z);
    double grad = 0;
    for (int j = 0; j < 3; ++j) {
      const size_t sj = nb(x, y, z, j, -1);                 // x - j
      const double g0 = fd(2 + j, s, nb(x, y, z, i, +1));    // forwDiff(A_j, i) at x
      const double g1 = fd(2 + j, sj, nb(x, y, z, i, +1, j, -1)); // ... at x - j
      const double t = (g0 - g1) / cfg.dx;                   // backDiff along j
      grad = j == 0 ? t : grad + t;
    }
    double ur, ui;
    link(s, i, ur, ui);
    const size_t sp = nb(x, y, z, i, +1);
    const double wr = ur * f(0)[sp] - ui * f(1)[sp], wi = ur * f(1)[sp] + ui * f(0)[sp];
    const double im = wr * f(1)[s] - wi * f(0)[s]; // Im(conj(w) phi)
    const double J = 2.0 / cfg.dx * rfo2() * (gQ() * im);
    const double normGrad = std::pow(aI, -1 + md.alpha), normSrc = std::pow(aI, 1 + md.alpha);
    return normGrad * (lap - grad) - normSrc * J;
  }

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

  double avCsPi2()
  {
    return average([&](int x, int y, int z) {
      const size_t s = at(x, y, z);
      return p(0)[s] * p(0)[s] + p(1)[s] * p(1)[s];
    });
  }
  double avU1Pi2()
  {
    return average([&](int x, int y, int z) {
      const size_t s = at(x, y, z);
      return (p(2)[s] * p(2)[s] + p(3)[s] * p(3)[s]) + p(4)[s] * p(4)[s];
    });
  }
  double csGrad2(int x, int y, int z) const // sum_j |D^+_j phi|^2 (fieldfunctionals.h:80-84)
  {
    const size_t s = at(x, y, z);
    double acc = 0;
    for (int j = 0; j < 3; ++j) {
      double ur, ui;
      link(s, j, ur, ui);
      const size_t sp = nb(x, y, z, j, +1);
      const double wr = ur * f(0)[sp] - ui * f(1)[sp], wi = ur * f(1)[sp] + ui * f(0)[sp];
      const double dr = (wr - f(0)[s]) / cfg.dx, di = (wi - f(1)[s]) / cfg.dx;
      const double n2 = dr * dr + di * di;
      acc = j == 0 ? n2 : acc + n2;
    }
    return acc;
  }
  double Fij(int i, int j, int x, int y, int z) const
  {
    const size_t s = at(x, y, z);
    return fd(2 + j, s, nb(x, y, z, i, +1)) - fd(2 + i, s, nb(x, y, z, j, +1));
  }
  double u1B2(int x, int y, int z) const // fieldfunctionals.h:133-141
  {
    const double f21 = Fij(1, 0, x, y, z), f31 = Fij(2, 0, x, y, z), f32 = Fij(2, 1, x, y, z);
    return f21 * f21 + (f31 * f31 + f32 * f32);
  }
  // PITensor.h's anisotropic tensor of lphi4U1 at (x, y, z): the complex scalar and the U(1) field
  void gwTensor(int x, int y, int z, double (&T)[6]) const
  {
    const size_t nbp[3] = {nb(x, y, z, 0, +1), nb(x, y, z, 1, +1), nb(x, y, z, 2, +1)};
    const double *const A[3] = {f(2), f(3), f(4)};
    const double *const pA[3] = {P.data() + 2 * n3, P.data() + 3 * n3, P.data() + 4 * n3};
    oracle_models::gw_gauge_tensor(f(0), f(1), A, pA, nbp, at(x, y, z), cfg.dx, gQ(), aI, rfo2(), true, T);
  }
  void gwKick(double w)
  {
    gw.kick(N, cfg.dx, aI, md.alpha, w * cfg.dt, [&](int x, int y, int z, double (&T)[6]) { gwTensor(x, y, z, T); });
  }

  double avCsGrad2() { return average([&](int x, int y, int z) { return csGrad2(x, y, z); }); }
  double avU1B2() { return average([&](int x, int y, int z) { return u1B2(x, y, z); }); }
  double avPot() { return average([&](int x, int y, int z) { return pot(at(x, y, z)); }); }

  // energies.h:47-97
  double kineticCS(double v) const { return v * ipow(aI, -6); }
  double gradientCS(double v) const { return v * ipow(aI, -2); }
  double electricU1(double v) const { return 0.5 * rof2() * ipow(aI, -4) * v * 1.0; }
  double magneticU1(double v) const { return 0.5 * rof2() * ipow(aI, -4) * v / 1.0; }

  double sfKernel() const // scalefactorkernels.h:73-77
  {
    const double al = md.alpha;
    const double Ekcs = kineticCS(csPi2I), Egcs = gradientCS(csGrad2I);
    const double Eel = electricU1(u1Pi2I), Emag = magneticU1(u1Mag2I);
    const double fm = md.fStar / md.MPl;
    return std::pow(aI, 2 * al + 1) / 3.0 * (fm * fm) *
           ((((al - 2) * Ekcs + al * Egcs) + (al - 1) * (1.0 * (Eel + Emag))) + (al + 1) * potI);
  }

  double sfKernelSI() const // ScaleFactorKernels::getSI (scalefactorkernels.h:83-119)
  {
    const double al = md.alpha;
    const double Ekcs = kineticCS(csPi2SI), Egcs = gradientCS(csGrad2SI);
    const double Eel = electricU1(u1Pi2SI), Emag = magneticU1(u1Mag2SI);
    const double fm = md.fStar / md.MPl;
    return std::pow(aI, 2 * al + 1) / 3.0 * (fm * fm) *
           ((((al - 2) * Ekcs + al * Egcs) + (al - 1) * (Eel + Emag)) + (al + 1) * potSI);
  }

  void setAllAverages() // averages.h:349-378
  {
    potI = avPot();
    potSI = potI;
    u1Pi2I = avU1Pi2();
    u1Pi2SI = u1Pi2I;
    u1Mag2I = avU1B2();
    csPi2I = avCsPi2();
    csPi2SI = csPi2I;
    csGrad2I = avCsGrad2();
  }

  void hubble(double out[3]) // hubbleconstraint.h:27-36 with energies.h:217-239
  {
    setAllAverages();
    const double rho = (((kineticCS(csPi2I) + gradientCS(csGrad2I)) + electricU1(u1Pi2I)) + magneticU1(u1Mag2I)) + potI;
    const double LHS = aDotI * aDotI;
    const double fm = md.fStar / md.MPl;
    const double RHS = std::pow(aI, 2 * md.alpha + 2) / 3. * (fm * fm) * rho;
    out[0] = (LHS - RHS) / (LHS + RHS);
    out[1] = LHS;
    out[2] = RHS;
  }

  // kicks with weight factors: CS gets hc K, U(1) gets hu K (the reference rounds them differently)
  void kick(double hc, double hu)
  {
    std::vector<double> K((size_t)5 * n3);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < N; ++x)
      for (int y = 0; y < N; ++y)
        for (int z = 0; z < N; ++z) {
          const size_t s = at(x, y, z);
          double kc[2];
          csKernel(x, y, z, kc);
          K[s] = kc[0];
          K[n3 + s] = kc[1];
          for (int i = 0; i < 3; ++i) K[(2 + i) * n3 + s] = u1Kernel(i, x, y, z);
        }
    for (size_t s = 0; s < n3; ++s) {
      p(0)[s] = p(0)[s] + hc * K[s];
      p(1)[s] = p(1)[s] + hc * K[n3 + s];
      for (int i = 0; i < 3; ++i) p(2 + i)[s] = p(2 + i)[s] + hu * K[(2 + i) * n3 + s];
    }
  }
  // drifts: phi += cc pi (cc = (pow(aSI,alpha-3) dt) w), A += (cu pi) 1 (cu = (pow(aSI,alpha-1) w) dt)
  void drift(double cc, double cu)
  {
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < n3; ++s) {
      for (int c = 0; c < 2; ++c) f(c)[s] = f(c)[s] + cc * p(c)[s];
      for (int i = 0; i < 3; ++i) f(2 + i)[s] = f(2 + i)[s] + cu * p(2 + i)[s] * 1.0;
    }
  }

  void evolveVV()
  {
    const double dt = cfg.dt;
    const size_t Pn = ws.size(), stages = (Pn - 1) * 2 + 1;
    const bool ex = cfg.expansion != 0;
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < Pn ? i : stages - i - 1];
      if (ex) aDotSI = aDotI + (dt / 2) * sfKernel() * w;
      kick(dt / 2 * w, dt * w / 2); // velocityverlet.h:140-157
      if (ex) {
        csPi2I = avCsPi2();
        u1Pi2I = avU1Pi2();
        aIM = aI;
        aI += dt * aDotSI * w;
        aSI = (aIM + aI) / 2.0;
      }
      drift(std::pow(aSI, md.alpha - 3) * dt * w, std::pow(aSI, md.alpha - 1) * w * dt); // :193-210
      if (ex) {
        csGrad2I = avCsGrad2();
        u1Mag2I = avU1B2();
        potI = avPot();
      }
      kick(dt / 2 * w, dt * w / 2);
      if (ex) {
        csPi2I = avCsPi2();
        u1Pi2I = avU1Pi2();
        aDotI = aDotSI + (dt / 2) * sfKernel() * w;
      }
    }
  }

  // PositionVerlet::evolve (positionverlet.h:45-99): driftCS / driftU1Vector (:182-185, :194-197),
  // kickCS / kickU1Vector (:138-157), the scale factor (:160-163, :207-235), averages (:238-276)
  void evolvePV()
  {
    const double dt = cfg.dt;
    const size_t Pn = ws.size(), stages = (Pn - 1) * 2 + 1;
    const bool ex = cfg.expansion != 0;
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < Pn ? i : stages - i - 1];
      drift(std::pow(aI, md.alpha - 3) * dt / 2 * w, std::pow(aI, md.alpha - 1) * w * dt / 2);
      if (ex) {
        aIM = aI;
        aI += dt / 2.0 * aDotI * w;
        aSI = aI;
        csGrad2SI = avCsGrad2();
        u1Mag2SI = avU1B2();
        potSI = avPot();
      }
      kick(dt * w, dt * w);
      if (ex) {
        csPi2IM = csPi2I;
        u1Pi2IM = u1Pi2I;
        csPi2I = avCsPi2();
        u1Pi2I = avU1Pi2();
        csPi2SI = 0.5 * (csPi2I + csPi2IM);
        u1Pi2SI = 0.5 * (u1Pi2I + u1Pi2IM);
        aDotI += dt * sfKernelSI() * w;
        aI += dt / 2.0 * aDotI * w;
        aSI = (aIM + aI) / 2.0;
      }
      drift(std::pow(aI, md.alpha - 3) * dt / 2 * w, std::pow(aI, md.alpha - 1) * w * dt / 2);
      if (ex) {
        csGrad2I = avCsGrad2();
        u1Mag2I = avU1B2();
        potI = avPot();
      }
    }
  }

  // fixed background: the VV (velocityverlet.h:74-118, 225-231; aSI is left as it was), the leapfrog
  // (leapfrog.h:55-89, 168-175) and position Verlet (positionverlet.h:45-99, 207-235) with a from
  // the closed form and no a-kicks or averages; one step from time t
  void evolveFB()
  {
    const double dt = cfg.dt, al = md.alpha;
    if (cfg.evolver == CLB_LF) {
      const double weight = synced ? 0.5 : 1.0;
      kick(weight * dt, weight * dt);
      aIM = aI;
      aI = aBg(t - cfg.t0 + dt);
      aSI = aBg(t - cfg.t0 + dt / 2.0);
      drift(std::pow(aSI, al - 3) * dt, std::pow(aSI, al - 1) * dt);
      synced = false;
      return;
    }
    const size_t Pn = ws.size(), stages = (Pn - 1) * 2 + 1;
    double tc = t - cfg.t0;
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < Pn ? i : stages - i - 1];
      if (cfg.evolver >= CLB_PV2) {
        drift(std::pow(aI, al - 3) * dt / 2 * w, std::pow(aI, al - 1) * w * dt / 2);
        aIM = aI;
        aI = aBg(tc + w * dt / 2.0);
        aSI = aI;
        kick(dt * w, dt * w);
        aI = aBg(tc + w * dt);
        drift(std::pow(aI, al - 3) * dt / 2 * w, std::pow(aI, al - 1) * w * dt / 2);
      } else {
        kick(dt / 2 * w, dt * w / 2);
        aIM = aI;
        aI = aBg(tc + w * dt);
        drift(std::pow(aSI, al - 3) * dt * w, std::pow(aSI, al - 1) * w * dt);
        kick(dt / 2 * w, dt * w / 2);
      }
      tc += dt * w;
    }
  }

  void evolveLF()
  {
    const double dt = cfg.dt;
    const bool ex = cfg.expansion != 0;
    const double weight = synced ? 0.5 : 1.0;
    kick(weight * dt, weight * dt); // leapfrog.h:141-155
    if (ex) {
      csPi2SIM = csPi2SI;
      csPi2SI = avCsPi2();
      csPi2I = 0.5 * (csPi2SIM + csPi2SI);
      u1Pi2SIM = u1Pi2SI;
      u1Pi2SI = avU1Pi2();
      u1Pi2I = 0.5 * (u1Pi2SIM + u1Pi2SI);
      aDotSIM = aDotSI;
      aDotSI += dt * sfKernel();
      aDotI = (aDotSIM + aDotSI) / 2.0;
      aIM = aI;
      aI += dt * aDotSI;
      aSI = (aIM + aI) / 2.0;
    }
    drift(std::pow(aSI, md.alpha - 3) * dt, std::pow(aSI, md.alpha - 1) * dt); // leapfrog.h:203-217
    if (ex) {
      csGrad2I = avCsGrad2();
      u1Mag2I = avU1B2();
      potI = avPot();
    }
    synced = false;
  }

  void syncLF()
  {
    if (!synced) {
      kick(0.5 * cfg.dt, 0.5 * cfg.dt);
      if (cfg.expansion) {
        csPi2I = avCsPi2();
        u1Pi2I = avU1Pi2();
        aDotI = aDotSI + cfg.dt / 2.0 * sfKernel();
      }
    }
    synced = true;
  }

  // GaussLaws::checkU1 (gausslaws.h:34-53)
  void gauss(double out[3]) const
  {
    const double dx = cfg.dx;
    const double nrm = 2 / dx * rfo2();
    auto per = [&](int x, int y, int z, int what) {
      const size_t s = at(x, y, z);
      double l[3];
      for (int i = 0; i < 3; ++i) l[i] = p(2 + i)[s] - p(2 + i)[nb(x, y, z, i, -1)];
      const double LHS = ((l[0] + l[1]) + l[2]) / dx;
      const double im = p(0)[s] * f(1)[s] - p(1)[s] * f(0)[s]; // Im(conj(pi) phi)
      const double rho = nrm * gQ() * im;
      const double RHS = -dx * rho;
      const double L1 = l[0] / dx, L2 = l[1] / dx, L3 = l[2] / dx;
      const double diff = LHS - (RHS + 0.0);
      const double sum = L1 * L1 + L2 * L2 + L3 * L3 + (RHS + 0.0) * (RHS + 0.0);
      switch (what) {
      case 0: return std::sqrt(diff * diff);
      case 1: return std::sqrt(sum * sum);
      case 2: return std::sqrt((RHS + 0.0) * (RHS + 0.0));
      default: return std::sqrt(LHS * LHS);
      }
    };
    auto *self = const_cast<U1Oracle *>(this);
    const double avDiff = self->average([&](int x, int y, int z) { return per(x, y, z, 0); });
    const double avSum = self->average([&](int x, int y, int z) { return per(x, y, z, 1); });
    const double avRHS = self->average([&](int x, int y, int z) { return per(x, y, z, 2); });
    const double avLHS = self->average([&](int x, int y, int z) { return per(x, y, z, 3); });
    out[0] = avDiff / avSum;
    out[1] = avLHS;
    out[2] = avRHS;
  }
  const double *p(int c) const { return P.data() + (size_t)c * n3; }
};

} // namespace

namespace oracle_models {

void *u1_create(const clb_config *cfg, const clb_model_desc *md, std::string &err)
{
  if (cfg->N < 2) {
    err = "N must be >= 2";
    return nullptr;
  }
  U1Oracle *o = new U1Oracle();
  o->cfg = *cfg;
  o->md = *md;
  o->N = cfg->N;
  o->n3 = (size_t)cfg->N * cfg->N * cfg->N;
  o->F.assign(5 * o->n3, 0.0);
  o->P.assign(5 * o->n3, 0.0);
  o->fb = cfg->expansion && cfg->fixed_background;
  if (o->fb) {
    o->pEoS = 2.0 / (3.0 * (1.0 + cfg->omega_eos) - 2.0 * md->alpha);
    o->H0fb = cfg->H0;
  }
  o->t = cfg->t0;
  if (cfg->evolver != CLB_LF) {
    o->ws = oracle_vv_weights(cfg->evolver >= CLB_PV2 ? cfg->evolver - CLB_PV2 + CLB_VV2 : cfg->evolver);
    if (o->ws.empty()) {
      delete o;
      err = "unsupported evolver";
      return nullptr;
    }
  }
  return o;
}

void u1_destroy(void *h) { delete static_cast<U1Oracle *>(h); }
std::string &u1_err(void *h) { return static_cast<U1Oracle *>(h)->err; }

int u1_set_state(void *h, const double *fields, const double *momenta, const clb_scalefactor *sf)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  std::memcpy(o->F.data(), fields, o->F.size() * sizeof(double));
  std::memcpy(o->P.data(), momenta, o->P.size() * sizeof(double));
  if (sf) {
    o->aI = sf->aI;
    o->aSI = sf->aSI;
    o->aIM = sf->aIM;
    o->aDotI = sf->aDotI;
    o->aDotSI = sf->aDotSI;
    o->aDotSIM = sf->aDotSIM;
  }
  o->initialized = false;
  return CLB_OK;
}

int u1_get_state(void *h, double *fields, double *momenta, clb_scalefactor *sf)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  if (fields) std::memcpy(fields, o->F.data(), o->F.size() * sizeof(double));
  if (momenta) std::memcpy(momenta, o->P.data(), o->P.size() * sizeof(double));
  if (sf) {
    sf->aI = o->aI;
    sf->aSI = o->aSI;
    sf->aIM = o->aIM;
    sf->aDotI = o->aDotI;
    sf->aDotSI = o->aDotSI;
    sf->aDotSIM = o->aDotSIM;
  }
  return CLB_OK;
}

int u1_initialize(void *h, int32_t correct_adot)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  o->setAllAverages();
  o->t = o->cfg.t0;
  if (o->cfg.expansion && correct_adot == 1 && !o->fb) {
    double hl[3];
    o->hubble(hl);
    o->aDotI = std::sqrt(hl[2]);
  }
  o->synced = true;
  o->gw.synced = correct_adot != CLB_INIT_RESTART; // evolver.h:52
  if (o->cfg.evolver == CLB_LF && o->cfg.expansion) o->aDotSI = o->aDotI - o->cfg.dt / 2.0 * o->sfKernel();
  o->initialized = true;
  return CLB_OK;
}

int u1_gws_enable(void *h)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  o->gw.enable(o->n3);
  return CLB_OK;
}
GWs *u1_gws(void *h) { return &static_cast<U1Oracle *>(h)->gw; }

int u1_evolve(void *h, int64_t n)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  if (!o->initialized) {
    o->err = "evolve before initialize";
    return CLB_ESTATE;
  }
  for (int64_t s = 0; s < n; ++s) {
    if (o->gw.on) { // evolver.h:104-107
      o->gwKick(o->gw.synced ? 0.5 : 1.0);
      o->gw.synced = false;
    }
    if (o->fb)
      o->evolveFB();
    else if (o->cfg.evolver == CLB_LF)
      o->evolveLF();
    else if (o->cfg.evolver >= CLB_PV2)
      o->evolvePV();
    else
      o->evolveVV();
    if (o->gw.on) o->gw.drift(std::pow(o->aSI, o->md.alpha - 3), o->cfg.dt); // evolver.h:123
    o->t += o->cfg.dt;
  }
  return CLB_OK;
}

int u1_sync(void *h)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  if (o->gw.on && !o->gw.synced) { // evolver.h:134-137
    o->gwKick(0.5);
    o->gw.synced = true;
  }
  if (o->fb) {
    if (o->cfg.evolver == CLB_LF && !o->synced) o->kick(0.5 * o->cfg.dt, 0.5 * o->cfg.dt);
    o->synced = true;
    o->aDotI = o->aBgDot(o->t - o->cfg.t0);
    return CLB_OK;
  }
  if (o->cfg.evolver == CLB_LF) o->syncLF();
  return CLB_OK;
}

int u1_measure(void *h, double e0, clb_measurement *m)
{
  U1Oracle *o = static_cast<U1Oracle *>(h);
  std::memset(m, 0, sizeof(*m));
  if (!o->cfg.expansion) o->potI = o->avPot(); // measurer.h:274-276
  const double am6 = ipow(o->aI, -6), am2 = ipow(o->aI, -2), ae = 0.5 * o->rof2() * ipow(o->aI, -4);
  const double Ekcs = o->average([&](int x, int y, int z) {
    const size_t s = o->at(x, y, z);
    return (o->p(0)[s] * o->p(0)[s] + o->p(1)[s] * o->p(1)[s]) * am6;
  });
  const double Egcs = o->average([&](int x, int y, int z) { return o->csGrad2(x, y, z) * am2; });
  const double Eel = o->average([&](int x, int y, int z) {
    const size_t s = o->at(x, y, z);
    return ae * ((o->p(2)[s] * o->p(2)[s] + o->p(3)[s] * o->p(3)[s]) + o->p(4)[s] * o->p(4)[s]) * 1.0;
  });
  const double Emag = o->average([&](int x, int y, int z) { return ae * o->u1B2(x, y, z) / 1.0; });
  const double V = o->average([&](int x, int y, int z) { return o->pot(o->at(x, y, z)); });
  double Etot = 0;
  Etot += Ekcs + Egcs;
  Etot += Eel + Emag;
  Etot += V;
  const double en[6] = {Ekcs, Egcs, Eel, Emag, V, Etot};
  for (int k = 0; k < 6; ++k) m->energies[k] = en[k];
  m->n_energies = 6;
  if (o->cfg.expansion)
    o->hubble(m->friedmann);
  else
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  // means (meansmeasurer.h:28-48) of sqrt2 Re, sqrt2 Im, |phi| and |E|, |B|
  const double am = std::pow(o->aI, o->md.alpha - 3), ag = std::pow(o->aI, o->md.alpha - 1);
  const double sq2 = std::sqrt(2.0);
  // fv, pv: per-site values for the first and second column pairs, as functions of (x, y, z)
  auto fill = [&](int row, auto fv, auto pv) {
    const double a1 = o->average(fv);
    const double a2 = o->average([&](int x, int y, int z) { const double v = fv(x, y, z); return v * v; });
    const double b1 = o->average(pv);
    const double b2 = o->average([&](int x, int y, int z) { const double v = pv(x, y, z); return v * v; });
    const double r1 = a2 - a1 * a1, r2 = b2 - b1 * b1;
    m->means[row][0] = a1;
    m->means[row][1] = b1;
    m->means[row][2] = a2;
    m->means[row][3] = b2;
    m->means[row][4] = r1 > 0 ? std::sqrt(r1) : 0;
    m->means[row][5] = r2 > 0 ? std::sqrt(r2) : 0;
  };
  auto S = [&](int x, int y, int z) { return o->at(x, y, z); };
  fill(0, [&](int x, int y, int z) { return sq2 * o->f(0)[S(x, y, z)]; },
       [&](int x, int y, int z) { return sq2 * o->p(0)[S(x, y, z)] * am; });
  fill(1, [&](int x, int y, int z) { return sq2 * o->f(1)[S(x, y, z)]; },
       [&](int x, int y, int z) { return sq2 * o->p(1)[S(x, y, z)] * am; });
  fill(2, [&](int x, int y, int z) { return o->norm(S(x, y, z)); },
       [&](int x, int y, int z) {
         const size_t s = S(x, y, z);
         const double a = o->p(0)[s] * am, b = o->p(1)[s] * am;
         return std::sqrt(a * a + b * b);
       });
  // gauge row: |E| = |pi_A a^(alpha-1)| and |B| with B_1 = forwDiff(A_2, 3) - forwDiff(A_3, 2) and cyclic
  fill(3,
       [&](int x, int y, int z) {
         const size_t s = S(x, y, z);
         const double e1 = o->p(2)[s] * ag, e2 = o->p(3)[s] * ag, e3 = o->p(4)[s] * ag;
         return std::sqrt(e1 * e1 + e2 * e2 + e3 * e3);
       },
       [&](int x, int y, int z) {
         const double b1 = o->Fij(2, 1, x, y, z), b2 = o->Fij(0, 2, x, y, z), b3 = o->Fij(1, 0, x, y, z);
         return std::sqrt(b1 * b1 + b2 * b2 + b3 * b3);
       });
  m->n_means = 4;
  o->gauss(m->gauss_u1);
  m->aI = o->aI;
  m->aDotI = o->aDotI;
  m->hubble = o->aDotI / o->aI;
  return CLB_OK;
}

} // namespace oracle_models
