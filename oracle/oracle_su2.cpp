// oracle_su2.cpp - FP64 CPU restatement of lphi4SU2U1: a real scalar S, a complex scalar phi
// (U(1) charged), an SU(2) doublet Phi (U(1) and SU(2) charged), one U(1) and one SU(2) field.
//
// TEST INFRASTRUCTURE ONLY (see oracle.cpp).  Restates models/lphi4SU2U1.h:117-212 with
//   evolvers/velocityverlet.h:51-266 and leapfrog.h:29-277 (kicks, drifts, SU(2) link drift
//   U <- exp(w a^(alpha-1) dx dt g pi) U at :212-222), evolvers/kernels/su2kernels.h:30-54,
//   su2doubletkernels.h:28-33, complexscalarkernels.h:28-35, u1kernels.h:31-52,
//   scalarsingletkernels.h:30-40, definitions/gaugederivatives.h:48-102, mattercurrents.h:27-119,
//   fieldfunctionals.h:52-223, gausslaws.h:34-80, energies.h:37-239, scalefactorkernels.h:27-80.
//
// TempLat's SU(2) types are not in the reference tree; the stated choices (parity unpinned):
//   * a link is a unit quaternion (q0, q) meaning q0 + i q.sigma; products and daggers follow;
//   * an algebra element (pi_1, pi_2, pi_3) means i pi_a sigma_a; exp(i p.sigma) = cos|p| + i sin|p| p/|p|;
//     the algebra part of a quaternion is its vector part;
//   * plaq(U, i, j) = U_i(x) U_j(x+i) U_i(x+j)^+ U_j(x)^+, and plaqBack(U, i, j) is the dagger of the
//     backward plaquette U_i(x) U_j(x+i-j)^+ U_i(x-j)^+ U_j(x-j), so that sum_j (plaq - plaqBack)
//     is the force of the Wilson term 4/(dx^4 g^2) sum (2 - tr P) (fieldfunctionals.h:201-209);
//   * a doublet is (Phi_0 + i Phi_1, Phi_2 + i Phi_3); scalar_prod(A, B) = A^+ B.
// With these the reference's normalisations (su2kernels.h:44-49, mattercurrents.h:86-119,
// fieldfunctionals.h:218-223) make the evolution conserve energy and both Gauss laws (tests).
//
// Field components: 0 S | 1,2 phi | 3..6 Phi | 7..9 A_x..A_z | 10 + 4 i + (0..3) link U_i.
// Momentum components: 0 | 1,2 | 3..6 | 7..9 | 10 + 3 i + (0..2) pi_SU2 of direction i.
// Couplings: [0] qG, [1] qH, [2] g_U1 Q_phi, [3] g_U1 Q_Phi, [4] g_SU2 Q_Phi, [5] c4 (|Phi|^4 coefficient).

#include "../include/clb200.h"
#include "oracle_models.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

namespace {

using cd = std::complex<double>;

inline double ipow(double x, int n)
{
  if (n == 0) return 1.0;
  if (n < 0) return 1.0 / ipow(x, -n);
  double r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return r;
}

struct Qt {
  double w, x, y, z;
};
inline Qt qmul(const Qt &a, const Qt &b)
{
  // (a0 + i a.s)(b0 + i b.s) = a0 b0 - a.b + i (a0 b + b0 a - a x b).s
  return Qt{a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z), a.w * b.x + b.w * a.x - (a.y * b.z - a.z * b.y),
            a.w * b.y + b.w * a.y - (a.z * b.x - a.x * b.z), a.w * b.z + b.w * a.z - (a.x * b.y - a.y * b.x)};
}
inline Qt qdag(const Qt &a) { return Qt{a.w, -a.x, -a.y, -a.z}; }
inline Qt qexp(double p1, double p2, double p3)
{
  const double n = std::sqrt(p1 * p1 + p2 * p2 + p3 * p3);
  if (n == 0) return Qt{1, 0, 0, 0};
  const double s = std::sin(n) / n;
  return Qt{std::cos(n), s * p1, s * p2, s * p3};
}
struct Dbl {
  cd u, v;
};
// U (u, v) with U = [[q0 + i q3, q2 + i q1], [-q2 + i q1, q0 - i q3]]
inline Dbl qapply(const Qt &q, const Dbl &d)
{
  return Dbl{cd(q.w, q.z) * d.u + cd(q.y, q.x) * d.v, cd(-q.y, q.x) * d.u + cd(q.w, -q.z) * d.v};
}
inline Dbl dscale(const cd &c, const Dbl &d) { return Dbl{c * d.u, c * d.v}; }
inline cd sprod(const Dbl &a, const Dbl &b) { return std::conj(a.u) * b.u + std::conj(a.v) * b.v; }
// i sigma_b applied to a doublet
inline Dbl isig(int b, const Dbl &d)
{
  const cd I(0, 1);
  if (b == 0) return Dbl{I * d.v, I * d.u};
  if (b == 1) return Dbl{d.v, -d.u};
  return Dbl{I * d.u, -I * d.v};
}

constexpr int NF = 22, NP = 19;

struct SU2Oracle {
  clb_config cfg;
  clb_model_desc md;
  int N;
  size_t n3;
  std::vector<double> F, P;
  double aI = 1, aSI = 1, aIM = 1, aDotI = 0, aDotSI = 0, aDotSIM = 0;
  // cached averages (scalarbase, complexscalarbase, su2doubletbase, u1base, su2base)
  double pi2S = 0, pi2SSI = 0, pi2SSIM = 0, g2S = 0;
  double pi2C = 0, pi2CSI = 0, pi2CSIM = 0, g2C = 0;
  double pi2D = 0, pi2DSI = 0, pi2DSIM = 0, g2D = 0;
  double pi2A = 0, pi2ASI = 0, pi2ASIM = 0, b2A = 0;
  double pi2G = 0, pi2GSI = 0, pi2GSIM = 0, b2G = 0;
  double potI = 0;
  // position Verlet: field averages at the half step (positionverlet.h:258-266)
  double g2S_SI = 0, g2C_SI = 0, g2D_SI = 0, b2A_SI = 0, b2G_SI = 0, potSI = 0;
  // fixed background (fixedbackgroundexpansion.h:21-45): pEoS, H0, the main loop's time t
  bool fb = false;
  double pEoS = 0, H0fb = 0, t = 0;
  double aBg(double d) const { return std::pow(1 + H0fb / pEoS * d, pEoS); }
  double aBgDot(double d) const { return H0fb * std::pow(1 + H0fb / pEoS * d, pEoS - 1); }

  bool synced = true, initialized = false;
  std::vector<double> ws;
  std::string err;
  oracle_models::GWs gw; // the GW sector (PITensor.h source: S, phi and A)

  double qG() const { return md.couplings[0]; }
  double qH() const { return md.couplings[1]; }
  double gC() const { return md.couplings[2]; }
  double gD() const { return md.couplings[3]; }
  double gS() const { return md.couplings[4]; }
  double c4() const { return md.couplings[5]; }
  double rfo2() const { const double r = md.fStar / md.omegaStar; return r * r; }
  double rof2() const { const double r = md.omegaStar / md.fStar; return r * r; }

  double *f(int c) { return F.data() + (size_t)c * n3; }
  const double *f(int c) const { return F.data() + (size_t)c * n3; }
  double *p(int c) { return P.data() + (size_t)c * n3; }
  const double *p(int c) const { return P.data() + (size_t)c * n3; }

  size_t at(int x, int y, int z) const { return ((size_t)x * N + y) * N + z; }
  int wrap(int i) const { return i < 0 ? i + N : (i >= N ? i - N : i); }

  // PITensor.h's anisotropic tensor of lphi4SU2U1 at (x, y, z): the singlet S, then the complex
  // scalar phi and the U(1) field; the doublet and the SU(2) field source none
  void gwTensor(int x, int y, int z, double (&T)[6]) const
  {
    const size_t s = at(x, y, z);
    const size_t nbp[3] = {at(wrap(x + 1), y, z), at(x, wrap(y + 1), z), at(x, y, wrap(z + 1))};
    double g[3];
    for (int i = 0; i < 3; ++i) g[i] = (f(0)[nbp[i]] - f(0)[s]) / cfg.dx;
    const int I[6] = {0, 0, 0, 1, 1, 2}, J[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) T[k] = g[I[k]] * g[J[k]];
    const double *const A[3] = {f(7), f(8), f(9)};
    const double *const pA[3] = {p(7), p(8), p(9)};
    oracle_models::gw_gauge_tensor(f(1), f(2), A, pA, nbp, s, cfg.dx, gC(), aI, rfo2(), false, T);
  }
  void gwKick(double w)
  {
    gw.kick(N, cfg.dx, aI, md.alpha, w * cfg.dt, [&](int x, int y, int z, double (&T)[6]) { gwTensor(x, y, z, T); });
  }
  size_t nb(int x, int y, int z, int d1, int s1, int d2 = 0, int s2 = 0) const
  {
    int c[3] = {x, y, z};
    c[d1] += s1;
    c[d2] += s2;
    return at(wrap(c[0]), wrap(c[1]), wrap(c[2]));
  }
  Qt link(int i, size_t s) const
  {
    const int b = 10 + 4 * i;
    return Qt{f(b)[s], f(b + 1)[s], f(b + 2)[s], f(b + 3)[s]};
  }
  Dbl dbl(size_t s) const { return Dbl{cd(f(3)[s], f(4)[s]), cd(f(5)[s], f(6)[s])}; }
  cd cs(size_t s) const { return cd(f(1)[s], f(2)[s]); }
  // U(1) link of a matter field of coupling g: complexPhase(-dx g A_i)  (gaugederivatives.h:92-115)
  cd phase(double g, int i, size_t s) const
  {
    const double th = (-cfg.dx * g) * f(7 + i)[s];
    return cd(std::cos(th), std::sin(th));
  }
  double normD(size_t s) const
  {
    double a = 0;
    for (int c = 0; c < 4; ++c) a = c == 0 ? f(3)[s] * f(3)[s] : a + f(3 + c)[s] * f(3 + c)[s];
    return std::sqrt(a);
  }
  double normC(size_t s) const { return std::sqrt(f(1)[s] * f(1)[s] + f(2)[s] * f(2)[s]); }
  // potential terms (lphi4SU2U1.h:147-160), with c4 on the quartic term
  double potTerm(int k, size_t s) const
  {
    const double nD = normD(s);
    if (k == 0) return c4() * ipow(nD, 4);
    if (k == 1) return qG() * ipow(nD * f(0)[s], 2);
    return 2 * qH() * ipow(nD * normC(s), 2);
  }
  double pot(size_t s) const { return (potTerm(0, s) + potTerm(1, s)) + potTerm(2, s); }

  // W_D = e^{i theta_D} (U_i Phi(x+i)): covariant forward neighbour of the doublet
  Dbl wD(int i, int x, int y, int z) const
  {
    const size_t s = at(x, y, z), sp = nb(x, y, z, i, +1);
    return dscale(phase(gD(), i, s), qapply(link(i, s), dbl(sp)));
  }
  cd wC(int i, int x, int y, int z) const
  {
    const size_t s = at(x, y, z), sp = nb(x, y, z, i, +1);
    return phase(gC(), i, s) * cs(sp);
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

  // ---- per-site kernels ----------------------------------------------------------------------
  double lapl(int comp, int x, int y, int z) const // gaugederivatives.h:36-40
  {
    const double *a = f(comp);
    const double c = a[at(x, y, z)];
    double t[3];
    for (int d = 0; d < 3; ++d) t[d] = (a[nb(x, y, z, d, +1)] + a[nb(x, y, z, d, -1)]) - 2 * c;
    return (1.0 / (cfg.dx * cfg.dx)) * ((t[0] + t[1]) + t[2]);
  }
  double fd(int comp, size_t s, size_t sp) const { return (f(comp)[sp] - f(comp)[s]) / cfg.dx; }

  // covariant Laplacians (gaugederivatives.h:48-65)
  cd covLapC(int x, int y, int z) const
  {
    const size_t s = at(x, y, z);
    cd plus(0, 0), minus(0, 0);
    for (int d = 0; d < 3; ++d) {
      const size_t sp = nb(x, y, z, d, +1), sm = nb(x, y, z, d, -1);
      const cd w = phase(gC(), d, s) * cs(sp);
      const cd m = std::conj(phase(gC(), d, sm)) * cs(sm);
      plus = d == 0 ? w : plus + w;
      minus = d == 0 ? m : minus + m;
    }
    const double dx2 = cfg.dx * cfg.dx;
    const cd c = cs(s);
    return cd(((plus.real() + minus.real()) - 6 * c.real()) / dx2, ((plus.imag() + minus.imag()) - 6 * c.imag()) / dx2);
  }
  Dbl covLapD(int x, int y, int z) const
  {
    const size_t s = at(x, y, z);
    Dbl plus{}, minus{};
    for (int d = 0; d < 3; ++d) {
      const size_t sp = nb(x, y, z, d, +1), sm = nb(x, y, z, d, -1);
      const Dbl w = qapply(link(d, s), dscale(phase(gD(), d, s), dbl(sp)));
      const Dbl m = qapply(qdag(link(d, sm)), dscale(std::conj(phase(gD(), d, sm)), dbl(sm)));
      if (d == 0) {
        plus = w;
        minus = m;
      } else {
        plus = Dbl{plus.u + w.u, plus.v + w.v};
        minus = Dbl{minus.u + m.u, minus.v + m.v};
      }
    }
    const double dx2 = cfg.dx * cfg.dx;
    const Dbl c = dbl(s);
    auto one = [&](const cd &pl, const cd &mi, const cd &cc) {
      return cd(((pl.real() + mi.real()) - 6 * cc.real()) / dx2, ((pl.imag() + mi.imag()) - 6 * cc.imag()) / dx2);
    };
    return Dbl{one(plus.u, minus.u, c.u), one(plus.v, minus.v, c.v)};
  }

  // all momentum kernels at a site, in momentum-component order
  void kernels(int x, int y, int z, double K[NP]) const
  {
    const size_t s = at(x, y, z);
    const double al = md.alpha;
    const double A = std::pow(aI, 1 + al), B = std::pow(aI, 3 + al), B2 = std::pow(aI, 3 + al) / 2;
    const double nD = normD(s), nC = normC(s), S = f(0)[s];
    // scalar singlet (scalarsingletkernels.h:34-38, lphi4SU2U1.h:167-170)
    K[0] = A * lapl(0, x, y, z) - B * (2 * qG() * ipow(nD, 2) * S);
    // complex scalar (complexscalarkernels.h:33-34, lphi4SU2U1.h:172-175)
    const cd cl = covLapC(x, y, z);
    const double ndC = 4 * qH() * ipow(nD, 2) * nC;
    K[1] = A * cl.real() - B2 * (ndC / nC * f(1)[s]);
    K[2] = A * cl.imag() - B2 * (ndC / nC * f(2)[s]);
    // doublet (su2doubletkernels.h:28-33, lphi4SU2U1.h:177-182)
    const Dbl dl = covLapD(x, y, z);
    const double ndD = c4() * (4 * ipow(nD, 3)) + nD * (2 * qG() * ipow(S, 2) + 4 * qH() * ipow(nC, 2));
    const double cl4[4] = {dl.u.real(), dl.u.imag(), dl.v.real(), dl.v.imag()};
    for (int c = 0; c < 4; ++c) K[3 + c] = A * cl4[c] - B2 * (ndD / nD * f(3 + c)[s]);
    // U(1) (u1kernels.h:31-52, mattercurrents.h:52-76)
    const Dbl D0 = dbl(s);
    const cd C0 = cs(s);
    for (int i = 0; i < 3; ++i) {
      const double lap = lapl(7 + i, x, y, z);
      double grad = 0;
      for (int j = 0; j < 3; ++j) {
        const size_t sj = nb(x, y, z, j, -1);
        const double g0 = fd(7 + j, s, nb(x, y, z, i, +1));
        const double g1 = fd(7 + j, sj, nb(x, y, z, i, +1, j, -1));
        const double t = (g0 - g1) / cfg.dx;
        grad = j == 0 ? t : grad + t;
      }
      const double Jc = gC() * (std::conj(wC(i, x, y, z)) * C0).imag();
      const double Jd = gD() * sprod(wD(i, x, y, z), D0).imag();
      const double J = 2.0 / cfg.dx * rfo2() * (Jc + Jd);
      K[7 + i] = std::pow(aI, -1 + al) * (lap - grad) - std::pow(aI, 1 + al) * J;
    }
    // SU(2) (su2kernels.h:30-54, mattercurrents.h:102-119)
    const double normGrad = ipow(1 / cfg.dx, 3) / gS() * std::pow(aI, -1 + al);
    const double normSrc = (1 / cfg.dx) * std::pow(aI, 1 + al);
    for (int i = 0; i < 3; ++i) {
      double gr[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
      bool first = true;
      for (int j = 0; j < 3; ++j) {
        if (j == i) continue;
        const Qt P = plaq(i, j, x, y, z), Pb = plaqBack(i, j, x, y, z);
        const double pv[3] = {P.x, P.y, P.z}, bv[3] = {Pb.x, Pb.y, Pb.z};
        for (int a = 0; a < 3; ++a) {
          gr[a] = first ? pv[a] : gr[a] + pv[a];
          gb[a] = first ? bv[a] : gb[a] + bv[a];
        }
        first = false;
      }
      const Dbl W = wD(i, x, y, z);
      for (int a = 0; a < 3; ++a) {
        const double J = rfo2() / 2 * (gS() * sprod(W, isig(a, D0)).real());
        K[10 + 3 * i + a] = -normGrad * (gr[a] - gb[a]) - normSrc * J;
      }
    }
  }

  Qt plaq(int i, int j, int x, int y, int z) const
  {
    const size_t s = at(x, y, z);
    return qmul(qmul(qmul(link(i, s), link(j, nb(x, y, z, i, +1))), qdag(link(i, nb(x, y, z, j, +1)))), qdag(link(j, s)));
  }
  Qt plaqBack(int i, int j, int x, int y, int z) const
  {
    const size_t s = at(x, y, z), sm = nb(x, y, z, j, -1);
    const Qt P = qmul(qmul(qmul(link(i, s), qdag(link(j, nb(x, y, z, i, +1, j, -1)))), qdag(link(i, sm))), link(j, sm));
    return qdag(P);
  }

  // kick factors per sector: S, phi, Phi, A, SU(2)
  void kick(const double h[5])
  {
    std::vector<double> K((size_t)NP * n3);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < N; ++x)
      for (int y = 0; y < N; ++y)
        for (int z = 0; z < N; ++z) {
          double k[NP];
          kernels(x, y, z, k);
          const size_t s = at(x, y, z);
          for (int c = 0; c < NP; ++c) K[(size_t)c * n3 + s] = k[c];
        }
    for (int c = 0; c < NP; ++c) {
      const double hc = c == 0 ? h[0] : c < 3 ? h[1] : c < 7 ? h[2] : c < 10 ? h[3] : h[4];
      double *pc = p(c);
      const double *kc = K.data() + (size_t)c * n3;
      for (size_t s = 0; s < n3; ++s) pc[s] = pc[s] + hc * kc[s];
    }
  }
  void vv_kick(double w)
  {
    const double dt = cfg.dt;
    const double h[5] = {w * dt / 2, dt / 2 * w, dt / 2 * w, dt * w / 2, dt / 2 * w}; // velocityverlet.h:129-162
    kick(h);
  }
  void lf_kick(double w)
  {
    const double h[5] = {w * cfg.dt, w * cfg.dt, w * cfg.dt, w * cfg.dt, w * cfg.dt}; // leapfrog.h:131-170
    kick(h);
  }
  // drifts (velocityverlet.h:181-222; leapfrog with w = 1)
  void drift(double w, bool lf) { driftWith(w, lf, cfg.dt, std::pow(aSI, md.alpha - 3), std::pow(aSI, md.alpha - 1)); }
  // position Verlet (positionverlet.h:170-222): pow(aI, .) and dt/2, whose halving is exact, so
  // pow (dt/2 w pi), ((pow dt)/2) w, ((pow w) dt)/2 and the link's (((w pow) dx) dt)/2 gQ are
  // the numbers of the formulas below with dt -> dt/2
  void driftPV(double w) { driftWith(w, false, cfg.dt / 2, std::pow(aI, md.alpha - 3), std::pow(aI, md.alpha - 1)); }
  void driftWith(double w, bool lf, double dt, double p3, double p1)
  {
    const double cS = p3;                                 // S: pow * (dt w pi)
    const double cC = lf ? p3 * dt : p3 * dt * w;         // phi, Phi: pow dt w pi
    const double cA = lf ? p1 * dt : p1 * w * dt;         // A: pow w dt pi
    const double cG = lf ? p1 * cfg.dx * dt * gS() : w * p1 * cfg.dx * dt * gS();
    const double dtw = lf ? dt : dt * w;
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < n3; ++s) {
      f(0)[s] = f(0)[s] + cS * (dtw * p(0)[s]);
      for (int c = 1; c < 7; ++c) f(c)[s] = f(c)[s] + cC * p(c)[s];
      for (int i = 0; i < 3; ++i) f(7 + i)[s] = f(7 + i)[s] + cA * p(7 + i)[s] * 1.0;
      for (int i = 0; i < 3; ++i) {
        const Qt E = qexp(cG * p(10 + 3 * i)[s], cG * p(10 + 3 * i + 1)[s], cG * p(10 + 3 * i + 2)[s]);
        const Qt U = qmul(E, link(i, s));
        f(10 + 4 * i)[s] = U.w;
        f(11 + 4 * i)[s] = U.x;
        f(12 + 4 * i)[s] = U.y;
        f(13 + 4 * i)[s] = U.z;
      }
    }
  }

  // ---- volume averages (fieldfunctionals.h, averages.h) --------------------------------------
  double sGrad2(int x, int y, int z) const // Grad2 with the forward difference
  {
    const size_t s = at(x, y, z);
    double acc = 0;
    for (int j = 0; j < 3; ++j) {
      const double g = fd(0, s, nb(x, y, z, j, +1));
      acc = j == 0 ? g * g : acc + g * g;
    }
    return acc;
  }
  double cGrad2(int x, int y, int z) const // grad2CS (fieldfunctionals.h:80-84)
  {
    const cd c = cs(at(x, y, z));
    double acc = 0;
    for (int j = 0; j < 3; ++j) {
      const cd d = (wC(j, x, y, z) - c) / cfg.dx;
      const double n2 = d.real() * d.real() + d.imag() * d.imag();
      acc = j == 0 ? n2 : acc + n2;
    }
    return acc;
  }
  double dGrad2(int x, int y, int z) const // grad2SU2Doublet (fieldfunctionals.h:105-109)
  {
    const size_t s = at(x, y, z);
    const Dbl c = dbl(s);
    double acc = 0;
    for (int j = 0; j < 3; ++j) {
      const Dbl w = qapply(link(j, s), dscale(phase(gD(), j, s), dbl(nb(x, y, z, j, +1))));
      const cd du = (w.u - c.u) / cfg.dx, dv = (w.v - c.v) / cfg.dx;
      const double n2 = (du.real() * du.real() + du.imag() * du.imag()) + (dv.real() * dv.real() + dv.imag() * dv.imag());
      acc = j == 0 ? n2 : acc + n2;
    }
    return acc;
  }
  double aB2(int x, int y, int z) const // B2U1 (fieldfunctionals.h:133-141)
  {
    const size_t s = at(x, y, z);
    auto F = [&](int i, int j) { return fd(7 + j, s, nb(x, y, z, i, +1)) - fd(7 + i, s, nb(x, y, z, j, +1)); };
    const double f21 = F(1, 0), f31 = F(2, 0), f32 = F(2, 1);
    return f21 * f21 + (f31 * f31 + f32 * f32);
  }
  double gB2(int x, int y, int z) const // B2SU2 (fieldfunctionals.h:201-209)
  {
    const double c = 4.0 / (ipow(cfg.dx, 4) * ipow(gS(), 2));
    auto t = [&](int i, int j) { return 2 - 2 * plaq(i, j, x, y, z).w; };
    return c * (t(1, 0) + (t(2, 0) + t(2, 1)));
  }
  double avPiS() const { return average([&](int x, int y, int z) { const double v = p(0)[at(x, y, z)]; return v * v; }); }
  double avPiC() const
  {
    return average([&](int x, int y, int z) { const size_t s = at(x, y, z); return p(1)[s] * p(1)[s] + p(2)[s] * p(2)[s]; });
  }
  double avPiD() const
  {
    return average([&](int x, int y, int z) {
      const size_t s = at(x, y, z);
      return ((p(3)[s] * p(3)[s] + p(4)[s] * p(4)[s]) + p(5)[s] * p(5)[s]) + p(6)[s] * p(6)[s];
    });
  }
  double avPiA() const
  {
    return average([&](int x, int y, int z) {
      const size_t s = at(x, y, z);
      return (p(7)[s] * p(7)[s] + p(8)[s] * p(8)[s]) + p(9)[s] * p(9)[s];
    });
  }
  double avPiG() const // pi2SU2 = sum_i sum_b 4 pi^2 (fieldfunctionals.h:218-223)
  {
    return average([&](int x, int y, int z) {
      const size_t s = at(x, y, z);
      double acc = 0;
      for (int i = 0; i < 3; ++i) {
        double ai = 0;
        for (int b = 0; b < 3; ++b) {
          const double e = p(10 + 3 * i + b)[s];
          ai = b == 0 ? 4 * (e * e) : ai + 4 * (e * e);
        }
        acc = i == 0 ? ai : acc + ai;
      }
      return acc;
    });
  }
  void storeMomenta()
  {
    pi2S = avPiS();
    pi2C = avPiC();
    pi2D = avPiD();
    pi2A = avPiA();
    pi2G = avPiG();
  }
  void storeFields()
  {
    g2S = average([&](int x, int y, int z) { return sGrad2(x, y, z); });
    g2C = average([&](int x, int y, int z) { return cGrad2(x, y, z); });
    g2D = average([&](int x, int y, int z) { return dGrad2(x, y, z); });
    b2A = average([&](int x, int y, int z) { return aB2(x, y, z); });
    b2G = average([&](int x, int y, int z) { return gB2(x, y, z); });
    potI = average([&](int x, int y, int z) { return pot(at(x, y, z)); });
  }
  void setAllAverages()
  {
    storeFields();
    storeMomenta();
    pi2SSI = pi2S;
    pi2CSI = pi2C;
    pi2DSI = pi2D;
    pi2ASI = pi2A;
    pi2GSI = pi2G;
  }

  // energies (energies.h:37-97) as functions of the cached averages
  struct En {
    double ks, gs, kc, gc, kd, gd, ea, ba, eg, bg;
  };
  En energies() const
  {
    const double a6 = ipow(aI, -6), a2 = ipow(aI, -2), e4 = 0.5 * rof2() * ipow(aI, -4);
    return En{0.5 * pi2S * a6, 0.5 * g2S * a2, pi2C * a6, g2C * a2, pi2D * a6, g2D * a2,
              e4 * pi2A * 1.0,  e4 * b2A / 1.0, e4 * pi2G, e4 * b2G};
  }
  double sfKernelSI() const // ScaleFactorKernels::getSI (scalefactorkernels.h:83-119)
  {
    const double al = md.alpha;
    const double a6 = ipow(aI, -6), a2 = ipow(aI, -2), e4 = 0.5 * rof2() * ipow(aI, -4);
    const En E{0.5 * pi2SSI * a6, 0.5 * g2S_SI * a2, pi2CSI * a6, g2C_SI * a2, pi2DSI * a6, g2D_SI * a2,
               e4 * pi2ASI * 1.0,  e4 * b2A_SI / 1.0, e4 * pi2GSI, e4 * b2G_SI};
    const double fm = md.fStar / md.MPl;
    return std::pow(aI, 2 * al + 1) / 3.0 * (fm * fm) *
           ((((al - 2) * ((E.ks + E.kc) + E.kd) + al * ((E.gs + E.gc) + E.gd)) +
             (al - 1) * (((E.ea + E.ba) + E.eg) + E.bg)) +
            (al + 1) * potSI);
  }
  double sfKernel() const // scalefactorkernels.h:73-77
  {
    const double al = md.alpha;
    const En E = energies();
    const double fm = md.fStar / md.MPl;
    return std::pow(aI, 2 * al + 1) / 3.0 * (fm * fm) *
           ((((al - 2) * ((E.ks + E.kc) + E.kd) + al * ((E.gs + E.gc) + E.gd)) +
             (al - 1) * ((1.0 * (E.ea + E.ba) + E.eg) + E.bg)) +
            (al + 1) * potI);
  }
  double rho() const // energies.h:217-239
  {
    const En E = energies();
    return ((((((((((E.ks + E.kc) + E.kd) + E.gs) + E.gc) + E.gd) + E.ea) + E.ba) + E.eg) + E.bg) + 0.0) + potI;
  }
  void hubble(double out[3])
  {
    setAllAverages();
    const double LHS = aDotI * aDotI;
    const double fm = md.fStar / md.MPl;
    const double RHS = std::pow(aI, 2 * md.alpha + 2) / 3. * (fm * fm) * rho();
    out[0] = (LHS - RHS) / (LHS + RHS);
    out[1] = LHS;
    out[2] = RHS;
  }

  // ---- schedules -------------------------------------------------------------------------------
  void evolveVV()
  {
    const double dt = cfg.dt;
    const size_t Pn = ws.size(), stages = (Pn - 1) * 2 + 1;
    const bool ex = cfg.expansion != 0;
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < Pn ? i : stages - i - 1];
      if (ex) aDotSI = aDotI + (dt / 2) * sfKernel() * w;
      vv_kick(w);
      if (ex) {
        storeMomenta();
        aIM = aI;
        aI += dt * aDotSI * w;
        aSI = (aIM + aI) / 2.0;
      }
      drift(w, false);
      if (ex) storeFields();
      vv_kick(w);
      if (ex) {
        storeMomenta();
        aDotI = aDotSI + (dt / 2) * sfKernel() * w;
      }
    }
  }
  // PositionVerlet::evolve (positionverlet.h:45-99, 160-276)
  void evolvePV()
  {
    const double dt = cfg.dt;
    const size_t Pn = ws.size(), stages = (Pn - 1) * 2 + 1;
    const bool ex = cfg.expansion != 0;
    auto upd = [](double &I, double &SI, double &IM, double v) {
      IM = I;
      I = v;
      SI = 0.5 * (I + IM);
    };
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < Pn ? i : stages - i - 1];
      driftPV(w);
      if (ex) {
        aIM = aI;
        aI += dt / 2.0 * aDotI * w;
        aSI = aI;
        storeFields();
        g2S_SI = g2S;
        g2C_SI = g2C;
        g2D_SI = g2D;
        b2A_SI = b2A;
        b2G_SI = b2G;
        potSI = potI;
      }
      const double h[5] = {w * dt, dt * w, dt * w, dt * w, dt * w}; // positionverlet.h:132-157
      kick(h);
      if (ex) {
        upd(pi2S, pi2SSI, pi2SSIM, avPiS());
        upd(pi2C, pi2CSI, pi2CSIM, avPiC());
        upd(pi2D, pi2DSI, pi2DSIM, avPiD());
        upd(pi2A, pi2ASI, pi2ASIM, avPiA());
        upd(pi2G, pi2GSI, pi2GSIM, avPiG());
        aDotI += dt * sfKernelSI() * w;
        aI += dt / 2.0 * aDotI * w;
        aSI = (aIM + aI) / 2.0;
      }
      driftPV(w);
      if (ex) storeFields();
    }
  }
  void lfStoreMomenta()
  {
    auto upd = [](double &I, double &SI, double &SIM, double v) {
      SIM = SI;
      SI = v;
      I = 0.5 * (SIM + SI);
    };
    upd(pi2S, pi2SSI, pi2SSIM, avPiS());
    upd(pi2C, pi2CSI, pi2CSIM, avPiC());
    upd(pi2D, pi2DSI, pi2DSIM, avPiD());
    upd(pi2A, pi2ASI, pi2ASIM, avPiA());
    upd(pi2G, pi2GSI, pi2GSIM, avPiG());
  }
  // fixed background, as in the U(1) oracle: VV (aSI left as it was), leapfrog and position Verlet
  // with a from the closed form, no a-kicks or averages; one step from time t
  void evolveFB()
  {
    const double dt = cfg.dt;
    if (cfg.evolver == CLB_LF) {
      lf_kick(synced ? 0.5 : 1.0);
      aIM = aI;
      aI = aBg(t - cfg.t0 + dt);
      aSI = aBg(t - cfg.t0 + dt / 2.0);
      drift(1.0, true);
      synced = false;
      return;
    }
    const size_t Pn = ws.size(), stages = (Pn - 1) * 2 + 1;
    double tc = t - cfg.t0;
    for (size_t i = 0; i < stages; ++i) {
      const double w = ws[i < Pn ? i : stages - i - 1];
      if (cfg.evolver >= CLB_PV2) {
        driftPV(w);
        aIM = aI;
        aI = aBg(tc + w * dt / 2.0);
        aSI = aI;
        const double h[5] = {w * dt, dt * w, dt * w, dt * w, dt * w};
        kick(h);
        aI = aBg(tc + w * dt);
        driftPV(w);
      } else {
        vv_kick(w);
        aIM = aI;
        aI = aBg(tc + w * dt);
        drift(w, false);
        vv_kick(w);
      }
      tc += dt * w;
    }
  }

  void evolveLF()
  {
    const double dt = cfg.dt;
    const bool ex = cfg.expansion != 0;
    lf_kick(synced ? 0.5 : 1.0);
    if (ex) {
      lfStoreMomenta();
      aDotSIM = aDotSI;
      aDotSI += dt * sfKernel();
      aDotI = (aDotSIM + aDotSI) / 2.0;
      aIM = aI;
      aI += dt * aDotSI;
      aSI = (aIM + aI) / 2.0;
    }
    drift(1.0, true);
    if (ex) storeFields();
    synced = false;
  }
  void syncLF()
  {
    if (!synced) {
      lf_kick(0.5);
      if (cfg.expansion) {
        storeMomenta();
        aDotI = aDotSI + cfg.dt / 2.0 * sfKernel();
      }
    }
    synced = true;
  }

  // ---- Gauss laws (gausslaws.h:34-80) -------------------------------------------------------------
  void gaussU1(double out[3]) const
  {
    const double dx = cfg.dx, nrm = 2 / dx * rfo2();
    auto per = [&](int x, int y, int z, int what) {
      const size_t s = at(x, y, z);
      double l[3];
      for (int i = 0; i < 3; ++i) l[i] = p(7 + i)[s] - p(7 + i)[nb(x, y, z, i, -1)];
      const double LHS = ((l[0] + l[1]) + l[2]) / dx;
      const double imc = (std::conj(cd(p(1)[s], p(2)[s])) * cs(s)).imag();
      const Dbl pd{cd(p(3)[s], p(4)[s]), cd(p(5)[s], p(6)[s])};
      const double imd = sprod(pd, dbl(s)).imag();
      const double rho = nrm * gC() * imc + nrm * gD() * imd;
      const double RHS = -dx * rho;
      const double L1 = l[0] / dx, L2 = l[1] / dx, L3 = l[2] / dx;
      const double diff = LHS - (RHS + 0.0), sum = L1 * L1 + L2 * L2 + L3 * L3 + (RHS + 0.0) * (RHS + 0.0);
      switch (what) {
      case 0: return std::sqrt(diff * diff);
      case 1: return std::sqrt(sum * sum);
      case 2: return std::sqrt(RHS * RHS);
      default: return std::sqrt(LHS * LHS);
      }
    };
    const double d = average([&](int x, int y, int z) { return per(x, y, z, 0); });
    const double sm = average([&](int x, int y, int z) { return per(x, y, z, 1); });
    out[0] = d / sm;
    out[1] = average([&](int x, int y, int z) { return per(x, y, z, 3); });
    out[2] = average([&](int x, int y, int z) { return per(x, y, z, 2); });
  }
  // LHS_b = sum_i (pi_i(x) - [U_i^+ pi_i U_i](x - i))_b / dx, RHS_b = -(fStar/omegaStar)^2/2 g Re((i s_b Phi)^+ pi_Phi)
  void gaussSU2(double out[3]) const
  {
    const double dx = cfg.dx;
    auto lr = [&](int x, int y, int z, double L[3], double R[3]) {
      const size_t s = at(x, y, z);
      for (int b = 0; b < 3; ++b) L[b] = 0;
      for (int i = 0; i < 3; ++i) {
        const size_t sm = nb(x, y, z, i, -1);
        const Qt Ui = link(i, sm);
        const Qt pim{0, p(10 + 3 * i)[sm], p(11 + 3 * i)[sm], p(12 + 3 * i)[sm]};
        const Qt r = qmul(qmul(qdag(Ui), pim), Ui);
        const double rv[3] = {r.x, r.y, r.z};
        for (int b = 0; b < 3; ++b) {
          const double t = (1 / dx) * (p(10 + 3 * i + b)[s] - rv[b]);
          L[b] = i == 0 ? t : L[b] + t;
        }
      }
      const Dbl D0 = dbl(s);
      const Dbl pd{cd(p(3)[s], p(4)[s]), cd(p(5)[s], p(6)[s])};
      for (int b = 0; b < 3; ++b) R[b] = (-1.0) * (rfo2() / 2 * (gS() * sprod(isig(b, D0), pd).real()));
    };
    double acc[4] = {0, 0, 0, 0};
    for (int b = 0; b < 3; ++b) {
      auto comp = [&](int what) {
        return average([&](int x, int y, int z) {
          double L[3], R[3];
          lr(x, y, z, L, R);
          const double v = what == 0 ? L[b] - R[b] : what == 1 ? L[b] + R[b] : what == 2 ? R[b] : L[b];
          return std::sqrt(v * v);
        });
      };
      for (int k = 0; k < 4; ++k) acc[k] = b == 0 ? comp(k) : acc[k] + comp(k);
    }
    out[0] = acc[0] / acc[1];
    out[1] = acc[3];
    out[2] = acc[2];
  }
  void means_row(clb_measurement *m, int r, double a1, double b1, double a2, double b2) const
  {
    const double r1 = a2 - a1 * a1, r2 = b2 - b1 * b1;
    m->means[r][0] = a1;
    m->means[r][1] = b1;
    m->means[r][2] = a2;
    m->means[r][3] = b2;
    m->means[r][4] = r1 > 0 ? std::sqrt(r1) : 0;
    m->means[r][5] = r2 > 0 ? std::sqrt(r2) : 0;
  }
  template <class G> void row_of(clb_measurement *m, int r, G fv, G pv) const
  {
    const double a1 = average(fv), b1 = average(pv);
    const double a2 = average([&](int x, int y, int z) { const double v = fv(x, y, z); return v * v; });
    const double b2 = average([&](int x, int y, int z) { const double v = pv(x, y, z); return v * v; });
    means_row(m, r, a1, b1, a2, b2);
  }
};

} // namespace

namespace oracle_models {

using GFn = std::function<double(int, int, int)>;

void *su2_create(const clb_config *cfg, const clb_model_desc *md, std::string &err)
{
  if (cfg->N < 2) {
    err = "N must be >= 2";
    return nullptr;
  }
  SU2Oracle *o = new SU2Oracle();
  o->cfg = *cfg;
  o->md = *md;
  o->N = cfg->N;
  o->n3 = (size_t)cfg->N * cfg->N * cfg->N;
  o->F.assign((size_t)NF * o->n3, 0.0);
  o->P.assign((size_t)NP * o->n3, 0.0);
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

void su2_destroy(void *h) { delete static_cast<SU2Oracle *>(h); }
std::string &su2_err(void *h) { return static_cast<SU2Oracle *>(h)->err; }

int su2_set_state(void *h, const double *fields, const double *momenta, const clb_scalefactor *sf)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
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

int su2_get_state(void *h, double *fields, double *momenta, clb_scalefactor *sf)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
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

int su2_initialize(void *h, int32_t correct_adot)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
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

int su2_gws_enable(void *h)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
  o->gw.enable(o->n3);
  return CLB_OK;
}
GWs *su2_gws(void *h) { return &static_cast<SU2Oracle *>(h)->gw; }

int su2_evolve(void *h, int64_t n)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
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

int su2_sync(void *h)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
  if (o->gw.on && !o->gw.synced) { // evolver.h:134-137
    o->gwKick(0.5);
    o->gw.synced = true;
  }
  if (o->fb) {
    if (o->cfg.evolver == CLB_LF && !o->synced) o->lf_kick(0.5);
    o->synced = true;
    o->aDotI = o->aBgDot(o->t - o->cfg.t0);
    return CLB_OK;
  }
  if (o->cfg.evolver == CLB_LF) o->syncLF();
  return CLB_OK;
}

// Energies in measurer order: E_kin, E_grad of S, phi, Phi; E_el, E_mag of U(1) and SU(2); the
// three potential terms; E_tot (energiesmeasurer.h:45-122).
int su2_measure(void *h, double e0, clb_measurement *m)
{
  SU2Oracle *o = static_cast<SU2Oracle *>(h);
  std::memset(m, 0, sizeof(*m));
  o->setAllAverages();
  const SU2Oracle::En E = o->energies();
  double V[3];
  for (int k = 0; k < 3; ++k) V[k] = o->average([&](int x, int y, int z) { return o->potTerm(k, o->at(x, y, z)); });
  const double en[10] = {E.ks, E.gs, E.kc, E.gc, E.kd, E.gd, E.ea, E.ba, E.eg, E.bg};
  double Etot = 0;
  int k = 0;
  for (int i = 0; i < 10; ++i) {
    m->energies[k++] = en[i];
    Etot += en[i];
  }
  for (int i = 0; i < 3; ++i) {
    m->energies[k++] = V[i];
    Etot += V[i];
  }
  m->energies[k++] = Etot;
  m->n_energies = k;
  if (o->cfg.expansion)
    o->hubble(m->friedmann);
  else
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  const double am = std::pow(o->aI, o->md.alpha - 3), ag = std::pow(o->aI, o->md.alpha - 1), r2 = std::sqrt(2.0);
  auto S = [&](int x, int y, int z) { return o->at(x, y, z); };
  o->row_of(m, 0, GFn([&](int x, int y, int z) { return o->f(0)[S(x, y, z)]; }),
            GFn([&](int x, int y, int z) { return o->p(0)[S(x, y, z)] * am; }));
  for (int c = 0; c < 2; ++c)
    o->row_of(m, 1 + c, GFn([&](int x, int y, int z) { return r2 * o->f(1 + c)[S(x, y, z)]; }),
              GFn([&](int x, int y, int z) { return r2 * o->p(1 + c)[S(x, y, z)] * am; }));
  o->row_of(m, 3, GFn([&](int x, int y, int z) { return o->normC(S(x, y, z)); }), GFn([&](int x, int y, int z) {
              const size_t s = S(x, y, z);
              const double a = o->p(1)[s] * am, b = o->p(2)[s] * am;
              return std::sqrt(a * a + b * b);
            }));
  o->row_of(m, 4, GFn([&](int x, int y, int z) { return o->normD(S(x, y, z)); }), GFn([&](int x, int y, int z) {
              const size_t s = S(x, y, z);
              double a = 0;
              for (int c = 0; c < 4; ++c) a += o->p(3 + c)[s] * o->p(3 + c)[s];
              return std::sqrt(a) * am;
            }));
  o->row_of(m, 5, GFn([&](int x, int y, int z) {
              const size_t s = S(x, y, z);
              const double e1 = o->p(7)[s] * ag, e2 = o->p(8)[s] * ag, e3 = o->p(9)[s] * ag;
              return std::sqrt(e1 * e1 + e2 * e2 + e3 * e3);
            }),
            GFn([&](int x, int y, int z) {
              const size_t s = S(x, y, z);
              auto Fij = [&](int i, int j) {
                return o->fd(7 + j, s, o->nb(x, y, z, i, +1)) - o->fd(7 + i, s, o->nb(x, y, z, j, +1));
              };
              const double b1 = Fij(2, 1), b2 = Fij(0, 2), b3 = Fij(1, 0);
              return std::sqrt(b1 * b1 + b2 * b2 + b3 * b3);
            }));
  // SU(2) |E|, |B| as sqrt of the site densities (su2measurer.h:60-64)
  o->row_of(m, 6, GFn([&](int x, int y, int z) {
              const size_t s = S(x, y, z);
              double acc = 0;
              for (int c = 0; c < 9; ++c) acc += 4 * o->p(10 + c)[s] * o->p(10 + c)[s];
              return ag * std::sqrt(acc);
            }),
            GFn([&](int x, int y, int z) { return std::sqrt(o->gB2(x, y, z)); }));
  m->n_means = 7;
  o->gaussU1(m->gauss_u1);
  o->gaussSU2(m->gauss_su2);
  m->aI = o->aI;
  m->aDotI = o->aDotI;
  m->hubble = o->aDotI / o->aI;
  return CLB_OK;
}

} // namespace oracle_models
