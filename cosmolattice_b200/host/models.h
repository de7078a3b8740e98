// models.h - host side of the three model headers (models/lphi4.h, models/lphi4U1.h,
// models/lphi4SU2U1.h of CosmoLattice) for the C++20 host program: the parameter-file keys each
// header reads, its rescalings (alpha, fStar, omegaStar), the homogeneous initial values in
// program units, the couplings the library's kernels take, pot0 and the masses at the homogeneous
// point (AbstractModel::setInitialPotentialAndMassesFromPotential, abstractmodel.h:220-248, with
// the 1e-14 floor of a vanishing condensate, :282), and the measurement files the reference's
// measurers write for the model (energiesmeasurer.h:127-150, meansmeasurer.h, complexscalarmeasurer.h,
// su2doubletmeasurer.h, u1measurer.h, su2measurer.h).
#pragma once

#include "../../include/clb200.h"

#include <cmath>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace host {

constexpr double kReducedPlanckGeV = 2.435e18;

// ParameterParser: "key = value" lines ('#' starts a comment), later keys override earlier ones.
struct Params {
  std::map<std::string, std::string> kv;

  void add_line(std::string line)
  {
    if (auto c = line.find('#'); c != std::string::npos) line.erase(c);
    const auto eq = line.find('=');
    if (eq == std::string::npos) return;
    auto trim = [](std::string s) {
      const auto a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
      return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    };
    const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
    if (!k.empty()) kv[k] = v;
  }
  bool has(const std::string &k) const { return kv.count(k) != 0; }
  std::string str(const std::string &k, const std::string &d) const { return has(k) ? kv.at(k) : d; }
  double num(const std::string &k, double d) const { return has(k) ? std::stod(kv.at(k)) : d; }
  double num(const std::string &k) const
  {
    if (!has(k)) throw std::runtime_error("Parameter " + k + " is missing.");
    return std::stod(kv.at(k));
  }
  std::vector<double> nums(const std::string &k) const
  {
    std::vector<double> out;
    if (!has(k)) return out;
    std::istringstream is(kv.at(k));
    for (double x; is >> x;) out.push_back(x);
    return out;
  }
  double first(const std::string &k, double d) const
  {
    const auto v = nums(k);
    return v.empty() ? d : v[0];
  }
  bool flag(const std::string &k, bool d) const
  {
    if (!has(k)) return d;
    const std::string v = kv.at(k);
    return v == "true" || v == "1" || v == "True" || v == "TRUE";
  }
};

// One spectra_<name>.txt: column groups, each the sum of the spectra of (which, comp) pairs.
struct SpectrumSet {
  std::string name;
  std::vector<std::vector<std::pair<int, int>>> columns;
};

struct HostModel {
  std::string name;
  int kind = CLB_MODEL_LPHI4;
  int n_scalars = 0;
  double alpha = 1.0, fStar = 1.0, omegaStar = 1.0, MPl = kReducedPlanckGeV;
  std::vector<double> couplings;
  std::vector<double> m2, f0, p0; // matter components in the model's order (program units)
  double charge[4] = {0, 0, 0, 0};
  double pot0 = 0.0, kin0 = 0.0;  // at the homogeneous point, program units
  double fluct_amplitude = -1.0;
  std::vector<std::string> energy_headers, mean_files, gauss_files;
  std::vector<SpectrumSet> spectra;

  clb_model_desc desc() const
  {
    clb_model_desc md{};
    md.kind = kind;
    md.n_scalars = n_scalars;
    md.alpha = alpha;
    md.fStar = fStar;
    md.omegaStar = omegaStar;
    md.MPl = MPl;
    for (size_t i = 0; i < couplings.size() && i < CLB_MAX_COUPLINGS; ++i) md.couplings[i] = couplings[i];
    return md;
  }
};

// deriv2ComponentFromNorm (potential.h:36-42) at a homogeneous point
inline double deriv2_component(double nd, double nd2, const std::vector<double> &comps, size_t c)
{
  double n2 = 0;
  for (double v : comps) n2 += v * v;
  const double n = std::sqrt(n2);
  return 1.0 / n2 * nd2 * comps[c] * comps[c] + nd / n * (1 - comps[c] * comps[c] / n2);
}

inline std::vector<std::string> means_header() { return {"t", "<phi>", "<pi>", "<phi^2>", "<pi^2>", "rms(phi)", "rms(pi)"}; }
inline std::vector<std::string> means_header_eb() { return {"t", "<|E|>", "<|B|>", "<|E|^2>", "<|B|^2>", "rms(|E|)", "rms(|B|)"}; }

// models/lphi4.h: V = c0/4 phi^4 + q/2 phi^2 chi^2 (one field: the daughter removed).  Keys:
// lambda, q, lambda_prog, initial_amplitudes (one or two), initial_momenta.
inline HostModel make_lphi4(const Params &par)
{
  HostModel m;
  std::vector<double> phi0 = par.nums("initial_amplitudes"), pi0 = par.nums("initial_momenta");
  if (phi0.empty() || phi0.size() > 2) throw std::runtime_error("initial_amplitudes takes one or two values");
  const int Ns = (int)phi0.size();
  pi0.resize(Ns, 0.0);
  m.name = Ns == 1 ? "lphi4_1f" : "lphi4";
  m.kind = CLB_MODEL_LPHI4;
  m.n_scalars = Ns;
  const double lambda = par.num("lambda"), q = Ns == 2 ? par.num("q", 0.0) : 0.0;
  const double c0 = par.num("lambda_prog", 1.0);
  m.fStar = phi0[0];
  m.omegaStar = std::sqrt(lambda) * m.fStar; // lphi4.h:125-127
  m.MPl = par.num("MPl", kReducedPlanckGeV);
  m.couplings = {c0, q};
  std::vector<double> f(Ns);
  for (int i = 0; i < Ns; ++i) {
    f[i] = phi0[i] / m.fStar;
    m.f0.push_back(f[i]);
    m.p0.push_back(pi0[i] / m.fStar / m.omegaStar);
    m.kin0 += 0.5 * m.p0[i] * m.p0[i]; // Energies::kineticS at a = 1
  }
  m.pot0 = 0.25 * c0 * std::pow(f[0], 4) + (Ns == 2 ? 0.5 * q * std::pow(f[0] * f[1], 2) : 0.0);
  m.m2.push_back(3 * c0 * f[0] * f[0] + (Ns == 2 ? q * f[1] * f[1] : 0.0));
  if (Ns == 2) m.m2.push_back(q * f[0] * f[0]);
  m.energy_headers = {"t"};
  for (int i = 0; i < Ns; ++i) {
    m.energy_headers.push_back("E^kin_scal" + std::to_string(i));
    m.energy_headers.push_back("E^grad_scal" + std::to_string(i));
    m.mean_files.push_back("scalar_" + std::to_string(i));
    m.spectra.push_back({"scalar_" + std::to_string(i), {{{0, i}}, {{1, i}}}});
  }
  for (int k = 0; k < Ns; ++k) m.energy_headers.push_back("Vpot_term_" + std::to_string(k));
  m.energy_headers.push_back("E_tot");
  return m;
}

// models/lphi4U1.h: one complex scalar under one U(1), V = c4 |phi|^4.  Keys: lambda, lambda_prog,
// cmplx_field_initial_norm, cmplx_momentum_initial_norm, gU1s, CSU1_charges.
inline HostModel make_lphi4U1(const Params &par)
{
  HostModel m;
  m.name = "lphi4U1";
  m.kind = CLB_MODEL_LPHI4U1;
  const double lambda = par.num("lambda"), c4 = par.num("lambda_prog", 1.0);
  const double n0 = par.num("cmplx_field_initial_norm"), np0 = par.num("cmplx_momentum_initial_norm", 0.0);
  const double gQ = par.first("gU1s", 1.0) * par.first("CSU1_charges", 1.0); // couplingsmanager.h
  m.fStar = n0;
  m.omegaStar = std::sqrt(lambda) * n0; // lphi4U1.h:95-97
  m.MPl = par.num("MPl", kReducedPlanckGeV);
  m.couplings = {c4, gQ};
  std::vector<double> c = {n0 / std::sqrt(2.0) / m.fStar, n0 / std::sqrt(2.0) / m.fStar};
  m.f0 = c;
  m.p0 = {np0 / std::sqrt(2.0) / m.fStar / m.omegaStar, np0 / std::sqrt(2.0) / m.fStar / m.omegaStar};
  m.kin0 = m.p0[0] * m.p0[0] + m.p0[1] * m.p0[1]; // Energies::kineticCS, no 1/2 (energies.h:47-50)
  const double n2 = c[0] * c[0] + c[1] * c[1];
  m.pot0 = c4 * n2 * n2;
  if (c[0] == 0 && c[1] == 0) c = {1e-14 * 0.70710678118654752, 1e-14 * 0.70710678118654752};
  const double n = std::sqrt(c[0] * c[0] + c[1] * c[1]);
  for (size_t i = 0; i < 2; ++i) m.m2.push_back(deriv2_component(c4 * 4 * n * n * n, c4 * 12 * n * n, c, i));
  m.charge[0] = gQ;
  m.energy_headers = {"t", "E^kin_cmplxscal0", "E^grad_cmplxscal0", "E^kin_U10", "E^grad_U10", "Vpot_term_0", "E_tot"};
  m.mean_files = {"cmplx_scalar_0_0", "cmplx_scalar_0_1", "norm_cmplx_scalar_0", "norm_U1_0"};
  m.gauss_files = {"gauss_U1_0"};
  m.spectra = {{"norm_cmplx_scalar_0", {{{0, 0}, {0, 1}}, {{1, 0}, {1, 1}}}}, {"norm_U1_0", {{{1, 2}, {1, 3}, {1, 4}}}}};
  return m;
}

// models/lphi4SU2U1.h: S, a complex scalar phi (U(1)), an SU(2) doublet Phi (U(1) x SU(2)),
// V = c4 |Phi|^4 + qG (|Phi| S)^2 + 2 qH (|Phi| |phi|)^2.  Keys: lambda, lambda_prog, qG, qH,
// initial_amplitudes, initial_momenta, cmplx_field_initial_norm, cmplx_momentum_initial_norm,
// SU2Doublet_initial_norm, SU2Doublet_initial_momenta_norm, gU1s, gSU2s, CSU1_charges,
// SU2DoubletU1_charges, SU2DoubletSU2_charges.
inline HostModel make_lphi4SU2U1(const Params &par)
{
  HostModel m;
  m.name = "lphi4SU2U1";
  m.kind = CLB_MODEL_LPHI4SU2U1;
  m.n_scalars = 1;
  const double lambda = par.num("lambda"), c4 = par.num("lambda_prog", 1.0);
  const double qG = par.num("qG"), qH = par.num("qH");
  const double nD = par.num("SU2Doublet_initial_norm"), npD = par.num("SU2Doublet_initial_momenta_norm", 0.0);
  const double nC = par.num("cmplx_field_initial_norm", 0.0), npC = par.num("cmplx_momentum_initial_norm", 0.0);
  const double gU1 = par.first("gU1s", 1.0), gSU2 = par.first("gSU2s", 1.0);
  const double gQ_C = par.first("CSU1_charges", 1.0) * gU1, gQ_D = par.first("SU2DoubletU1_charges", 1.0) * gU1;
  const double gQ_S = par.first("SU2DoubletSU2_charges", 1.0) * gSU2;
  m.fStar = nD;
  m.omegaStar = std::sqrt(lambda) * nD; // lphi4SU2U1.h:118-121
  m.MPl = par.num("MPl", kReducedPlanckGeV);
  m.couplings = {qG, qH, gQ_C, gQ_D, gQ_S, c4};
  const double fs = m.fStar, ws = m.omegaStar;
  const double S = par.num("initial_amplitudes", 0.0) / fs, pS = par.num("initial_momenta", 0.0) / fs / ws;
  std::vector<double> C(2, nC / std::sqrt(2.0) / fs), D(4, nD / 2 / fs);
  const double pC = npC / std::sqrt(2.0) / fs / ws, pD = npD / 2 / fs / ws;
  m.f0 = {S, C[0], C[1], D[0], D[1], D[2], D[3]};
  m.p0 = {pS, pC, pC, pD, pD, pD, pD};
  m.kin0 = 0.5 * pS * pS + 2 * pC * pC + 4 * pD * pD; // kineticS, kineticCS, kineticSU2Doublet
  if (C[0] == 0 && C[1] == 0) C = {1e-14 * 0.70710678118654752, 1e-14 * 0.70710678118654752};
  if (D[0] == 0 && D[1] == 0 && D[2] == 0 && D[3] == 0) D = std::vector<double>(4, 1e-14 / 2);
  auto norm = [](const std::vector<double> &v) {
    double s = 0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
  };
  const double nDv = norm(D), nCv = norm(C);
  m.pot0 = c4 * std::pow(nDv, 4) + qG * std::pow(nDv * S, 2) + 2 * qH * std::pow(nDv * nCv, 2);
  m.m2.push_back(2 * qG * nDv * nDv);
  const double ndC = 4 * qH * nDv * nDv * nCv, nd2C = 4 * qH;
  for (size_t i = 0; i < 2; ++i) m.m2.push_back(deriv2_component(ndC, nd2C, C, i));
  const double ndD = 4 * c4 * std::pow(nDv, 3) + nDv * (2 * qG * S * S + 4 * qH * nCv * nCv);
  const double nd2D = 12 * c4 * nDv * nDv + 2 * qG * S * S + 4 * qH * nCv * nCv;
  for (size_t i = 0; i < 4; ++i) m.m2.push_back(deriv2_component(ndD, nd2D, D, i));
  m.charge[0] = gQ_S;
  m.charge[1] = gQ_C;
  m.charge[2] = gQ_D;
  m.energy_headers = {"t", "E^kin_scal0", "E^grad_scal0", "E^kin_cmplxscal0", "E^grad_cmplxscal0", "E^kin_SU2matter",
                      "E^grad_SU2matter", "E^kin_U10", "E^grad_U10", "E^kin_SU2", "E^grad_SU2", "Vpot_term_0",
                      "Vpot_term_1", "Vpot_term_2", "E_tot"};
  m.mean_files = {"scalar_0", "cmplx_scalar_0_0", "cmplx_scalar_0_1", "norm_cmplx_scalar_0", "norm_SU2Doublet_0",
                  "norm_U1_0", "norm_SU2_0"};
  m.gauss_files = {"gauss_U1_0", "gauss_SU2_0"};
  m.spectra = {{"scalar_0", {{{0, 0}}, {{1, 0}}}},
               {"norm_cmplx_scalar_0", {{{0, 1}, {0, 2}}, {{1, 1}, {1, 2}}}},
               {"norm_SU2Doublet_scalar_0", {{{0, 3}, {0, 4}, {0, 5}, {0, 6}}, {{1, 3}, {1, 4}, {1, 5}, {1, 6}}}},
               {"norm_U1_0", {{{1, 7}, {1, 8}, {1, 9}}}}};
  return m;
}

inline HostModel make_model(const std::string &name, const Params &par)
{
  HostModel m;
  if (name == "lphi4") m = make_lphi4(par);
  else if (name == "lphi4U1") m = make_lphi4U1(par);
  else if (name == "lphi4SU2U1") m = make_lphi4SU2U1(par);
  else throw std::runtime_error("unknown model " + name + " (lphi4, lphi4U1, lphi4SU2U1)");
  if (par.has("fluct_amplitude")) m.fluct_amplitude = par.num("fluct_amplitude");
  return m;
}

} // namespace host
