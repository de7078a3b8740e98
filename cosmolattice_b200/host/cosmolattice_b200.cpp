// cosmolattice_b200.cpp - C++20 host of the lphi4 model over the libclb200 C ABI.
//
// The reference's main (source/cosmolattice.cpp:134-201) for the lphi4 header (models/lphi4.h): the
// run parameters and model keys of a reference parameter file, the initial state drawn on the GPU
// (clb_generate_state, the FluctuationsGenerator recipe), clb_initialize (ModelInitializer's scale
// factor and aDot correction, modelinitializer.h:47-81), then the time loop
//   while (t < tMax - dt/2) { measure every round(tOutputFreq/dt) steps (after sync); evolve; }
// writing average_energies.txt, average_energy_conservation.txt, average_scale_factor.txt and
// average_scalar_<i>.txt as the reference's MeasurementsSaver does (15 significant digits,
// measurementssaverstd.h:61-82).  Steps between two measurements go to the GPU in one clb_evolve.
//
// Usage: cosmolattice_b200 [input.in] [key=value ...]
// Keys (runparameters.h:60-236, lphi4.h:120-226): N, kIR or lSide, dt, tMax, t0, evolver,
// expansion, fixedBackground, omegaEoS, H0, a0, tOutputFreq, kCutOff, outputfile, print_headers,
// lambda, q, lambda_prog, initial_amplitudes (1 or 2 values: one or two fields), initial_momenta,
// fluct_amplitude, MPl; host keys: precision (fp64 | fp32), path (fused | reference), deviceSeed
// (the Philox key; default: FNV-1a of baseSeed).

#include "../../include/clb200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;
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
  bool flag(const std::string &k, bool d) const
  {
    if (!has(k)) return d;
    const std::string v = kv.at(k);
    return v == "true" || v == "1" || v == "True" || v == "TRUE";
  }
};

int evolver_id(const std::string &v) // evolvertype.h:39-82
{
  static const std::map<std::string, int> ids = {{"LF", CLB_LF},   {"VV2", CLB_VV2},     {"VV4", CLB_VV4},
                                                 {"VV6", CLB_VV6}, {"VV8", CLB_VV8},     {"VV10", CLB_VV10},
                                                 {"VV6_2", CLB_VV6_2}, {"PV2", CLB_PV2}, {"PV4", CLB_PV4},
                                                 {"PV6", CLB_PV6}, {"PV8", CLB_PV8},     {"PV10", CLB_PV10},
                                                 {"PV6_2", CLB_PV6_2}};
  if (auto it = ids.find(v); it != ids.end()) return it->second;
  return std::stoi(v);
}

uint64_t fnv1a(const std::string &s)
{
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) h = (h ^ c) * 1099511628211ull;
  return h;
}

void check(clb_handle *h, int rc, const char *what)
{
  if (rc != CLB_OK) throw std::runtime_error(std::string(what) + ": " + clb_last_error(h));
}

struct Out {
  std::ofstream f;
  void row(const std::vector<double> &v)
  {
    char buf[64];
    for (size_t i = 0; i < v.size(); ++i) {
      std::snprintf(buf, sizeof(buf), "%.15g", v[i]);
      f << (i ? "    " : "") << buf;
    }
    f << '\n';
    f.flush();
  }
};

} // namespace

int main(int argc, char **argv)
try {
  Params par;
  int first = 1;
  if (argc > 1 && std::string(argv[1]).find('=') == std::string::npos) {
    std::ifstream in(argv[1]);
    if (!in) throw std::runtime_error(std::string("cannot read ") + argv[1]);
    for (std::string line; std::getline(in, line);) par.add_line(line);
    first = 2;
  }
  for (int i = first; i < argc; ++i) par.add_line(argv[i]);

  // ---- RunParameters (runparameters.h:60-236)
  const int N = (int)par.num("N");
  const double dt = par.num("dt");
  double dx;
  if (par.has("kIR")) dx = 2 * kPi / (N * par.num("kIR"));
  else dx = par.num("lSide") / N;
  const double t0 = par.num("t0", 0.0), tMax = par.num("tMax");
  const bool expansion = par.flag("expansion", true);
  const bool fixedBg = expansion && par.flag("fixedBackground", false);
  const double tOut = par.num("tOutputFreq", 10 * dt);
  const int outFreq = std::max(1, (int)std::lround(tOut / dt)); // measurer.h:48-53
  double kCut = par.num("kCutOff", -1.0);
  if (kCut < 0) kCut = 2 * std::sqrt(3.0) * kPi / dx;
  const std::string outdir = par.str("outputfile", "./");

  // ---- the lphi4 header (models/lphi4.h:120-226): alpha = 1, fStar = phi0, omegaStar = sqrt(lambda) phi0
  std::vector<double> phi0 = par.nums("initial_amplitudes"), pi0 = par.nums("initial_momenta");
  if (phi0.empty() || phi0.size() > 2) throw std::runtime_error("initial_amplitudes takes one or two values");
  const int Ns = (int)phi0.size();
  pi0.resize(Ns, 0.0);
  const double lambda = par.num("lambda"), q = Ns == 2 ? par.num("q", 0.0) : 0.0;
  const double c0 = par.num("lambda_prog", 1.0);
  const double fStar = phi0[0], omegaStar = std::sqrt(lambda) * fStar, MPl = par.num("MPl", kReducedPlanckGeV);
  std::vector<double> f0(Ns), p0(Ns), m2(Ns);
  for (int i = 0; i < Ns; ++i) {
    f0[i] = phi0[i] / fStar;
    p0[i] = pi0[i] / fStar / omegaStar;
  }
  // pot0 and masses2 at the homogeneous point (abstractmodel.h:220-248, lphi4.h:154-206)
  double pot0 = 0.25 * c0 * std::pow(f0[0], 4);
  if (Ns == 2) pot0 += 0.5 * q * std::pow(f0[0] * f0[1], 2);
  m2[0] = 3 * c0 * std::pow(f0[0], 2) + (Ns == 2 ? q * std::pow(f0[1], 2) : 0.0);
  if (Ns == 2) m2[1] = q * std::pow(f0[0], 2);

  clb_config cfg{};
  cfg.N = N;
  cfg.dx = dx;
  cfg.dt = dt;
  cfg.evolver = evolver_id(par.str("evolver", "LF"));
  cfg.expansion = expansion ? 1 : 0;
  cfg.precision = par.str("precision", "fp64") == "fp32" ? CLB_PREC_FP32_SPLIT : CLB_PREC_FP64;
  cfg.path = par.str("path", "fused") == "reference" ? CLB_PATH_REFERENCE : CLB_PATH_FUSED;
  cfg.t0 = t0;
  if (fixedBg) {
    cfg.fixed_background = 1;
    cfg.omega_eos = par.num("omegaEoS", 1.0 / 3.0);
    cfg.H0 = par.num("H0") / omegaStar;
  }
  clb_model_desc md{};
  md.kind = CLB_MODEL_LPHI4;
  md.n_scalars = Ns;
  md.alpha = 1.0;
  md.fStar = fStar;
  md.omegaStar = omegaStar;
  md.MPl = MPl;
  md.couplings[0] = c0;
  md.couplings[1] = q;
  clb_handle *h = nullptr;
  check(nullptr, clb_create(&cfg, &md, &h), "clb_create");

  // ---- ScaleFactorInitializer (scalefactorinitializer.h:37-65) and the fluctuations on the GPU
  double aDot = 0.0;
  if (fixedBg) aDot = cfg.H0;
  else if (expansion) {
    double kin = 0;
    for (int i = 0; i < Ns; ++i) kin += 0.5 * std::pow(pi0[i] / fStar / omegaStar, 2);
    aDot = fStar / MPl * std::sqrt((kin + pot0) / 3.0);
  }
  const double a0 = fixedBg ? 1.0 : (expansion ? par.num("a0", 1.0) : 1.0);
  clb_ic_params ic{};
  ic.seed = par.has("deviceSeed") ? std::stoull(par.str("deviceSeed", "0")) : fnv1a(par.str("baseSeed", "0"));
  ic.amplitude = par.num("fluct_amplitude", omegaStar / fStar);
  ic.k_cutoff = kCut;
  ic.adot = aDot;
  for (int i = 0; i < Ns; ++i) {
    ic.mass2[i] = m2[i];
    ic.fld0[i] = f0[i];
    ic.pi0[i] = p0[i];
  }
  clb_scalefactor sf{a0, a0, a0, aDot, aDot, 0.0};
  check(h, clb_generate_state(h, &ic, &sf), "clb_generate_state");
  check(h, clb_initialize(h, 1), "clb_initialize");

  // ---- output files (measurementssaverstd.h:61-82)
  const bool headers = par.flag("print_headers", false);
  auto open = [&](const std::string &name, const std::string &hdr) {
    Out o;
    o.f.open(outdir + "/average_" + name + ".txt");
    if (!o.f) throw std::runtime_error("cannot write " + outdir + "/average_" + name + ".txt");
    if (headers) o.f << '#' << hdr << '\n';
    return o;
  };
  std::string eh = "t";
  for (int i = 0; i < Ns; ++i) eh += "    E^kin_scal" + std::to_string(i) + "    E^grad_scal" + std::to_string(i);
  for (int k = 0; k < Ns; ++k) eh += "    Vpot_term_" + std::to_string(k);
  eh += "    E_tot";
  Out en = open("energies", eh);
  Out cons = open("energy_conservation", expansion ? "t    rel_diff_friedmann    LHS_friedmann    RHS_friedmann"
                                                   : "t    energy_cons");
  Out sfo;
  if (expansion) sfo = open("scale_factor", "t    a    aDot    H");
  std::vector<Out> means;
  for (int i = 0; i < Ns; ++i)
    means.push_back(open("scalar_" + std::to_string(i), "t    <phi>    <pi>    <phi^2>    <pi^2>    rms(phi)    rms(pi)"));

  // ---- the time loop (cosmolattice.cpp:168-201)
  double t = t0, e0 = 0.0;
  bool have_e0 = false;
  for (int64_t i = 0; t < tMax - dt / 2.0;) {
    if (i % outFreq == 0) {
      check(h, clb_sync(h), "clb_sync");
      clb_measurement m{};
      check(h, clb_measure(h, have_e0 ? e0 : 1.0, &m), "clb_measure");
      if (!have_e0) {
        e0 = m.energies[m.n_energies - 1];
        have_e0 = true;
        if (!expansion) m.friedmann[0] = 0.0;
      }
      std::vector<double> row{t};
      row.insert(row.end(), m.energies, m.energies + m.n_energies);
      en.row(row);
      if (expansion) cons.row({t, m.friedmann[0], m.friedmann[1], m.friedmann[2]});
      else cons.row({t, m.friedmann[0]});
      if (expansion) sfo.row({t, m.aI, m.aDotI, m.hubble});
      for (int f = 0; f < Ns; ++f) {
        std::vector<double> r{t};
        r.insert(r.end(), m.means[f], m.means[f] + 6);
        means[f].row(r);
      }
    }
    int64_t n = outFreq - i % outFreq;
    const int64_t n_left = std::llround((tMax - t) / dt);
    n = std::max<int64_t>(1, std::min(n, n_left));
    check(h, clb_evolve(h, n), "clb_evolve");
    t += n * dt;
    i += n;
  }
  double ms = 0;
  clb_last_evolve_ms(h, &ms);
  std::printf("lphi4 N=%d %s: t = %.6g, last evolve %.3f ms\n", N, par.str("evolver", "LF").c_str(), t, ms);
  clb_destroy(h);
  return 0;
} catch (const std::exception &e) {
  std::fprintf(stderr, "cosmolattice_b200: %s\n", e.what());
  return 1;
}
