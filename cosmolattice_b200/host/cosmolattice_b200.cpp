// cosmolattice_b200.cpp - C++20 host of the lphi4, lphi4U1 and lphi4SU2U1 models over the libclb200
// C ABI.
//
// The reference's main (source/cosmolattice.cpp:134-201) for one model header (models.h; the key
// `model` names it, where the reference picks it at compile time): the run parameters and model
// keys of a reference parameter file; the initial state drawn on the GPU (clb_generate_state, the
// FluctuationsGenerator recipe and the Gauss solves), then clb_initialize (ModelInitializer's scale
// factor and aDot correction, modelinitializer.h:47-81) - or, with restart = true, the state of a
// restart file (SimulationManager::loadSim, simulationmanager.h:69-100); then the time loop
//   while (t < tMax - dt/2) { sync and measure every round(tOutputFreq/dt) steps, spectra every
//   round(tOutputInfreq/dt) steps; evolve; backup every round(tBackupFreq/dt) steps }
// writing the measurers' files: average_energies.txt, average_energy_conservation.txt,
// average_scale_factor.txt, the means files of every field, the Gauss-law files of the gauge
// fields (measurementssaverstd.h:61-82, 15 significant digits) and spectra_<name>.txt
// (spectrumsaverstd.h:54-96); with withGWs, spectra_energy_gws.txt and average_energies_gws.txt at
// the spectra cadence (gwsmeasurer.h:41-53).  Steps between two measurements go to the GPU in one
// clb_evolve.
//
// Usage: cosmolattice_b200 [input.in] [key=value ...]
// Keys (runparameters.h:60-236 and the model headers, models.h): N, kIR or lSide, dt, tMax, t0,
// evolver, expansion, fixedBackground, omegaEoS, H0, a0, tOutputFreq, tOutputInfreq, kCutOff,
// outputfile, print_headers, PS_type, PS_version, deltaKBin, restart, restartFile, tBackupFreq,
// backupPath, saveFile, withGWs, doLFforGWs, GWprojectorType, and the model's keys; host keys:
// model (lphi4 | lphi4U1 | lphi4SU2U1), precision (fp64 | fp32), path (fused | reference),
// deviceSeed (the Philox key; default: FNV-1a of baseSeed).
//
// Restart files use the layout of cosmolattice_b200/restart.py (HDF5 is not available): a magic,
// a header, each sector's field then momentum arrays in the reference's save order (with GWs, their
// five field/momentum pairs after the scalar singlets), the six scale-factor values and tSave, and
// the parameter lines.

#include "../../include/clb200.h"
#include "models.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using host::HostModel;
using host::Params;

constexpr double kPi = 3.14159265358979323846;

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

std::string fmt15(double v)
{
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.15g", v);
  return buf;
}

struct Out {
  std::ofstream f;
  void row(const std::vector<double> &v, const char *sep = "    ")
  {
    for (size_t i = 0; i < v.size(); ++i) f << (i ? sep : "") << fmt15(v[i]);
    f << '\n';
    f.flush();
  }
};

std::string join(const std::vector<std::string> &v, const char *sep = "    ")
{
  std::string s;
  for (size_t i = 0; i < v.size(); ++i) s += (i ? sep : "") + v[i];
  return s;
}

// ---- restart files (the layout of cosmolattice_b200/restart.py) -------------------------------
const char kMagic[16] = {'C', 'L', 'B', '2', '0', '0', '-', 'R', 'E', 'S', 'T', 'A', 'R', 'T', 0, 0};

// (first field, field count, first momentum, momentum count) per sector, in the reference's save
// order (simulationmanager.h:112-125)
std::vector<std::array<int, 4>> sectors(const HostModel &m)
{
  if (m.kind == CLB_MODEL_LPHI4SU2U1) return {{0, 1, 0, 1}, {1, 2, 1, 2}, {3, 4, 3, 4}, {7, 3, 7, 3}, {10, 12, 10, 9}};
  if (m.kind == CLB_MODEL_LPHI4U1) return {{0, 2, 0, 2}, {2, 3, 2, 3}};
  std::vector<std::array<int, 4>> s;
  for (int i = 0; i < m.n_scalars; ++i) s.push_back({i, 1, i, 1});
  return s;
}

// Index of the first sector after the scalar singlets, where the GW arrays sit (simulationmanager.h:112-114).
size_t gw_slot(const HostModel &m, size_t nsec)
{
  return m.kind == CLB_MODEL_LPHI4SU2U1 ? 1 : m.kind == CLB_MODEL_LPHI4U1 ? 0 : nsec;
}

void save_sim(clb_handle *h, const HostModel &m, int N, double t, const Params &par, const std::string &path, bool gws)
{
  int32_t nf = 0, np = 0;
  clb_num_components(h, &nf, &np);
  const size_t n3 = (size_t)N * N * N;
  std::vector<double> f((size_t)nf * n3), p((size_t)np * n3), gu, gp;
  clb_scalefactor sf{};
  check(h, clb_get_state(h, f.data(), p.data(), &sf), "clb_get_state");
  if (gws) {
    gu.resize(5 * n3);
    gp.resize(5 * n3);
    check(h, clb_gws_get_state(h, gu.data(), gp.data()), "clb_gws_get_state");
  }
  const auto secs = sectors(m);
  const std::string tmp = path + ".part";
  {
    std::ofstream o(tmp, std::ios::binary);
    if (!o) throw std::runtime_error("cannot write " + tmp);
    o.write(kMagic, 16);
    const int64_t hdr[8] = {1, m.kind, N, nf, np, (int64_t)n3, (int64_t)secs.size(), gws ? 1 : 0};
    o.write(reinterpret_cast<const char *>(hdr), sizeof(hdr));
    for (size_t k = 0; k <= secs.size(); ++k) {
      if (gws && k == gw_slot(m, secs.size()))
        for (int c = 0; c < 5; ++c) { // each GW field component, then its momentum
          o.write(reinterpret_cast<const char *>(gu.data() + (size_t)c * n3), (std::streamsize)(n3 * 8));
          o.write(reinterpret_cast<const char *>(gp.data() + (size_t)c * n3), (std::streamsize)(n3 * 8));
        }
      if (k == secs.size()) break;
      const auto &s = secs[k];
      o.write(reinterpret_cast<const char *>(f.data() + (size_t)s[0] * n3), (std::streamsize)(s[1] * n3 * 8));
      o.write(reinterpret_cast<const char *>(p.data() + (size_t)s[2] * n3), (std::streamsize)(s[3] * n3 * 8));
    }
    const double sc[7] = {sf.aSI, sf.aI, sf.aIM, sf.aDotSI, sf.aDotI, sf.aDotSIM, t};
    o.write(reinterpret_cast<const char *>(sc), sizeof(sc));
    std::string text;
    for (const auto &[k, v] : par.kv) text += k + " = " + v + "\n";
    const int64_t len = (int64_t)text.size();
    o.write(reinterpret_cast<const char *>(&len), 8);
    o.write(text.data(), len);
    if (!o) throw std::runtime_error("write failed: " + tmp);
  }
  std::filesystem::rename(tmp, path);
}

double load_sim(clb_handle *h, const HostModel &m, int N, const std::string &path, bool gws)
{
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot read restart file " + path);
  char magic[16];
  in.read(magic, 16);
  int64_t hdr[8];
  in.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
  if (!in || std::memcmp(magic, kMagic, 16) != 0 || hdr[0] != 1)
    throw std::runtime_error(path + ": not a restart file of this format");
  if (hdr[1] != m.kind || hdr[2] != N)
    throw std::runtime_error(path + ": saved for another model or lattice size");
  const size_t n3 = (size_t)hdr[5];
  std::vector<double> f((size_t)hdr[3] * n3), p((size_t)hdr[4] * n3), gu, gp;
  const auto secs = sectors(m);
  // header word 7, bit 0: the five GW field and momentum pairs follow the scalar singlets; a run
  // without GWs steps over them (loadSim reads them only for a model with GWs)
  const bool file_gws = (hdr[7] & 1) != 0;
  if (gws && !file_gws) throw std::runtime_error(path + ": the run has GWs, the restart file has none");
  for (size_t k = 0; k <= secs.size(); ++k) {
    if (file_gws && k == gw_slot(m, secs.size())) {
      if (gws) {
        gu.resize(5 * n3);
        gp.resize(5 * n3);
        for (int c = 0; c < 5; ++c) {
          in.read(reinterpret_cast<char *>(gu.data() + (size_t)c * n3), (std::streamsize)(n3 * 8));
          in.read(reinterpret_cast<char *>(gp.data() + (size_t)c * n3), (std::streamsize)(n3 * 8));
        }
      } else {
        in.seekg((std::streamoff)(10 * n3 * 8), std::ios::cur);
      }
    }
    if (k == secs.size()) break;
    const auto &s = secs[k];
    in.read(reinterpret_cast<char *>(f.data() + (size_t)s[0] * n3), (std::streamsize)(s[1] * n3 * 8));
    in.read(reinterpret_cast<char *>(p.data() + (size_t)s[2] * n3), (std::streamsize)(s[3] * n3 * 8));
  }
  double sc[7];
  in.read(reinterpret_cast<char *>(sc), sizeof(sc));
  if (!in) throw std::runtime_error(path + ": truncated");
  const clb_scalefactor sf{sc[1], sc[0], sc[2], sc[4], sc[3], sc[5]};
  check(h, clb_set_state(h, f.data(), p.data(), &sf), "clb_set_state");
  if (gws) check(h, clb_gws_set_state(h, gu.data(), gp.data()), "clb_gws_set_state");
  check(h, clb_initialize(h, CLB_INIT_RESTART), "clb_initialize");
  return sc[6];
}

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
  const double kIR = 2 * kPi / (N * dx);
  const double t0 = par.num("t0", 0.0), tMax = par.num("tMax");
  const bool expansion = par.flag("expansion", true);
  const bool fixedBg = expansion && par.flag("fixedBackground", false);
  const int outFreq = std::max(1, (int)std::lround(par.num("tOutputFreq", 10 * dt) / dt)); // measurer.h:48-53
  const int specFreq = std::max(1, (int)std::lround(par.num("tOutputInfreq", 100 * dt) / dt));
  const int backupFreq = par.has("tBackupFreq") ? std::max(1, (int)std::lround(par.num("tBackupFreq") / dt)) : 0;
  double kCut = par.num("kCutOff", -1.0);
  if (kCut < 0) kCut = 2 * std::sqrt(3.0) * kPi / dx;
  const std::string outdir = par.str("outputfile", "./");
  const int psType = (int)par.num("PS_type", 1), psVersion = (int)par.num("PS_version", 1);
  const double dk = par.num("deltaKBin", 1.0);
  const int nbins = (int)std::floor(std::sqrt(3.0) / 2.0 * N / dk); // runparameters.h:98
  // GWs (runparameters.h:120-123): the reference's default leapfrog over the matter evolver
  const bool withGWs = par.flag("withGWs", false);
  const int gwPrj = (int)par.num("GWprojectorType", 2);
  if (withGWs && !par.flag("doLFforGWs", true))
    throw std::runtime_error("the GWs run as a leapfrog over the matter evolver (doLFforGWs = true) here");
  if (withGWs && (gwPrj < 1 || gwPrj > 3)) throw std::runtime_error("GWprojectorType is 1, 2 or 3");

  const HostModel m = host::make_model(par.str("model", "lphi4"), par);

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
    cfg.H0 = par.num("H0") / m.omegaStar;
  }
  const clb_model_desc md = m.desc();
  clb_handle *h = nullptr;
  check(nullptr, clb_create(&cfg, &md, &h), "clb_create");
  std::unique_ptr<clb_handle, void (*)(clb_handle *)> guard(h, clb_destroy);
  if (withGWs) check(h, clb_gws_enable(h), "clb_gws_enable");

  double t = t0;
  if (par.flag("restart", false)) {
    t = load_sim(h, m, N, par.str("restartFile", outdir + "/" + m.name + "_backup.clb"), withGWs);
  } else {
    // ScaleFactorInitializer (scalefactorinitializer.h:37-65) and the fluctuations on the GPU
    double aDot = 0.0;
    if (fixedBg) aDot = cfg.H0;
    else if (expansion) aDot = m.fStar / m.MPl * std::sqrt((m.kin0 + m.pot0) / 3.0);
    const double a0 = fixedBg ? 1.0 : (expansion ? par.num("a0", 1.0) : 1.0);
    clb_ic_params ic{};
    ic.seed = par.has("deviceSeed") ? std::stoull(par.str("deviceSeed", "0")) : fnv1a(par.str("baseSeed", "0"));
    ic.amplitude = m.fluct_amplitude >= 0 ? m.fluct_amplitude : m.omegaStar / m.fStar;
    ic.k_cutoff = kCut;
    ic.adot = aDot;
    for (size_t i = 0; i < m.m2.size() && i < CLB_IC_MAX; ++i) {
      ic.mass2[i] = m.m2[i];
      ic.fld0[i] = m.f0[i];
      ic.pi0[i] = m.p0[i];
    }
    for (int i = 0; i < 4; ++i) ic.charge[i] = m.charge[i];
    clb_scalefactor sf{a0, a0, a0, aDot, aDot, 0.0};
    check(h, clb_generate_state(h, &ic, &sf), "clb_generate_state");
    check(h, clb_initialize(h, 1), "clb_initialize");
  }

  // ---- output files (measurementssaverstd.h:61-82, spectrumsaverstd.h:54-96)
  const bool headers = par.flag("print_headers", false);
  const bool append = par.flag("appendToFiles", false);
  auto open = [&](const std::string &name, const std::string &hdr) {
    Out o;
    const std::string path = outdir + "/" + name + ".txt";
    o.f.open(path, append ? std::ios::app : std::ios::out);
    if (!o.f) throw std::runtime_error("cannot write " + path);
    if (headers && !append) o.f << hdr << '\n';
    return o;
  };
  Out en = open("average_energies", "#" + join(m.energy_headers));
  Out cons = open("average_energy_conservation", expansion ? "#t    rel_diff_friedmann    LHS_friedmann    RHS_friedmann"
                                                           : "#t    energy_cons");
  Out sfo;
  if (expansion) sfo = open("average_scale_factor", "#t    a    aDot    H");
  std::vector<Out> means, gauss;
  for (const auto &name : m.mean_files)
    means.push_back(open("average_" + name, "#" + join(name.find("U1") != std::string::npos ||
                                                               name.find("norm_SU2_") != std::string::npos
                                                           ? host::means_header_eb()
                                                           : host::means_header())));
  for (const auto &name : m.gauss_files)
    gauss.push_back(open("average_" + name, "#t    av|LHS-RHS|_over_av|LHS+RHS|    av|LHS|    av|RHS|"));
  std::vector<Out> spec;
  for (const auto &s : m.spectra) {
    std::string hdr = "1:binCentralValue";
    for (size_t c = 0; c < s.columns.size(); ++c) hdr += " " + std::to_string(c + 2) + ":PS";
    spec.push_back(open("spectra_" + s.name, hdr));
  }
  // GWsMeasurer::measureSpectra (gwsmeasurer.h:41-53)
  Out gwspec, gwen;
  if (withGWs) {
    gwspec = open("spectra_energy_gws", "1:binCentralValue 2:PS");
    gwen = open("average_energies_gws", "#t    rhoGW_over_rho    rhoGW");
  }

  // ---- the time loop (cosmolattice.cpp:168-201)
  double e0 = 0.0;
  bool have_e0 = false;
  std::vector<double> bins(nbins), acc(nbins);
  for (int64_t i = 0; t < tMax - dt / 2.0;) {
    const bool freq = i % outFreq == 0, infreq = i % specFreq == 0;
    if (freq || infreq) check(h, clb_sync(h), "clb_sync");
    if (freq) {
      clb_measurement mm{};
      check(h, clb_measure(h, have_e0 ? e0 : 1.0, &mm), "clb_measure");
      if (!have_e0) {
        e0 = mm.energies[mm.n_energies - 1];
        have_e0 = true;
        if (!expansion) mm.friedmann[0] = 0.0;
      }
      std::vector<double> row{t};
      row.insert(row.end(), mm.energies, mm.energies + mm.n_energies);
      en.row(row);
      if (expansion) cons.row({t, mm.friedmann[0], mm.friedmann[1], mm.friedmann[2]});
      else cons.row({t, mm.friedmann[0]});
      if (expansion) sfo.row({t, mm.aI, mm.aDotI, mm.hubble});
      for (size_t f = 0; f < means.size() && (int)f < mm.n_means; ++f) {
        std::vector<double> r{t};
        r.insert(r.end(), mm.means[f], mm.means[f] + 6);
        means[f].row(r);
      }
      if (!gauss.empty()) gauss[0].row({t, mm.gauss_u1[0], mm.gauss_u1[1], mm.gauss_u1[2]});
      if (gauss.size() > 1) gauss[1].row({t, mm.gauss_su2[0], mm.gauss_su2[1], mm.gauss_su2[2]});
    }
    if (infreq) {
      for (size_t s = 0; s < m.spectra.size(); ++s) {
        std::vector<std::vector<double>> cols;
        for (const auto &group : m.spectra[s].columns) {
          std::fill(acc.begin(), acc.end(), 0.0);
          for (const auto &[which, comp] : group) {
            check(h, clb_spectrum(h, which, comp, psType, psVersion, dk, nbins, 1, nullptr, bins.data(), nullptr),
                  "clb_spectrum");
            for (int b = 0; b < nbins; ++b) acc[b] += bins[b];
          }
          cols.push_back(acc);
        }
        for (int b = 0; b < nbins; ++b) {
          std::vector<double> r{(b + 0.5) * dk * kIR};
          for (const auto &c : cols) r.push_back(c[b]);
          spec[s].row(r, " ");
        }
        spec[s].f << '\n';
        spec[s].f.flush();
      }
      if (withGWs) {
        double frac = 0.0;
        check(h, clb_gw_spectrum(h, gwPrj, psType, psVersion, dk, nbins, 1, nullptr, bins.data(), nullptr, &frac),
              "clb_gw_spectrum");
        for (int b = 0; b < nbins; ++b) gwspec.row({(b + 0.5) * dk * kIR, bins[b]}, " ");
        gwspec.f << '\n';
        gwspec.f.flush();
        clb_measurement mm{};
        check(h, clb_measure(h, have_e0 ? e0 : 1.0, &mm), "clb_measure");
        const double rho = mm.energies[mm.n_energies - 1];
        gwen.row({t, frac, frac * rho});
      }
    }
    int64_t n = std::min(outFreq - i % outFreq, specFreq - i % specFreq);
    if (backupFreq) n = std::min(n, backupFreq - i % backupFreq);
    const int64_t n_left = std::llround((tMax - t) / dt);
    n = std::max<int64_t>(1, std::min(n, n_left));
    check(h, clb_evolve(h, n), "clb_evolve");
    t += n * dt;
    i += n;
    if (backupFreq && i % backupFreq == 0) { // simulationmanager.h:143-149
      const std::string path = par.str("backupPath", outdir) + "/" + m.name + "_backup.clb";
      if (std::filesystem::exists(path)) std::filesystem::rename(path, path + "~");
      save_sim(h, m, N, t, par, path, withGWs);
    }
  }
  if (par.has("saveFile")) save_sim(h, m, N, t, par, par.str("saveFile", ""), withGWs);
  double ms = 0;
  clb_last_evolve_ms(h, &ms);
  std::printf("%s N=%d %s: t = %.6g, last evolve %.3f ms\n", m.name.c_str(), N, par.str("evolver", "LF").c_str(), t, ms);
  return 0;
} catch (const std::exception &e) {
  std::fprintf(stderr, "cosmolattice_b200: %s\n", e.what());
  return 1;
}
