// clb_handle.cuh - the libclb200 handle and the launch accounting shared by the API units.
#pragma once

#include "../../include/clb200.h"
#include "clb_internal.cuh"
#include "clb_scalar.cuh"
#include "clb_sweep.cuh"

#include <cuda.h>
#include <cufft.h>

#include <cmath>

#include <string>
#include <vector>

namespace clb {
struct U1Sector;
struct SU2Sector;
struct GWSector;
}
using clb::GWSector;
using clb::U1Sector;
using clb::SU2Sector;
using namespace clb;

struct clb_handle {
  clb_config cfg;
  clb_model_desc md;
  int N = 0;
  size_t n3 = 0;
  int NS = 0;
  bool fp32 = false;
  size_t esz = 8;
  void *fld[2] = {nullptr, nullptr};
  void *pi[2] = {nullptr, nullptr};
  int cf = 0, cp = 0; // current field / momentum buffer
  Pad pd{};           // padded component layout (clb_sweep.cuh)
  CUtensorMap tm_f[2], tm_p[2];
  int S = 3;          // sweep ring stages
  int rs = 0;         // FP32 split storage: current reference slot in DevState
  int shape = 0;      // sweep block shape: 0 ShapeW, 1 ShapeQ, 2 ShapeH (clb_sweep.cuh)
  bool pdl = true;     // programmatic dependent launch in the fused VV loop (CLB_PDL=0: off)
  bool pdl_now = false; // set while the fused loop issues its sweeps and tails
  int bz = 64, by = 8; // sites per block tile in z and y
  size_t sweep_smem = 0;
  int *d_err = nullptr; // set by a sweep whose bounded wait gave up
  DevState *d_st = nullptr;
  double *d_part = nullptr;
  double *d_sums = nullptr;
  size_t part_rows = 0;
  cudaStream_t stream = nullptr;
  std::vector<double> ws;
  // fixed background: a(t - t0) = (1 + H0/p (t - t0))^p (fixedbackgroundexpansion.h:37-45); fb_t is
  // the time t, t0 at clb_initialize and advanced by dt per step as the reference's main loop does
  bool fb = false;
  double fb_p = 0, fb_H0 = 0, fb_t = 0;
  double fb_a(double dtm) const { return std::pow(1 + fb_H0 / fb_p * dtm, fb_p); }
  double fb_adot(double dtm) const { return fb_H0 * std::pow(1 + fb_H0 / fb_p * dtm, fb_p - 1); }
  bool has_state = false, initialized = false, synced = true;
  ScalarArgs sa{};
  SweepArgs sw{};
  SFParams sp{};
  dim3 sweep_grid;
  int sweep_blocks = 0;
  std::string err;
  U1Sector *u1 = nullptr;   // complex scalar + U(1) sector state (clb_u1.cu), null for other models
  SU2Sector *su2 = nullptr; // lphi4SU2U1 state (clb_su2.cu), null for other models
  GWSector *gw = nullptr;   // gravitational waves of the scalar singlets (clb_gws.cu), null when off

  // instrumentation: launch counts always; per-launch CUDA events on the stream when prof
  bool prof = false;
  struct Pend {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> ev_pool;
  std::vector<Pend> pend;
  int64_t launches[16] = {};
  int64_t timed[16] = {};
  double kernel_ms[16] = {};
  cudaEvent_t ev_call[2] = {nullptr, nullptr};
  double last_evolve_ms = 0;
  // per-step history rows of the last evolve call
  double *d_hist = nullptr;
  int64_t hist_cap = 0, hist_rows = 0;
  // staging buffer for FP32 <-> FP64 host transfers
  double *d_stage = nullptr;
  size_t stage_n = 0;
  // spectra: in-place D2Z buffer, cuFFT plan and binning scratch (allocated on first use)
  double *d_spec = nullptr;
  double *d_spec2 = nullptr; // the tangent's transform (clb_tangent_spectrum)
  bool plan_ok = false;
  cufftHandle plan = 0;
  bool plan_inv_ok = false; // Z2D, for spectrum-observable gradients
  cufftHandle plan_inv = 0;
  double *d_spec_part = nullptr;
  unsigned long long *d_spec_cnt = nullptr;
  double *d_spec_out = nullptr;
  unsigned long long *d_spec_outc = nullptr;
  int spec_nbins_cap = 0;

  int fail(int code, const std::string &m)
  {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char *where)
  {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return CLB_ECUDA;
  }
};

namespace {

#define CLB_CHECK_LAUNCH(h, where)                                                                                     \
  do {                                                                                                                 \
    cudaError_t e_ = cudaGetLastError();                                                                               \
    if (e_ != cudaSuccess) return (h)->cuda_fail(e_, where);                                                           \
  } while (0)

enum KKind {
  K_FUSED, K_KICK, K_DRIFT_SWEEP, K_DRIFT, K_RED_PI2, K_RED_FIELDS, K_TAIL, K_MEASURE, K_CONVERT, K_SPECTRUM,
  K_U1_KICK, K_U1_DRIFT, K_U1_REDUCE, K_U1_ADJ, K_INIT, K_GW, K_NKINDS
};
const char *const kKindNames[K_NKINDS] = {"scalar_fused_sweep", "scalar_kick_sweep", "scalar_drift_sweep",
                                          "scalar_drift",       "reduce_pi2",        "reduce_fields",
                                          "tail",               "measure",           "convert",
                                          "spectrum",           "gauge_kick_sweep",  "gauge_drift",
                                          "gauge_reduce",       "u1_adjoint_sweep",  "initial_conditions",
                                          "gw_sweep"};

cudaEvent_t take_event(clb_handle *h)
{
  if (!h->ev_pool.empty()) {
    cudaEvent_t e = h->ev_pool.back();
    h->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Counts a launch and, when profiling, brackets it with events on the handle's stream.
struct ProfScope {
  clb_handle *h;
  int kind;
  cudaEvent_t a = nullptr;
  ProfScope(clb_handle *hh, int k) : h(hh), kind(k)
  {
    ++h->launches[kind];
    if (h->prof) {
      a = take_event(h);
      cudaEventRecord(a, h->stream);
    }
  }
  ~ProfScope()
  {
    if (h->prof) {
      cudaEvent_t b = take_event(h);
      cudaEventRecord(b, h->stream);
      h->pend.push_back({kind, a, b});
    }
  }
};
#define CLB_LAUNCH(h, kind, ...)                                                                                       \
  do {                                                                                                                 \
    ProfScope ps_((h), (kind));                                                                                        \
    __VA_ARGS__;                                                                                                       \
  } while (0)

void collect_profile(clb_handle *h)
{
  for (auto &p : h->pend) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      h->kernel_ms[p.kind] += ms;
      ++h->timed[p.kind];
    }
    h->ev_pool.push_back(p.a);
    h->ev_pool.push_back(p.b);
  }
  h->pend.clear();
}

} // namespace
