// clb_su2.cu - lphi4SU2U1 (real scalar, complex scalar, SU(2) doublet, U(1) and SU(2) fields)
// behind the libclb200 C ABI.  Compiled without FMA contraction (see build.py): the kernels'
// plain expressions then round in the reference's order.
//
// Schedules restate VelocityVerlet::evolve (velocityverlet.h:51-114) and LeapFrog::evolve / sync
// (leapfrog.h:42-116) with every sector of the model; the second kick of a VV stage and the first
// of the next share one sweep (no field or a(t) change in between), as in the other sectors.

#include "clb_gws.cuh"
#include "clb_handle.cuh"
#include "clb_su2.cuh"
#include "clb_vv.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace clb {

using namespace su2d;

namespace {
constexpr int kSU2Blocks = 148 * 8; // 128-thread grid-stride sweeps
}

struct SU2Sector {
  void *f = nullptr, *p = nullptr; // 22 and 19 x N^3 of double (FP64) or float (FP32 form)
  bool fp32 = false;
  size_t esz = 8;
  State *d_st = nullptr;
  double *d_part = nullptr, *d_sums = nullptr;
  double *d_stage = nullptr; // one FP64 component, for FP32 conversions
  void *ph = nullptr;        // U(1) link phases (12 x N^3, storage type), kept by the drifts
  // kick sweeps: 0 one sweep, 1 two halves, 2 three parts, 3 four parts (S and phi; Phi; A; SU(2))
  // (CLB_SU2_SPLIT sets both forms).  su2_create takes four parts in FP64 and three in FP32, by
  // timing at 384^3 VV2 since the kick forms the field averages from its own products (ms per
  // step): FP64 83.0 whole, 58.3 halves, 45.2 three parts, 40.9 four parts; FP32 44.0, 26.9, 23.3,
  // 23.3 (at 192^3: FP64 9.20, 6.53, 5.10, 4.73; FP32 4.93, 3.18, 2.90, 2.93).  The tangent-linear
  // sweep takes four parts in both (256^3 VV2, ms per tangent step, three / four parts: FP64 37.9,
  // 31.4; FP32 21.5, 19.5).  Every form gives the same state to the last bit.
  int split = 2;
  int tan_split = 3;
  int64_t steps_since_unitarize = 0;
  Params prm{};
  // tangent-linear form: d(state) along the coupling direction tan_cd, active while tangent
  bool tangent = false;
  CoupDot tan_cd{};
  void *df = nullptr, *dp = nullptr;
  TState *d_tst = nullptr;
  double *d_tpart = nullptr, *d_tsums = nullptr;
};

// FP32 form: links re-unitarised every this many steps
constexpr int64_t kUnitarizeEvery = 10;

namespace {
// PITensor.h's GW source for lphi4SU2U1: the singlet S (component 0), the complex scalar phi
// (1, 2) and the U(1) field (7..9, momenta 7..9), in the order scalarSinglet + complexScalar +
// electricU1 + magneticU1; the doublet and the SU(2) field source none.
template <class R> struct SU2GWSource {
  const R *f, *p;
  size_t n3;
  int N;
  R dx, ndxg, rfo2;
  const double *aI;
  __device__ __forceinline__ void operator()(size_t s, int x, int y, int z, int xp, int yp, int zp, R (&P)[6]) const
  {
    using A = Ar<R>;
    const size_t nb[3] = {((size_t)xp * N + y) * N + z, ((size_t)x * N + yp) * N + z, ((size_t)x * N + y) * N + zp};
    const R c = f[s];
    R g[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] = A::sub(f[nb[i]], c) / dx;
#pragma unroll
    for (int k = 0; k < 6; ++k) P[k] = A::mul(g[gw_pair_i(k)], g[gw_pair_j(k)]);
    gw_gauge_tensor<R>(f + n3, f + 2 * n3, f + 7 * n3, p + 7 * n3, n3, nb, s, dx, ndxg, (R)*aI, rfo2, false, P);
  }
};
} // namespace

namespace {

Params su2_params(const clb_handle *h)
{
  Params a{};
  const clb_config &c = h->cfg;
  const clb_model_desc &m = h->md;
  a.N = c.N;
  a.n3 = h->n3;
  a.dx = c.dx;
  a.dx2 = c.dx * c.dx;
  a.inv_dx2 = 1.0 / (c.dx * c.dx);
  a.inv_dx = 1.0 / c.dx;
  a.qG = m.couplings[0];
  a.qH = m.couplings[1];
  a.gC = m.couplings[2];
  a.gD = m.couplings[3];
  a.gS = m.couplings[4];
  a.c4 = m.couplings[5];
  const double rfo = m.fStar / m.omegaStar, rof = m.omegaStar / m.fStar;
  a.rfo2 = rfo * rfo;
  a.rof2 = rof * rof;
  const double fm = m.fStar / m.MPl;
  a.alpha = m.alpha;
  a.fm2 = fm * fm;
  a.dt = c.dt;
  a.inv_n3 = 1.0 / (double)h->n3;
  a.order = gauge_site_order(c.N, true);
  return a;
}

template <class T> void coefs(StateT<T> &s, double al)
{
  s.kA = pow(s.aI, 1 + al);
  s.kB = pow(s.aI, 3 + al);
  s.kB2 = pow(s.aI, 3 + al) / 2;
  s.kG = pow(s.aI, -1 + al);
  s.p3 = pow(s.aSI, al - 3);
  s.p1 = pow(s.aSI, al - 1);
}

// Kick factors (velocityverlet.h:129-162; leapfrog.h:131-170): S (w dt)/2, phi, Phi and SU(2)
// (dt/2) w, U(1) (dt w)/2 on the VV; (w dt) for all on the leapfrog.
Kick vv_kick(double dt, double wa, double wb)
{
  Kick k{};
  const double w[2] = {wa, wb};
  for (int i = 0; i < 2; ++i) {
    k.h[i][0] = w[i] * dt / 2;
    k.h[i][1] = k.h[i][2] = k.h[i][4] = dt / 2 * w[i];
    k.h[i][3] = dt * w[i] / 2;
  }
  return k;
}
Kick lf_kick(double dt, double w)
{
  Kick k{};
  for (int g = 0; g < 5; ++g) k.h[0][g] = w * dt;
  return k;
}

template <class S> void sweep_t(clb_handle *h, int nk, bool rf, bool rp, const Kick &kc)
{
  SU2Sector *u = h->su2;
  const int kind = nk == 0 ? K_U1_REDUCE : K_U1_KICK;
  const S *f = static_cast<const S *>(u->f);
  S *p = static_cast<S *>(u->p);
  // kick sweeps run as two halves (sectors S, phi, Phi, A; then SU(2)) or three parts (S, phi, Phi;
  // A; SU(2)), which hold fewer registers than one sweep over every sector; reduction-only sweeps
  // run whole
#define CLB_SU2K1(NK, RF, RP, SECT)                                                                                     \
  CLB_LAUNCH(h, kind, k_kick<S, NK, RF, RP, SECT><<<kSU2Blocks, 128, 0, h->stream>>>(                                  \
                          f, p, u->prm, kc, u->d_st, u->d_part, static_cast<const S *>(u->ph)))
#define CLB_SU2K(NK, RF, RP)                                                                                            \
  do {                                                                                                                 \
    if (NK > 0 && u->split == 3) {                                                                                     \
      CLB_SU2K1(NK, RF, RP, 5);                                                                                        \
      CLB_SU2K1(NK, RF, RP, 6);                                                                                        \
      CLB_SU2K1(NK, RF, RP, 4);                                                                                        \
      CLB_SU2K1(NK, RF, RP, 2);                                                                                        \
    } else if (NK > 0 && u->split == 2) {                                                                              \
      CLB_SU2K1(NK, RF, RP, 3);                                                                                        \
      CLB_SU2K1(NK, RF, RP, 4);                                                                                        \
      CLB_SU2K1(NK, RF, RP, 2);                                                                                        \
    } else if (NK > 0 && u->split) {                                                                                   \
      CLB_SU2K1(NK, RF, RP, 1);                                                                                        \
      CLB_SU2K1(NK, RF, RP, 2);                                                                                        \
    } else {                                                                                                           \
      CLB_SU2K1(NK, RF, RP, 0);                                                                                        \
    }                                                                                                                  \
  } while (0)
  if (nk == 0) {
    if (rf && rp)
      CLB_SU2K(0, true, true);
    else if (rf)
      CLB_SU2K(0, true, false);
    else
      CLB_SU2K(0, false, true);
  } else if (nk == 1) {
    if (rf && rp)
      CLB_SU2K(1, true, true);
    else if (rp)
      CLB_SU2K(1, false, true);
    else
      CLB_SU2K(1, false, false);
  } else {
    if (rf && rp)
      CLB_SU2K(2, true, true);
    else
      CLB_SU2K(2, false, false);
  }
#undef CLB_SU2K
#undef CLB_SU2K1
}

template <class S> void sweep_tan_t(clb_handle *h, int nk, bool rf, bool rp, const Kick &kc)
{
  SU2Sector *u = h->su2;
  const int kind = nk == 0 ? K_U1_REDUCE : K_U1_KICK;
  const S *f = static_cast<const S *>(u->f), *df = static_cast<const S *>(u->df);
  S *p = static_cast<S *>(u->p), *dp = static_cast<S *>(u->dp);
#define CLB_SU2T1(NK, RF, RP, SECT)                                                                                     \
  CLB_LAUNCH(h, kind,                                                                                                   \
             k_kick_tan<S, NK, RF, RP, SECT><<<kSU2Blocks, 128, 0, h->stream>>>(f, df, p, dp, u->prm, kc, u->d_tst,    \
                                                                                  u->tan_cd, u->d_tpart))
#define CLB_SU2T(NK, RF, RP)                                                                                            \
  do {                                                                                                                 \
    if (NK > 0 && u->tan_split == 3) {                                                                                 \
      CLB_SU2T1(NK, RF, RP, 5);                                                                                        \
      CLB_SU2T1(NK, RF, RP, 6);                                                                                        \
      CLB_SU2T1(NK, RF, RP, 4);                                                                                        \
      CLB_SU2T1(NK, RF, RP, 2);                                                                                        \
    } else if (NK > 0 && u->tan_split == 2) {                                                                          \
      CLB_SU2T1(NK, RF, RP, 3);                                                                                        \
      CLB_SU2T1(NK, RF, RP, 4);                                                                                        \
      CLB_SU2T1(NK, RF, RP, 2);                                                                                        \
    } else if (NK > 0 && u->tan_split) {                                                                               \
      CLB_SU2T1(NK, RF, RP, 1);                                                                                        \
      CLB_SU2T1(NK, RF, RP, 2);                                                                                        \
    } else {                                                                                                           \
      CLB_SU2T1(NK, RF, RP, 0);                                                                                        \
    }                                                                                                                  \
  } while (0)
  if (nk == 0) {
    if (rf && rp)
      CLB_SU2T(0, true, true);
    else if (rf)
      CLB_SU2T(0, true, false);
    else
      CLB_SU2T(0, false, true);
  } else if (nk == 1) {
    if (rf && rp)
      CLB_SU2T(1, true, true);
    else if (rp)
      CLB_SU2T(1, false, true);
    else
      CLB_SU2T(1, false, false);
  } else {
    if (rf && rp)
      CLB_SU2T(2, true, true);
    else
      CLB_SU2T(2, false, false);
  }
#undef CLB_SU2T
#undef CLB_SU2T1
}

void sweep(clb_handle *h, int nk, bool rf, bool rp, const Kick &kc)
{
  SU2Sector *u = h->su2;
  if (u->tangent) {
    if (u->fp32)
      sweep_tan_t<float>(h, nk, rf, rp, kc);
    else
      sweep_tan_t<double>(h, nk, rf, rp, kc);
  } else if (u->fp32) {
    sweep_t<float>(h, nk, rf, rp, kc);
  } else {
    sweep_t<double>(h, nk, rf, rp, kc);
  }
}

template <class S> void drift_tan_t(clb_handle *h, double w, bool lf)
{
  SU2Sector *u = h->su2;
  CLB_LAUNCH(h, K_U1_DRIFT,
             k_drift_tan<S><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<S *>(u->f), static_cast<S *>(u->df),
                                                               static_cast<const S *>(u->p), static_cast<const S *>(u->dp),
                                                               u->prm, w, lf ? 1 : 0, u->d_tst, u->tan_cd));
}

void drift(clb_handle *h, double w, bool lf, double dtd = -1.0)
{
  if (dtd < 0) dtd = h->cfg.dt;
  SU2Sector *u = h->su2;
  if (u->tangent) {
    if (u->fp32)
      drift_tan_t<float>(h, w, lf);
    else
      drift_tan_t<double>(h, w, lf);
    return;
  }
  if (u->fp32)
    CLB_LAUNCH(h, K_U1_DRIFT, k_drift<float><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<float *>(u->f),
                                                                                 static_cast<const float *>(u->p),
                                                                                 u->prm, w, lf ? 1 : 0, u->d_st,
                                                                                 static_cast<float *>(u->ph), dtd));
  else
    CLB_LAUNCH(h, K_U1_DRIFT, k_drift<double><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<double *>(u->f),
                                                                                  static_cast<const double *>(u->p),
                                                                                  u->prm, w, lf ? 1 : 0, u->d_st,
                                                                                  static_cast<double *>(u->ph), dtd));
}

// FP32 form: after the drift of every kUnitarizeEvery-th step the links are projected back to
// unit quaternions.
void step_done(clb_handle *h)
{
  SU2Sector *u = h->su2;
  if (!u->fp32) return;
  if (++u->steps_since_unitarize < kUnitarizeEvery) return;
  u->steps_since_unitarize = 0;
  if (u->tangent)
    CLB_LAUNCH(h, K_U1_DRIFT, k_unitarize_tan<float><<<kSU2Blocks, 256, 0, h->stream>>>(
                                  static_cast<float *>(u->f), static_cast<float *>(u->df), h->n3));
  else
    CLB_LAUNCH(h, K_U1_DRIFT, k_unitarize<float><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<float *>(u->f), h->n3));
}

void tail(clb_handle *h, uint32_t flags, bool reduced, double w = 0, double w2 = 0, int64_t hist_row = -1,
          double fa = 0, double fb = 0)
{
  SU2Sector *u = h->su2;
  TailOp op{flags, reduced ? kSU2Blocks : 0, w, w2, hist_row >= 0 ? h->d_hist : nullptr, hist_row, fa, fb};
  if (u->tangent)
    CLB_LAUNCH(h, K_TAIL, su2d::k_tail<Tan<double>><<<1, 256, 0, h->stream>>>(u->d_tpart, op, u->d_tst, u->prm));
  else
    CLB_LAUNCH(h, K_TAIL, su2d::k_tail<double><<<1, 256, 0, h->stream>>>(u->d_part, op, u->d_st, u->prm));
}

// Value part of the tangent-form scalar state.
State values_of(const TState &t)
{
  State s{};
  zip_state(s, t, [](double &x, const Tan<double> &y) { x = y.v; });
  s.status = t.status;
  return s;
}

int check(clb_handle *h, const char *where)
{
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  collect_profile(h);
  SU2Sector *u = h->su2;
  State s;
  if (u->tangent) {
    // the tangent form advances d_tst; its value part is the state the plain calls read
    TState t;
    e = cudaMemcpy(&t, u->d_tst, sizeof(t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
      s = values_of(t);
      e = cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice);
    }
  } else {
    e = cudaMemcpy(&s, u->d_st, sizeof(s), cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  if (s.status != 0) return h->fail(CLB_ENONFINITE, std::string(where) + ": a volume average or a(t) is not finite");
  return CLB_OK;
}

} // namespace

__attribute__((visibility("hidden"))) int su2_create(clb_handle *h)
{
  SU2Sector *u = new SU2Sector();
  h->su2 = u;
  h->NS = NF;
  u->prm = su2_params(h);
  u->fp32 = h->cfg.precision == CLB_PREC_FP32_SPLIT;
  u->esz = u->fp32 ? sizeof(float) : sizeof(double);
  u->split = u->fp32 ? 2 : 3;
  if (const char *env = std::getenv("CLB_SU2_SPLIT")) {
    u->split = std::max(0, std::min(3, std::atoi(env)));
    u->tan_split = u->split;
  }
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc(&u->f, NF * h->n3 * u->esz) == cudaSuccess;
  ok = ok && cudaMalloc(&u->p, NP * h->n3 * u->esz) == cudaSuccess;
  ok = ok && cudaMemset(u->f, 0, NF * h->n3 * u->esz) == cudaSuccess;
  ok = ok && cudaMemset(u->p, 0, NP * h->n3 * u->esz) == cudaSuccess;
  ok = ok && cudaMalloc(&u->ph, 12 * h->n3 * u->esz) == cudaSuccess;
  if (u->fp32) ok = ok && cudaMalloc(&u->d_stage, h->n3 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_st, sizeof(State)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_part, (size_t)kSU2Blocks * kMeas * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_sums, kMeas * sizeof(double)) == cudaSuccess;
  ok = ok && cudaEventCreate(&h->ev_call[0]) == cudaSuccess && cudaEventCreate(&h->ev_call[1]) == cudaSuccess;
  if (!ok) return CLB_ENOMEM;
  State s{};
  s.aI = s.aSI = s.aIM = 1.0;
  coefs(s, h->md.alpha);
  return cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice) == cudaSuccess ? CLB_OK : CLB_ECUDA;
}

namespace {
void free_tangent(SU2Sector *u)
{
  for (void *q : {u->df, u->dp, (void *)u->d_tst, (void *)u->d_tpart, (void *)u->d_tsums})
    if (q) cudaFree(q);
  u->df = u->dp = nullptr;
  u->d_tst = nullptr;
  u->d_tpart = u->d_tsums = nullptr;
  u->tangent = false;
}
} // namespace

__attribute__((visibility("hidden"))) void su2_destroy(clb_handle *h)
{
  SU2Sector *u = h->su2;
  if (!u) return;
  free_tangent(u);
  for (void *q : {(void *)u->f, (void *)u->p, (void *)u->d_st, (void *)u->d_part, (void *)u->d_sums, (void *)u->d_stage,
                  u->ph})
    if (q) cudaFree(q);
  delete u;
  h->su2 = nullptr;
}

__attribute__((visibility("hidden"))) int su2_set_state(clb_handle *h, const double *fields, const double *momenta,
                                                        const clb_scalefactor *sf)
{
  SU2Sector *u = h->su2;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  free_tangent(u); // a new state ends the tangent-linear form
  if (!u->fp32) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(u->f, fields, NF * h->n3 * sizeof(double), cudaMemcpyDefault, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(u->p, momenta, NP * h->n3 * sizeof(double), cudaMemcpyDefault, h->stream);
  } else {
    // one component at a time through the FP64 staging buffer
    for (int c = 0; c < NF + NP && e == cudaSuccess; ++c) {
      const double *src = c < NF ? fields + (size_t)c * h->n3 : momenta + (size_t)(c - NF) * h->n3;
      float *dst = static_cast<float *>(c < NF ? u->f : u->p) + (size_t)(c < NF ? c : c - NF) * h->n3;
      e = cudaMemcpyAsync(u->d_stage, src, h->n3 * sizeof(double), cudaMemcpyDefault, h->stream);
      if (e == cudaSuccess) k_convert<double, float><<<kSU2Blocks, 256, 0, h->stream>>>(u->d_stage, dst, h->n3);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
  }
  if (e == cudaSuccess) {
    // the link phases of the new A
    if (u->fp32)
      k_phases<float><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<const float *>(u->f), static_cast<float *>(u->ph), u->prm);
    else
      k_phases<double><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<const double *>(u->f), static_cast<double *>(u->ph), u->prm);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  u->steps_since_unitarize = 0;
  State s{};
  s.aI = s.aSI = s.aIM = 1.0;
  if (sf) {
    s.aI = sf->aI;
    s.aSI = sf->aSI;
    s.aIM = sf->aIM;
    s.aDotI = sf->aDotI;
    s.aDotSI = sf->aDotSI;
    s.aDotSIM = sf->aDotSIM;
  }
  coefs(s, h->md.alpha);
  if ((e = cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice)) != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  h->has_state = true;
  h->initialized = false;
  h->synced = true;
  return CLB_OK;
}

__attribute__((visibility("hidden"))) int su2_get_state(clb_handle *h, double *fields, double *momenta,
                                                        clb_scalefactor *sf)
{
  SU2Sector *u = h->su2;
  State s;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (!u->fp32) {
    if (e == cudaSuccess && fields) e = cudaMemcpyAsync(fields, u->f, NF * h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && momenta) e = cudaMemcpyAsync(momenta, u->p, NP * h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  } else {
    for (int c = 0; c < NF + NP && e == cudaSuccess; ++c) {
      double *dst = c < NF ? (fields ? fields + (size_t)c * h->n3 : nullptr) : (momenta ? momenta + (size_t)(c - NF) * h->n3 : nullptr);
      if (!dst) continue;
      const float *src = static_cast<const float *>(c < NF ? u->f : u->p) + (size_t)(c < NF ? c : c - NF) * h->n3;
      k_convert<float, double><<<kSU2Blocks, 256, 0, h->stream>>>(src, u->d_stage, h->n3);
      e = cudaMemcpyAsync(dst, u->d_stage, h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&s, u->d_st, sizeof(s), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_get_state");
  if (sf) {
    sf->aI = s.aI;
    sf->aSI = s.aSI;
    sf->aIM = s.aIM;
    sf->aDotI = s.aDotI;
    sf->aDotSI = s.aDotSI;
    sf->aDotSIM = s.aDotSIM;
  }
  return CLB_OK;
}

__attribute__((visibility("hidden"))) int su2_initialize(clb_handle *h, int32_t correct_adot)
{
  sweep(h, 0, true, true, Kick{});
  uint32_t fl = T_STORE_ALL;
  if (h->cfg.expansion && correct_adot == 1 && !h->fb) fl |= T_CORRECT_ADOT; // modelinitializer.h:74-80
  if (h->cfg.expansion && h->cfg.evolver == CLB_LF && correct_adot != CLB_INIT_RESTART) fl |= T_LF_CTOR;
  tail(h, fl, true);
  h->synced = !(correct_adot == CLB_INIT_RESTART && h->cfg.evolver == CLB_LF); // leapfrog.h:30-31
  return check(h, "clb_initialize");
}

void gw_kick_step(clb_handle *h);
void gw_drift(clb_handle *h);
void gw_sync(clb_handle *h);

__attribute__((visibility("hidden"))) bool su2_tangent_active(const clb_handle *h) { return h->su2->tangent; }

// The GW kick (weight w of dt) with the lphi4SU2U1 source, at the current fields, momenta and a_I.
__attribute__((visibility("hidden"))) void su2_gw_kick(clb_handle *h, double w)
{
  SU2Sector *u = h->su2;
  GWSector *g = h->gw;
  const double r = h->md.fStar / h->md.omegaStar; // pow<2>(fStar / omegaStar)
  const double inv_dx2 = 1.0 / (h->cfg.dx * h->cfg.dx), hd = w * h->cfg.dt;
  const double ndxg = -u->prm.dx * u->prm.gC;     // the phase of Site::phaseC
  auto go = [&](auto zero) {
    using R = decltype(zero);
    const SU2GWSource<R> src{static_cast<const R *>(u->f), static_cast<const R *>(u->p), h->n3, h->N, (R)h->cfg.dx,
                             (R)ndxg, (R)(r * r), &u->d_st->aI};
    CLB_LAUNCH(h, K_GW, (k_gw_kick<R, SU2GWSource<R>><<<kGWBlocks, 256, 0, h->stream>>>(
                            static_cast<const R *>(g->u), static_cast<R *>(g->pi), h->N, inv_dx2, hd, &u->d_st->kA, src)));
  };
  if (u->fp32) go(0.0f);
  else go(0.0);
}

// The GW drift with the a_SI of the matter step just taken (State::p3 = pow(a_SI, alpha - 3) on the
// VV and the leapfrog).
__attribute__((visibility("hidden"))) void su2_gw_drift(clb_handle *h)
{
  SU2Sector *u = h->su2;
  GWSector *g = h->gw;
  const size_t n = 5 * h->n3;
  const bool pv = is_pv(h->cfg.evolver); // p3 is then a_I's: the drift forms a_SI's
  if (u->fp32)
    CLB_LAUNCH(h, K_GW, launch_gw_drift<float>(static_cast<float *>(g->u), static_cast<const float *>(g->pi), n,
                                               h->cfg.dt, &u->d_st->p3, &u->d_st->aSI, h->md.alpha, pv, h->stream));
  else
    CLB_LAUNCH(h, K_GW, launch_gw_drift<double>(static_cast<double *>(g->u), static_cast<const double *>(g->pi), n,
                                                h->cfg.dt, &u->d_st->p3, &u->d_st->aSI, h->md.alpha, pv, h->stream));
}

namespace {
// VelocityVerlet::evolve over nsteps with merged kicks; the history rows start at row0.
void vv_steps(clb_handle *h, int64_t nsteps, int64_t row0)
{
  const double dt = h->cfg.dt;
  const bool ex = h->cfg.expansion != 0;
  const std::vector<double> &ws = h->ws;
  const size_t P = ws.size(), S = 2 * P - 1;
  auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
  const int64_t total = nsteps * (int64_t)S;
  const double w0 = wof(0);
  if (ex) tail(h, T_VV_KICK_HALF, false, 0, w0);
  sweep(h, 1, false, ex, vv_kick(dt, w0, 0.0));
  if (ex) tail(h, T_STORE_PI2_I | T_VV_DRIFT, true, 0, w0);
  for (int64_t k = 0; k < total; ++k) {
    const size_t i = (size_t)(k % (int64_t)S);
    const double w = wof(i);
    const bool more = k + 1 < total;
    const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
    drift(h, w, false);
    if (i + 1 == S) step_done(h);
    sweep(h, more ? 2 : 1, ex, ex, vv_kick(dt, w, wn));
    if (ex) {
      uint32_t fl = T_STORE_FIELDS | T_STORE_PI2_I | T_VV_KICK_ONE;
      if (more) fl |= T_VV_KICK_HALF | T_STORE_PI2_B | T_VV_DRIFT;
      tail(h, fl, true, w, wn, i + 1 == S ? row0 + k / (int64_t)S : -1);
    }
  }
}

} // namespace

__attribute__((visibility("hidden"))) int su2_evolve(clb_handle *h, int64_t nsteps)
{
  const double dt = h->cfg.dt;
  const bool ex = h->cfg.expansion != 0;
  cudaEventRecord(h->ev_call[0], h->stream);
  if (h->fb) {
    // fixed background (velocityverlet.h:74-118, leapfrog.h:55-89, positionverlet.h:45-99 with the
    // fixed branches): a from the closed form at the reference's stage times, no a-kicks and no
    // averages; the VV a-drift leaves aSI, which its field drifts read, as it was
    const double t0 = h->cfg.t0;
    const std::vector<double> &ws = h->ws;
    const size_t P = ws.size(), S = 2 * P - 1;
    auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
    if (h->cfg.evolver == CLB_LF) {
      for (int64_t s = 0; s < nsteps; ++s) {
        if (h->gw) gw_kick_step(h); // evolver.h:102-124, as in the self-consistent leapfrog
        sweep(h, 1, false, false, lf_kick(dt, h->synced ? 0.5 : 1.0));
        const double tm = h->fb_t - t0;
        tail(h, T_FB_AIM | T_FB_AI | T_FB_ASI, false, 0, 0, -1, h->fb_a(tm + dt), h->fb_a(tm + dt / 2.0));
        drift(h, 1.0, true);
        if (h->gw) gw_drift(h);
        step_done(h);
        h->fb_t += dt;
        h->synced = false;
      }
    } else if (is_pv(h->cfg.evolver)) {
      tail(h, T_PV_MODE, false);
      for (int64_t s = 0; s < nsteps; ++s) {
        if (h->gw) gw_kick_step(h); // evolver.h:102-124
        double tc = h->fb_t - t0;
        for (size_t i = 0; i < S; ++i) {
          const double w = wof(i);
          drift(h, w, false, dt / 2);
          tail(h, T_PV_MODE | T_FB_PV_HALF, false, 0, 0, -1, 0.0, h->fb_a(tc + w * dt / 2.0));
          sweep(h, 1, false, false, lf_kick(dt, w));
          tail(h, T_PV_MODE | T_FB_AI, false, 0, 0, -1, h->fb_a(tc + w * dt));
          drift(h, w, false, dt / 2);
          tc += dt * w;
        }
        if (h->gw) gw_drift(h);
        step_done(h);
        h->fb_t += dt;
      }
    } else {
      auto vv_fb = [&](int64_t n) {
        const int64_t total = n * (int64_t)S;
        sweep(h, 1, false, false, vv_kick(dt, wof(0), 0.0));
        double tc = h->fb_t - t0;
        for (int64_t k = 0; k < total; ++k) {
          const size_t i = (size_t)(k % (int64_t)S);
          const double w = wof(i);
          const bool more = k + 1 < total;
          const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
          tail(h, T_FB_AIM | T_FB_AI, false, 0, 0, -1, h->fb_a(tc + w * dt));
          drift(h, w, false);
          if (i + 1 == S) { step_done(h); }
          sweep(h, more ? 2 : 1, false, false, vv_kick(dt, w, wn));
          tc += dt * w;
          if (i + 1 == S) {
            h->fb_t += dt;
            tc = h->fb_t - t0;
          }
        }
      };
      if (h->gw) {
        // one step at a time, as in the self-consistent VV with GWs
        for (int64_t s = 0; s < nsteps; ++s) {
          gw_kick_step(h);
          vv_fb(1);
          gw_drift(h);
        }
      } else {
        vv_fb(nsteps);
      }
    }
  } else if (h->cfg.evolver == CLB_LF) {
    // With GWs (evolver.h:102-124): a GW kick before each step's kick (the step's fields, the
    // momenta half a step back, a_I) and a GW drift after its drift (its a_SI)
    if (h->gw) gw_kick_step(h);
    sweep(h, 1, false, ex, lf_kick(dt, h->synced ? 0.5 : 1.0));
    if (ex) tail(h, T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true);
    for (int64_t s = 0; s < nsteps; ++s) {
      drift(h, 1.0, true);
      if (h->gw) gw_drift(h);
      step_done(h);
      if (s + 1 < nsteps) {
        if (h->gw) gw_kick_step(h);
        sweep(h, 1, ex, ex, lf_kick(dt, 1.0));
        if (ex) tail(h, T_STORE_FIELDS | T_HIST_EARLY | T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true, 0, 0, s);
      } else if (ex) {
        sweep(h, 0, true, false, Kick{});
        tail(h, T_STORE_FIELDS | T_HIST_EARLY, true, 0, 0, s);
      }
    }
    h->synced = false;
  } else if (is_pv(h->cfg.evolver)) {
    // PositionVerlet::evolve (positionverlet.h:45-99), as for lphi4U1: drift(dt/2 w), kick(w dt)
    // at the half-step a with the half-step field sums and the momentum sums, the a-kick and a
    // half-drifts in the tails, drift(dt/2 w); a field-sum sweep ends each step
    const std::vector<double> &ws = h->ws;
    const size_t P = ws.size(), S = 2 * P - 1;
    auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
    // With GWs (evolver.h:102-124): the GW kick before each step (a_I before the step's first a
    // half-drift) and the GW drift after its last field drift (its a_SI), both before the tail that
    // starts the next step's a half-drift.
    const double w0 = wof(0);
    if (h->gw) gw_kick_step(h);
    tail(h, T_PV_MODE | (ex ? T_PV_DRIFT_A1 : 0u), false, 0, w0);
    for (int64_t s = 0; s < nsteps; ++s)
      for (size_t i = 0; i < S; ++i) {
        const double w = wof(i);
        const bool last = i + 1 == S;
        drift(h, w, false, dt / 2);
        sweep(h, 1, ex, ex, lf_kick(dt, w));
        if (ex)
          tail(h, T_PV_MODE | T_PV_STORE_SI | T_PV_STORE_PI2 | T_PV_KICK | T_PV_DRIFT_A2 | (last ? 0u : T_PV_DRIFT_A1),
               true, w, last ? 0.0 : wof(i + 1));
        drift(h, w, false, dt / 2);
        if (last && h->gw) {
          gw_drift(h);
          if (s + 1 < nsteps) gw_kick_step(h);
        }
        if (last) {
          step_done(h);
          if (ex) {
            sweep(h, 0, true, false, Kick{});
            tail(h, T_PV_MODE | T_STORE_FIELDS | (s + 1 < nsteps ? T_PV_DRIFT_A1 : 0u), true, 0, w0, s);
          }
        }
      }
  } else if (h->gw) {
    // the GW leapfrog around each matter step (evolver.h:102-124): its kick reads the gauge
    // momenta at integer time, which the merged sweep between two steps never stores, so the steps
    // run one by one (the schedule of one-step clb_evolve calls)
    for (int64_t s = 0; s < nsteps; ++s) {
      gw_kick_step(h);
      vv_steps(h, 1, s);
      gw_drift(h);
    }
  } else {
    vv_steps(h, nsteps, 0);
  }
  cudaEventRecord(h->ev_call[1], h->stream);
  const int r = check(h, "clb_evolve");
  float ms = 0;
  if (cudaEventElapsedTime(&ms, h->ev_call[0], h->ev_call[1]) == cudaSuccess) h->last_evolve_ms = ms;
  return r;
}

__attribute__((visibility("hidden"))) int su2_sync(clb_handle *h)
{
  if (h->gw) gw_sync(h); // evolver.h:134-137, before the matter sync
  if (h->cfg.evolver == CLB_LF && !h->synced) {
    sweep(h, 1, false, h->cfg.expansion != 0 && !h->fb, lf_kick(h->cfg.dt, 0.5));
    if (h->cfg.expansion && !h->fb) tail(h, T_STORE_PI2_I | T_LF_SYNC, true);
  }
  if (h->fb) tail(h, T_FB_ADOT, false, 0, 0, -1, 0.0, h->fb_adot(h->fb_t - h->cfg.t0));
  h->synced = true;
  return check(h, "clb_sync");
}

// Measurement (energiesmeasurer.h:45-122 and the sector measurers): energies E_kin, E_grad of S,
// phi, Phi; E_el, E_mag of U(1) and SU(2); the three potential terms; E_tot.  Means rows: S,
// sqrt2 Re phi, sqrt2 Im phi, |phi|, |Phi|, U(1) |E| |B|, SU(2) |E| |B|.  Both Gauss checks.
// Energies::rho's setAllAverages side effect (energies.h:219) is applied to the cached averages.
__attribute__((visibility("hidden"))) int su2_measure(clb_handle *h, double e0, clb_measurement *m)
{
  SU2Sector *u = h->su2;
  State s;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&s, u->d_st, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  const double al = h->md.alpha;
  const double am = std::pow(s.aI, al - 3), ag = std::pow(s.aI, al - 1);
  if (u->fp32)
    CLB_LAUNCH(h, K_MEASURE, su2d::k_measure<float><<<kSU2Blocks, 128, 0, h->stream>>>(
                                 static_cast<const float *>(u->f), static_cast<const float *>(u->p), u->prm, am, ag, u->d_part));
  else
    CLB_LAUNCH(h, K_MEASURE, su2d::k_measure<double><<<kSU2Blocks, 128, 0, h->stream>>>(
                                 static_cast<const double *>(u->f), static_cast<const double *>(u->p), u->prm, am, ag, u->d_part));
  CLB_LAUNCH(h, K_MEASURE, k_sum_partials<kMeas><<<1, 256, 0, h->stream>>>(u->d_part, kSU2Blocks, u->d_sums));
  double v[kMeas];
  e = cudaMemcpyAsync(v, u->d_sums, sizeof(v), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  collect_profile(h);
  const double inv = u->prm.inv_n3;
  for (double &x : v) x *= inv;
  // setAllAverages
  for (int g = 0; g < 5; ++g) s.pi2[g] = s.pi2SI[g] = v[g];
  s.g2S = v[5];
  s.g2C = v[6];
  s.g2D = v[7];
  s.b2A = v[8];
  s.b2G = v[9];
  s.potI = v[10];
  std::memset(m, 0, sizeof(*m));
  const En E = energies_of(s, u->prm);
  const double en[10] = {E.ks, E.gs, E.kc, E.gc, E.kd, E.gd, E.ea, E.ba, E.eg, E.bg};
  double Etot = 0;
  int k = 0;
  for (int i = 0; i < 10; ++i) {
    m->energies[k++] = en[i];
    Etot += en[i];
  }
  for (int i = 0; i < 3; ++i) {
    m->energies[k++] = v[11 + i];
    Etot += v[11 + i];
  }
  m->energies[k++] = Etot;
  m->n_energies = k;
  if (h->cfg.expansion) {
    const double LHS = s.aDotI * s.aDotI;
    const double RHS = std::pow(s.aI, 2 * al + 2) / 3. * u->prm.fm2 * rho_of(s, u->prm);
    m->friedmann[0] = (LHS - RHS) / (LHS + RHS);
    m->friedmann[1] = LHS;
    m->friedmann[2] = RHS;
  } else {
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  }
  if ((e = cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice)) != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  if (u->tangent) {
    // the same refresh of the cached values in the tangent form (tangents kept: the refreshed
    // averages differ from the cached ones by the reduction order only)
    TState t;
    e = cudaMemcpy(&t, u->d_tst, sizeof(t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
      zip_state(t, s, [](Tan<double> &x, const double &y) { x.v = y; });
      e = cudaMemcpy(u->d_tst, &t, sizeof(t), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  }
  for (int r = 0; r < 7; ++r) {
    const double a1 = v[14 + 4 * r], a2 = v[15 + 4 * r], b1 = v[16 + 4 * r], b2 = v[17 + 4 * r];
    const double r1 = a2 - a1 * a1, rr = b2 - b1 * b1;
    m->means[r][0] = a1;
    m->means[r][1] = b1;
    m->means[r][2] = a2;
    m->means[r][3] = b2;
    m->means[r][4] = r1 > 0 ? std::sqrt(r1) : 0;
    m->means[r][5] = rr > 0 ? std::sqrt(rr) : 0;
  }
  m->n_means = 7;
  m->gauss_u1[0] = v[42] / v[43];
  m->gauss_u1[1] = v[45];
  m->gauss_u1[2] = v[44];
  double gs[4] = {0, 0, 0, 0};
  for (int b = 0; b < 3; ++b)
    for (int q = 0; q < 4; ++q) gs[q] = b == 0 ? v[46 + 4 * b + q] : gs[q] + v[46 + 4 * b + q];
  m->gauss_su2[0] = gs[0] / gs[1];
  m->gauss_su2[1] = gs[3];
  m->gauss_su2[2] = gs[2];
  m->aI = s.aI;
  m->aDotI = s.aDotI;
  m->hubble = s.aDotI / s.aI;
  return CLB_OK;
}

// Device array of one state component (clb_spectrum): which 0 fields (22), 1 momenta (19); gauge
// tells whether the component belongs to the U(1) or SU(2) field.
__attribute__((visibility("hidden"))) const double *su2_component(clb_handle *h, int which, int comp, bool *gauge)
{
  SU2Sector *u = h->su2;
  if (comp < 0 || comp >= (which == 0 ? NF : NP)) return nullptr;
  *gauge = comp >= 7;
  if (!u->fp32) return static_cast<const double *>(which == 0 ? u->f : u->p) + (size_t)comp * h->n3;
  // FP32 form: the component in FP64 in the staging buffer (ordered on the handle's stream)
  const float *src = static_cast<const float *>(which == 0 ? u->f : u->p) + (size_t)comp * h->n3;
  k_convert<float, double><<<kSU2Blocks, 256, 0, h->stream>>>(src, u->d_stage, h->n3);
  return u->d_stage;
}

// ---- tangent-linear form -------------------------------------------------------------------------
namespace {
// n components of N^3 FP64 host values into device storage of either form (and back).
cudaError_t upload_comps(clb_handle *h, void *dst, const double *src, int n)
{
  SU2Sector *u = h->su2;
  cudaError_t e = cudaSuccess;
  if (!u->fp32) {
    if (src) return cudaMemcpyAsync(dst, src, n * h->n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    return cudaMemsetAsync(dst, 0, n * h->n3 * sizeof(double), h->stream);
  }
  if (!src) return cudaMemsetAsync(dst, 0, n * h->n3 * sizeof(float), h->stream);
  for (int c = 0; c < n && e == cudaSuccess; ++c) {
    e = cudaMemcpyAsync(u->d_stage, src + (size_t)c * h->n3, h->n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      k_convert<double, float><<<kSU2Blocks, 256, 0, h->stream>>>(u->d_stage, static_cast<float *>(dst) + (size_t)c * h->n3, h->n3);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  }
  return e;
}
cudaError_t download_comps(clb_handle *h, double *dst, const void *src, int n)
{
  SU2Sector *u = h->su2;
  cudaError_t e = cudaSuccess;
  if (!dst) return e;
  if (!u->fp32) return cudaMemcpyAsync(dst, src, n * h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  for (int c = 0; c < n && e == cudaSuccess; ++c) {
    k_convert<float, double><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<const float *>(src) + (size_t)c * h->n3,
                                                                 u->d_stage, h->n3);
    e = cudaMemcpyAsync(dst + (size_t)c * h->n3, u->d_stage, h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  }
  return e;
}
} // namespace

// Starts the tangent-linear form: from here clb_initialize, clb_evolve and clb_sync also advance
// the derivative of the state along couplings_dot (the six couplings' derivatives), starting from
// the given start-state tangent (null: zero).
__attribute__((visibility("hidden"))) int su2_tangent_begin(clb_handle *h, const double *couplings_dot, int32_t n,
                                                            const double *fields_dot, const double *momenta_dot,
                                                            const clb_scalefactor *sf_dot)
{
  SU2Sector *u = h->su2;
  if (is_pv(h->cfg.evolver))
    return h->fail(CLB_EUNSUPPORTED, "clb_tangent_begin: the tangent-linear form covers the LF and VV evolvers");
  if (h->fb) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_begin: the tangent-linear form covers the self-consistent expansion");
  if (h->gw) return h->fail(CLB_EUNSUPPORTED, "clb_tangent_begin: the tangent-linear form runs without the GW sector");
  if (n < 0 || n > 6 || (n > 0 && !couplings_dot))
    return h->fail(CLB_EINVAL, "clb_tangent_begin: up to 6 coupling derivatives");
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_tangent_begin");
  free_tangent(u);
  bool ok = cudaMalloc(&u->df, NF * h->n3 * u->esz) == cudaSuccess && cudaMalloc(&u->dp, NP * h->n3 * u->esz) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_tst, sizeof(TState)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_tpart, (size_t)kSU2Blocks * 2 * kRed * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_tsums, 2 * kRed * sizeof(double)) == cudaSuccess;
  if (!ok) {
    free_tangent(u);
    return h->fail(CLB_ENOMEM, "clb_tangent_begin: tangent storage does not fit");
  }
  if ((e = upload_comps(h, u->df, fields_dot, NF)) != cudaSuccess || (e = upload_comps(h, u->dp, momenta_dot, NP)) != cudaSuccess) {
    free_tangent(u);
    return h->cuda_fail(e, "clb_tangent_begin");
  }
  State s;
  if ((e = cudaMemcpy(&s, u->d_st, sizeof(s), cudaMemcpyDeviceToHost)) != cudaSuccess) {
    free_tangent(u);
    return h->cuda_fail(e, "clb_tangent_begin");
  }
  TState t{};
  zip_state(t, s, [](Tan<double> &x, const double &y) { x = Tan<double>(y, 0.0); });
  if (sf_dot) {
    t.aI.d = sf_dot->aI;
    t.aSI.d = sf_dot->aSI;
    t.aIM.d = sf_dot->aIM;
    t.aDotI.d = sf_dot->aDotI;
    t.aDotSI.d = sf_dot->aDotSI;
    t.aDotSIM.d = sf_dot->aDotSIM;
  }
  coefs(t, h->md.alpha);
  t.status = s.status;
  if ((e = cudaMemcpy(u->d_tst, &t, sizeof(t), cudaMemcpyHostToDevice)) != cudaSuccess) {
    free_tangent(u);
    return h->cuda_fail(e, "clb_tangent_begin");
  }
  for (int k = 0; k < 6; ++k) u->tan_cd.v[k] = k < n ? couplings_dot[k] : 0.0;
  u->tangent = true;
  return CLB_OK;
}

__attribute__((visibility("hidden"))) int su2_tangent_get_state(clb_handle *h, double *fields_dot, double *momenta_dot,
                                                                clb_scalefactor *sf_dot)
{
  SU2Sector *u = h->su2;
  if (!u->tangent) return h->fail(CLB_ESTATE, "clb_tangent_get_state: call clb_tangent_begin first");
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = download_comps(h, fields_dot, u->df, NF);
  if (e == cudaSuccess) e = download_comps(h, momenta_dot, u->dp, NP);
  TState t;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&t, u->d_tst, sizeof(t), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_tangent_get_state");
  if (sf_dot) {
    sf_dot->aI = t.aI.d;
    sf_dot->aSI = t.aSI.d;
    sf_dot->aIM = t.aIM.d;
    sf_dot->aDotI = t.aDotI.d;
    sf_dot->aDotSI = t.aDotSI.d;
    sf_dot->aDotSIM = t.aDotSIM.d;
  }
  return CLB_OK;
}

// The 11 energies (E_kin, E_grad of S, phi, Phi; E_el, E_mag of U(1), SU(2); V) at the current
// state with their tangents, from one tangent reduction sweep.
static int tangent_energies(clb_handle *h, const char *where, Tan<double> (&en)[11])
{
  SU2Sector *u = h->su2;
  if (!u->tangent) return h->fail(CLB_ESTATE, std::string(where) + ": call clb_tangent_begin first");
  if (h->cfg.evolver == CLB_LF && !h->synced) return h->fail(CLB_ESTATE, std::string(where) + ": call clb_sync first");
  sweep(h, 0, true, true, Kick{});
  CLB_LAUNCH(h, K_MEASURE, k_sum_partials<2 * kRed><<<1, 256, 0, h->stream>>>(u->d_tpart, kSU2Blocks, u->d_tsums));
  double v[2 * kRed];
  TState t;
  cudaError_t e = cudaMemcpyAsync(v, u->d_tsums, sizeof(v), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&t, u->d_tst, sizeof(t), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  collect_profile(h);
  using T = Tan<double>;
  const double inv = u->prm.inv_n3;
  auto av = [&](int k) { return T(v[k] * inv, v[kRed + k] * inv); };
  for (int g = 0; g < 5; ++g) t.pi2[g] = av(g);
  t.g2S = av(5);
  t.g2C = av(6);
  t.g2D = av(7);
  t.b2A = av(8);
  t.b2G = av(9);
  t.potI = av(10);
  const EnT<T> E = energies_of(t, u->prm);
  const T all[11] = {E.ks, E.gs, E.kc, E.gc, E.kd, E.gd, E.ea, E.ba, E.eg, E.bg, t.potI};
  for (int k = 0; k < 11; ++k) en[k] = all[k];
  return CLB_OK;
}

__attribute__((visibility("hidden"))) int su2_tangent_energies(clb_handle *h, double *E, double *dE)
{
  Tan<double> en[11];
  const int r = tangent_energies(h, "clb_tangent_energies", en);
  if (r != CLB_OK) return r;
  for (int k = 0; k < 11; ++k) {
    if (E) E[k] = en[k].v;
    if (dE) dE[k] = en[k].d;
  }
  return CLB_OK;
}

// O = sum_k w_k E_k / E_tot over the 11 energies and its derivative along the tangent.
__attribute__((visibility("hidden"))) int su2_tangent_observable(clb_handle *h, const double *w, int32_t nw, double *obs,
                                                                 double *dobs)
{
  if (nw < 0 || nw > 11 || (nw > 0 && !w)) return h->fail(CLB_EINVAL, "clb_tangent_observable: up to 11 energy weights");
  using T = Tan<double>;
  T en[11];
  const int r = tangent_energies(h, "clb_tangent_observable", en);
  if (r != CLB_OK) return r;
  T Et(0.0), Ew(0.0);
  for (int k = 0; k < 11; ++k) {
    Et = Et + en[k];
    if (k < nw) Ew = Ew + w[k] * en[k];
  }
  const T O = Ew / Et;
  if (obs) *obs = O.v;
  if (dobs) *dobs = O.d;
  return CLB_OK;
}

__attribute__((visibility("hidden"))) int su2_tangent_end(clb_handle *h)
{
  SU2Sector *u = h->su2;
  // the tangent form's kicks form the link phases themselves; the plain kicks read them again
  if (u->fp32)
    k_phases<float><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<const float *>(u->f), static_cast<float *>(u->ph), u->prm);
  else
    k_phases<double><<<kSU2Blocks, 256, 0, h->stream>>>(static_cast<const double *>(u->f), static_cast<double *>(u->ph), u->prm);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  free_tangent(u);
  return e == cudaSuccess ? CLB_OK : h->cuda_fail(e, "clb_tangent_end");
}

// Tangent of one state component (clb_tangent_spectrum): raw storage (float in the FP32 form) and
// the scale factor with its tangent.
__attribute__((visibility("hidden"))) const void *su2_tangent_component(clb_handle *h, int which, int comp, bool *f32,
                                                                        double *aI, double *daI)
{
  SU2Sector *u = h->su2;
  if (!u->tangent || comp < 0 || comp >= (which == 0 ? NF : NP)) return nullptr;
  TState t;
  if (cudaMemcpy(&t, u->d_tst, sizeof(t), cudaMemcpyDeviceToHost) != cudaSuccess) return nullptr;
  *aI = t.aI.v;
  *daI = t.aI.d;
  *f32 = u->fp32;
  const char *base = static_cast<const char *>(which == 0 ? u->df : u->dp);
  return base + (size_t)comp * h->n3 * u->esz;
}

} // namespace clb
