// clb_u1.cu - complex scalar + U(1) gauge sector (lphi4U1) behind the libclb200 C ABI.
//
// Schedules restate VelocityVerlet::evolve (evolvers/velocityverlet.h:51-114, 140-210) and
// LeapFrog::evolve / sync (evolvers/leapfrog.h:42-116, 141-217) for a model with one complex
// scalar and one U(1) field.  The second kick of a VV stage and the first kick of the next use the
// same kernel (no field or scale-factor change in between), so they run as one sweep that applies
// both kicks in sequence and reduces the momenta after each; on the leapfrog the field averages of
// a step are reduced by the next step's kick sweep, which reads the same fields.

#include "clb_adjoint.cuh"
#include "clb_gws.cuh"
#include "clb_handle.cuh"
#include "clb_u1.cuh"
#include "clb_vv.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace clb {

namespace {
constexpr int kU1Blocks = 148 * 8; // grid-stride sweeps: 8 resident 256-thread blocks per SM

// PITensor.h's GW source for lphi4U1: the complex scalar (components 0, 1) and the U(1) field
// (components 2..4, momenta 2..4); no singlets.
template <class R> struct U1GWSource {
  const R *f, *p;
  size_t n3;
  int N;
  R dx, ndxg, rfo2;
  const double *aI;
  __device__ __forceinline__ void operator()(size_t s, int x, int y, int z, int xp, int yp, int zp, R (&P)[6]) const
  {
    const size_t nb[3] = {((size_t)xp * N + y) * N + z, ((size_t)x * N + yp) * N + z, ((size_t)x * N + y) * N + zp};
    gw_gauge_tensor<R>(f, f + n3, f + 2 * n3, p + 2 * n3, n3, nb, s, dx, ndxg, (R)*aI, rfo2, true, P);
  }
};
} // namespace

struct U1Sector {
  void *f = nullptr, *p = nullptr; // 5 x N^3 each, FP64 or FP32 (esz bytes per value)
  int tile_lx = 8;                  // x-run of the staged kick; 0: the site-by-site kick
  int adj_lx = 16;                  // x-run of the staged adjoint sweep (CLB_U1_ADJ_LX)
  bool fp32 = false;
  size_t esz = 8;
  double *d_stage = nullptr; // one FP64 component, for FP32 conversions
  U1State *d_st = nullptr;
  double *d_part = nullptr; // kU1Blocks x kU1Meas
  double *d_sums = nullptr; // kU1Meas
  U1Params prm{};
  // adjoint: checkpoints every K steps, one segment of stage-boundary states, cotangents
  struct Ckpt {
    void *f = nullptr, *p = nullptr;
    U1State st{};
  };
  std::vector<Ckpt> ckpt;
  char *seg = nullptr;   // (K S + 1) boundary states of 10 N^3 values
  int64_t seg_cap = 0;   // boundary states the segment buffer holds
  U1State *d_rec = nullptr;
  double *qbar = nullptr, *pbar[2] = {nullptr, nullptr};
  double *d_apart = nullptr, *d_asums = nullptr;
  int64_t fwd_steps = -1, fwd_K = 0;
  // leapfrog: the forward's first kick weight (1/2 right after a sync), and whether it started
  // right after clb_initialize, where the previous half step's <pi^2> is that of the start momenta
  double fwd_w0 = 0.5;
  bool fwd_fresh = false;
  bool lf_fresh = false;      // no step since clb_initialize (not a restart)
  bool init_corrected = false; // clb_initialize set aDot = sqrt(RHS)
  double fwd_w[5] = {0, 0, 0, 0, 0};
  double fwd_avg[5] = {0, 0, 0, 0, 0}; // final <|pi_phi|^2>, <|D phi|^2>, <pi_A^2>, <B^2>, <V>
  double fwd_a = 1, fwd_obs = 0;
  // spectrum observable (clb_forward_spectrum): the cotangent of one component at the end state
  int seed_which = -1, seed_comp = 0; // -1: the energy observable of u1_forward
  double seed_abar = 0;
  double *seed = nullptr; // N^3
};

namespace {

U1Params make_params(const clb_handle *h)
{
  U1Params a{};
  const clb_config &c = h->cfg;
  const clb_model_desc &m = h->md;
  a.N = c.N;
  a.n3 = h->n3;
  a.dx = c.dx;
  a.dx2 = c.dx * c.dx;
  a.inv_dx2 = 1.0 / (c.dx * c.dx);
  a.gQ = m.couplings[1];
  a.c4 = m.couplings[0];
  a.ndxg = -c.dx * a.gQ;
  const double rfo = m.fStar / m.omegaStar, rof = m.omegaStar / m.fStar;
  a.J0 = 2.0 / c.dx * (rfo * rfo);
  a.el0 = 0.5 * (rof * rof);
  const double fm = m.fStar / m.MPl;
  a.alpha = m.alpha;
  a.fm2 = fm * fm;
  a.dt = c.dt;
  a.inv_n3 = 1.0 / (double)h->n3;
  a.order = gauge_site_order(c.N, c.precision == CLB_PREC_FP32_SPLIT);
  return a;
}

void set_coefs(U1State &s, double alpha)
{
  s.cs_drift = std::pow(s.aSI, alpha - 3);
  s.u1_drift = std::pow(s.aSI, alpha - 1);
  s.kA = std::pow(s.aI, 1 + alpha);
  s.kB2 = std::pow(s.aI, 3 + alpha) / 2;
  s.kG = std::pow(s.aI, -1 + alpha);
}

// Kick factors: complex scalar (dt/2) w and U(1) (dt w)/2 on the VV; (w dt) for both on the leapfrog.
U1Kick vv_kick(double dt, double wa, double wb)
{
  return U1Kick{{dt / 2 * wa, dt / 2 * wb}, {dt * wa / 2, dt * wb / 2}};
}
U1Kick lf_kick(double dt, double w) { return U1Kick{{w * dt, 0.0}, {w * dt, 0.0}}; }

// The staged kick (k_u1_kick_tile) unless CLB_U1_TILE=0; CLB_U1_TILE_LX sets its x-run.
template <int NK, bool RF, bool RP, class S> void kick_t(clb_handle *h, int kind, const U1Kick &kc)
{
  U1Sector *u = h->u1;
  if (u->tile_lx > 0) {
    static bool attr = false; // the ring is above the default 48 KB of dynamic shared memory
    if (!attr) {
      cudaFuncSetAttribute(k_u1_kick_tile<NK, RF, RP, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           U1Ring<S>::BYTES);
      attr = true;
    }
    CLB_LAUNCH(h, kind,
               k_u1_kick_tile<NK, RF, RP, S><<<kU1Blocks, 256, U1Ring<S>::BYTES, h->stream>>>(
                   static_cast<const S *>(u->f), static_cast<S *>(u->p), u->prm, kc, u->d_st, u->d_part, u->tile_lx));
    return;
  }
  CLB_LAUNCH(h, kind,
             k_u1_kick<NK, RF, RP, S><<<kU1Blocks, 256, 0, h->stream>>>(static_cast<const S *>(u->f),
                                                                         static_cast<S *>(u->p), u->prm, kc, u->d_st,
                                                                         u->d_part));
}
template <int NK, bool RF, bool RP> void kick(clb_handle *h, int kind, const U1Kick &kc)
{
  if (h->u1->fp32) return kick_t<NK, RF, RP, float>(h, kind, kc);
  kick_t<NK, RF, RP, double>(h, kind, kc);
}

template <class S> void drift_t(clb_handle *h, double w, double dtd)
{
  U1Sector *u = h->u1;
  CLB_LAUNCH(h, K_U1_DRIFT,
             k_u1_drift<S><<<kU1Blocks, 256, 0, h->stream>>>(static_cast<S *>(u->f), static_cast<const S *>(u->p),
                                                              h->n3, w, dtd, u->d_st));
}
// field drifts of weight w over dt (the position Verlet's half drifts pass dt/2: halving is exact,
// so ((pow dt)/2) w and ((pow w) dt)/2 of positionverlet.h:182-197 are the same numbers)
void drift(clb_handle *h, double w, double dtd = -1.0)
{
  if (dtd < 0) dtd = h->cfg.dt;
  if (h->u1->fp32) return drift_t<float>(h, w, dtd);
  drift_t<double>(h, w, dtd);
}

// One measurement sweep of the live state into d_sums (unnormalised sums, kU1Meas slots).
void measure_sums(clb_handle *h)
{
  U1Sector *u = h->u1;
  if (u->fp32)
    CLB_LAUNCH(h, K_MEASURE, k_u1_measure<float><<<kU1Blocks, 256, 0, h->stream>>>(
                                 static_cast<const float *>(u->f), static_cast<const float *>(u->p), u->prm, u->d_part));
  else
    CLB_LAUNCH(h, K_MEASURE, k_u1_measure<double><<<kU1Blocks, 256, 0, h->stream>>>(
                                 static_cast<const double *>(u->f), static_cast<const double *>(u->p), u->prm, u->d_part));
  CLB_LAUNCH(h, K_MEASURE, k_sum_partials<kU1Meas><<<1, 256, 0, h->stream>>>(u->d_part, kU1Blocks, u->d_sums));
}

void tail(clb_handle *h, uint32_t flags, bool reduced, double w = 0, double w2 = 0, int64_t hist_row = -1,
          double fa = 0, double fb = 0)
{
  U1Sector *u = h->u1;
  TailOp op{flags, reduced ? kU1Blocks : 0, w, w2, hist_row >= 0 ? h->d_hist : nullptr, hist_row, fa, fb};
  CLB_LAUNCH(h, K_TAIL, k_u1_tail<<<1, 256, 0, h->stream>>>(u->d_part, op, u->d_st, u->prm));
}

// Kick-sweep variants by (number of kicks, field reductions, momentum reductions).
void kick_sweep(clb_handle *h, int nk, bool rf, bool rp, const U1Kick &kc)
{
  const int kind = nk == 0 ? K_U1_REDUCE : K_U1_KICK;
  if (nk == 0) {
    if (rf && rp) return kick<0, true, true>(h, kind, kc);
    if (rf) return kick<0, true, false>(h, kind, kc);
    return kick<0, false, true>(h, kind, kc);
  }
  if (nk == 1) {
    if (rf && rp) return kick<1, true, true>(h, kind, kc);
    if (rp) return kick<1, false, true>(h, kind, kc);
    return kick<1, false, false>(h, kind, kc);
  }
  if (rf && rp) return kick<2, true, true>(h, kind, kc);
  return kick<2, false, false>(h, kind, kc);
}

cudaError_t copy_state(clb_handle *h, void *f, void *p, bool to_live)
{
  U1Sector *u = h->u1;
  const size_t bytes = 5 * h->n3 * u->esz;
  cudaError_t e = cudaMemcpyAsync(to_live ? u->f : f, to_live ? f : u->f, bytes, cudaMemcpyDeviceToDevice, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(to_live ? u->p : p, to_live ? p : u->p, bytes, cudaMemcpyDeviceToDevice, h->stream);
  return e;
}

// Boundary states and scalar records of a recomputed segment (adjoint).
struct SegSave {
  char *seg;     // boundary b at seg + 2 b half: fields, then momenta
  size_t half;   // bytes of 5 N^3 values
  U1State *rec;  // row b: the scalar state at boundary b
};

template <int NK, bool RED, class S> void kick_save_t(clb_handle *h, const U1Kick &kc, char *slot, size_t half)
{
  U1Sector *u = h->u1;
  if (u->tile_lx > 0) {
    static bool attr = false; // the ring is above the default 48 KB of dynamic shared memory
    if (!attr) {
      cudaFuncSetAttribute(k_u1_kick_tile<NK, RED, RED, S, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           U1Ring<S>::BYTES);
      attr = true;
    }
    CLB_LAUNCH(h, K_U1_KICK,
               k_u1_kick_tile<NK, RED, RED, S, true, true><<<kU1Blocks, 256, U1Ring<S>::BYTES, h->stream>>>(
                   static_cast<const S *>(u->f), static_cast<S *>(u->p), u->prm, kc, u->d_st, u->d_part, u->tile_lx,
                   reinterpret_cast<S *>(slot), reinterpret_cast<S *>(slot + half)));
    return;
  }
  CLB_LAUNCH(h, K_U1_KICK,
             k_u1_kick<NK, RED, RED, S, true, true><<<kU1Blocks, 256, 0, h->stream>>>(
                 static_cast<const S *>(u->f), static_cast<S *>(u->p), u->prm, kc, u->d_st, u->d_part,
                 reinterpret_cast<S *>(slot), reinterpret_cast<S *>(slot + half)));
}
template <class S> void kick_save_s(clb_handle *h, int nk, bool red, const U1Kick &kc, char *slot, size_t half)
{
  if (nk == 2)
    red ? kick_save_t<2, true, S>(h, kc, slot, half) : kick_save_t<2, false, S>(h, kc, slot, half);
  else
    red ? kick_save_t<1, true, S>(h, kc, slot, half) : kick_save_t<1, false, S>(h, kc, slot, half);
}

// VelocityVerlet::evolve over nsteps with merged kicks (as u1_evolve).  With sv, the state and the
// scalar record at every stage boundary are kept: the merged sweep writes the state between its
// two kicks, and its tail is split at the boundary so the record can be taken there.
// hist: per-step history rows (clb_evolve sizes that buffer; the adjoint's runs write none), the
// first at row row0.
void vv_run(clb_handle *h, int64_t nsteps, const SegSave *sv, bool hist = true, int64_t row0 = 0)
{
  const double dt = h->cfg.dt;
  const bool ex = h->cfg.expansion != 0;
  const std::vector<double> &ws = h->ws;
  const size_t P = ws.size(), S = 2 * P - 1;
  auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
  const int64_t total = nsteps * (int64_t)S;
  const double w0 = wof(0);
  if (sv) {
    copy_state(h, sv->seg, sv->seg + sv->half, false);
    k_u1_record<<<1, 1, 0, h->stream>>>(h->u1->d_st, sv->rec, 0);
  }
  if (ex) tail(h, T_VV_KICK_HALF, false, 0, w0); // kickScaleFactorHalf
  kick_sweep(h, 1, false, ex, vv_kick(dt, w0, 0.0));
  if (ex) tail(h, T_STORE_PI2_I | T_VV_DRIFT, true, 0, w0); // <pi^2>, driftScaleFactor
  for (int64_t k = 0; k < total; ++k) {
    const size_t i = (size_t)(k % (int64_t)S);
    const double w = wof(i);
    const bool more = k + 1 < total;
    const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
    drift(h, w);
    if (!sv) {
      kick_sweep(h, more ? 2 : 1, ex, ex, vv_kick(dt, w, wn));
      if (ex) {
        uint32_t fl = T_STORE_FIELDS | T_STORE_PI2_I | T_VV_KICK_ONE;
        if (more) fl |= T_VV_KICK_HALF | T_STORE_PI2_B | T_VV_DRIFT;
        tail(h, fl, true, w, wn, hist && i + 1 == S ? row0 + k / (int64_t)S : -1);
      }
    } else {
      char *slot = sv->seg + (size_t)(k + 1) * 2 * sv->half;
      if (h->u1->fp32)
        kick_save_s<float>(h, more ? 2 : 1, ex, vv_kick(dt, w, wn), slot, sv->half);
      else
        kick_save_s<double>(h, more ? 2 : 1, ex, vv_kick(dt, w, wn), slot, sv->half);
      if (ex) {
        // first kick's tail, the boundary record, second kick's tail: one launch
        U1Sector *u = h->u1;
        const TailOp a{T_STORE_FIELDS | T_STORE_PI2_I | T_VV_KICK_ONE, kU1Blocks, w, 0.0, nullptr, -1};
        const TailOp b{more ? (uint32_t)(T_VV_KICK_HALF | T_STORE_PI2_B | T_VV_DRIFT) : 0u, kU1Blocks, w, wn, nullptr, -1};
        CLB_LAUNCH(h, K_TAIL, k_u1_tail_split<<<1, 256, 0, h->stream>>>(u->d_part, a, b, u->d_st, u->prm, sv->rec, k + 1));
      } else {
        k_u1_record<<<1, 1, 0, h->stream>>>(h->u1->d_st, sv->rec, k + 1);
      }
    }
  }
}

// LeapFrog::evolve over nsteps (as u1_evolve's leapfrog branch, the same launches, no history rows).  With sv, the
// state before every kick (boundary b: the fields of step b and the momenta half a step earlier)
// goes to boundary slot b, the scalar state after the step's kick tail to record row b, and the
// end state to slot nsteps.
void lf_run(clb_handle *h, int64_t nsteps, const SegSave *sv)
{
  const double dt = h->cfg.dt;
  const bool ex = h->cfg.expansion != 0;
  const double w0 = h->synced ? 0.5 : 1.0;
  auto slot = [&](int64_t b) { return sv->seg + (size_t)b * 2 * sv->half; };
  for (int64_t s = 0; s < nsteps; ++s) {
    if (sv) copy_state(h, slot(s), slot(s) + sv->half, false);
    if (s == 0) {
      kick_sweep(h, 1, false, ex, lf_kick(dt, w0));
      if (ex) tail(h, T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true);
    } else {
      kick_sweep(h, 1, ex, ex, lf_kick(dt, 1.0));
      if (ex) tail(h, T_STORE_FIELDS | T_HIST_EARLY | T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true);
    }
    if (sv) k_u1_record<<<1, 1, 0, h->stream>>>(h->u1->d_st, sv->rec, s);
    drift(h, 1.0);
  }
  if (ex) {
    kick_sweep(h, 0, true, false, U1Kick{});
    tail(h, T_STORE_FIELDS | T_HIST_EARLY, true);
  }
  if (sv) {
    copy_state(h, slot(nsteps), slot(nsteps) + sv->half, false);
    k_u1_record<<<1, 1, 0, h->stream>>>(h->u1->d_st, sv->rec, nsteps);
  }
  h->synced = false;
}

int check(clb_handle *h, const char *where)
{
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  collect_profile(h);
  U1State s;
  e = cudaMemcpy(&s, h->u1->d_st, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, where);
  if (s.status != 0) return h->fail(CLB_ENONFINITE, std::string(where) + ": a volume average or a(t) is not finite");
  return CLB_OK;
}

} // namespace

void gw_kick_step(clb_handle *h);
void gw_drift(clb_handle *h);
void gw_sync(clb_handle *h);

// The GW kick (weight w of dt) with the lphi4U1 source, at the current fields, momenta and a_I.
__attribute__((visibility("hidden"))) void u1_gw_kick(clb_handle *h, double w)
{
  U1Sector *u = h->u1;
  GWSector *g = h->gw;
  const double r = h->md.fStar / h->md.omegaStar; // pow<2>(fStar / omegaStar)
  const double inv_dx2 = 1.0 / (h->cfg.dx * h->cfg.dx), hd = w * h->cfg.dt;
  auto go = [&](auto zero) {
    using R = decltype(zero);
    const U1GWSource<R> src{static_cast<const R *>(u->f), static_cast<const R *>(u->p), h->n3, h->N, (R)h->cfg.dx,
                            (R)u->prm.ndxg, (R)(r * r), &u->d_st->aI};
    CLB_LAUNCH(h, K_GW, (k_gw_kick<R, U1GWSource<R>><<<kGWBlocks, 256, 0, h->stream>>>(
                            static_cast<const R *>(g->u), static_cast<R *>(g->pi), h->N, inv_dx2, hd, &u->d_st->kA, src)));
  };
  if (u->fp32) go(0.0f);
  else go(0.0);
}

// The GW drift with the a_SI of the matter step just taken (U1State::cs_drift = pow(a_SI, alpha - 3)
// on the VV and the leapfrog).
__attribute__((visibility("hidden"))) void u1_gw_drift(clb_handle *h)
{
  U1Sector *u = h->u1;
  GWSector *g = h->gw;
  const size_t n = 5 * h->n3;
  const bool pv = is_pv(h->cfg.evolver); // cs_drift is then a_I's: the drift forms a_SI's
  if (u->fp32)
    CLB_LAUNCH(h, K_GW, launch_gw_drift<float>(static_cast<float *>(g->u), static_cast<const float *>(g->pi), n,
                                               h->cfg.dt, &u->d_st->cs_drift, &u->d_st->aSI, h->md.alpha, pv,
                                               h->stream));
  else
    CLB_LAUNCH(h, K_GW, launch_gw_drift<double>(static_cast<double *>(g->u), static_cast<const double *>(g->pi), n,
                                                h->cfg.dt, &u->d_st->cs_drift, &u->d_st->aSI, h->md.alpha, pv,
                                                h->stream));
}

__attribute__((visibility("hidden"))) int u1_create(clb_handle *h)
{
  U1Sector *u = new U1Sector();
  h->u1 = u;
  h->NS = 5;
  u->prm = make_params(h);
  u->fp32 = h->cfg.precision == CLB_PREC_FP32_SPLIT;
  u->esz = u->fp32 ? sizeof(float) : sizeof(double);
  // x-run of the staged kick: 8 planes FP64, 32 FP32 (128^3 VV4, ms per step: FP64 0.726 / 0.751 /
  // 0.742 for 8 / 16 / 32, FP32 0.340 / 0.340 / 0.325; the site-by-site kick 0.885 and 0.386)
  u->tile_lx = u->fp32 ? 32 : 8;
  if (const char *env = std::getenv("CLB_U1_TILE")) u->tile_lx = std::atoi(env) == 0 ? 0 : u->tile_lx;
  if (const char *env = std::getenv("CLB_U1_TILE_LX"))
    if (u->tile_lx > 0) u->tile_lx = std::max(1, std::atoi(env));
  if (const char *env = std::getenv("CLB_U1_ADJ_LX")) u->adj_lx = std::max(1, std::atoi(env));
  const size_t bytes = 5 * h->n3 * u->esz;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc(&u->f, bytes) == cudaSuccess && cudaMalloc(&u->p, bytes) == cudaSuccess;
  ok = ok && cudaMemset(u->f, 0, bytes) == cudaSuccess && cudaMemset(u->p, 0, bytes) == cudaSuccess;
  if (u->fp32) ok = ok && cudaMalloc(&u->d_stage, h->n3 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_st, sizeof(U1State)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_part, (size_t)kU1Blocks * kU1Meas * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&u->d_sums, kU1Meas * sizeof(double)) == cudaSuccess;
  ok = ok && cudaEventCreate(&h->ev_call[0]) == cudaSuccess && cudaEventCreate(&h->ev_call[1]) == cudaSuccess;
  if (!ok) return CLB_ENOMEM;
  U1State s{};
  s.aI = s.aSI = s.aIM = 1.0;
  set_coefs(s, h->md.alpha);
  return cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice) == cudaSuccess ? CLB_OK : CLB_ECUDA;
}

static void free_adjoint(U1Sector *u)
{
  for (auto &c : u->ckpt) {
    if (c.f) cudaFree(c.f);
    if (c.p) cudaFree(c.p);
  }
  u->ckpt.clear();
  if (u->seg) cudaFree(u->seg);
  if (u->d_rec) cudaFree(u->d_rec);
  u->seg = nullptr;
  u->d_rec = nullptr;
  u->seg_cap = 0;
  for (double **b : {&u->qbar, &u->pbar[0], &u->pbar[1], &u->d_apart, &u->d_asums, &u->seed}) {
    if (*b) cudaFree(*b);
    *b = nullptr;
  }
  u->fwd_steps = -1;
  u->seed_which = -1;
}

__attribute__((visibility("hidden"))) void u1_destroy(clb_handle *h)
{
  U1Sector *u = h->u1;
  if (!u) return;
  free_adjoint(u);
  if (u->f) cudaFree(u->f);
  if (u->p) cudaFree(u->p);
  if (u->d_st) cudaFree(u->d_st);
  if (u->d_part) cudaFree(u->d_part);
  if (u->d_sums) cudaFree(u->d_sums);
  if (u->d_stage) cudaFree(u->d_stage);
  delete u;
  h->u1 = nullptr;
}

__attribute__((visibility("hidden"))) int u1_set_state(clb_handle *h, const double *fields, const double *momenta,
                                                       const clb_scalefactor *sf)
{
  U1Sector *u = h->u1;
  const size_t bytes = 5 * h->n3 * sizeof(double);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (!u->fp32) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(u->f, fields, bytes, cudaMemcpyDefault, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(u->p, momenta, bytes, cudaMemcpyDefault, h->stream);
  } else {
    // one component at a time through the FP64 staging buffer, rounded once to FP32
    for (int c = 0; c < 10 && e == cudaSuccess; ++c) {
      const double *src = (c < 5 ? fields : momenta) + (size_t)(c % 5) * h->n3;
      float *dst = static_cast<float *>(c < 5 ? u->f : u->p) + (size_t)(c % 5) * h->n3;
      e = cudaMemcpyAsync(u->d_stage, src, h->n3 * sizeof(double), cudaMemcpyDefault, h->stream);
      if (e == cudaSuccess) k_convert<double, float><<<kU1Blocks, 256, 0, h->stream>>>(u->d_stage, dst, h->n3);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  U1State s{};
  s.aI = s.aSI = s.aIM = 1.0;
  if (sf) {
    s.aI = sf->aI;
    s.aSI = sf->aSI;
    s.aIM = sf->aIM;
    s.aDotI = sf->aDotI;
    s.aDotSI = sf->aDotSI;
    s.aDotSIM = sf->aDotSIM;
  }
  set_coefs(s, h->md.alpha);
  e = cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_set_state");
  h->has_state = true;
  h->initialized = false;
  h->synced = true;
  return CLB_OK;
}

__attribute__((visibility("hidden"))) int u1_get_state(clb_handle *h, double *fields, double *momenta,
                                                       clb_scalefactor *sf)
{
  U1Sector *u = h->u1;
  const size_t bytes = 5 * h->n3 * sizeof(double);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (!u->fp32) {
    if (e == cudaSuccess && fields) e = cudaMemcpyAsync(fields, u->f, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && momenta) e = cudaMemcpyAsync(momenta, u->p, bytes, cudaMemcpyDeviceToHost, h->stream);
  } else {
    for (int c = 0; c < 10 && e == cudaSuccess; ++c) {
      double *dst = c < 5 ? fields : momenta;
      if (!dst) continue;
      dst += (size_t)(c % 5) * h->n3;
      const float *src = static_cast<const float *>(c < 5 ? u->f : u->p) + (size_t)(c % 5) * h->n3;
      k_convert<float, double><<<kU1Blocks, 256, 0, h->stream>>>(src, u->d_stage, h->n3);
      e = cudaMemcpyAsync(dst, u->d_stage, h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
  }
  U1State s;
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

// ModelInitializer tail (modelinitializer.h:74-80) and the leapfrog constructor (leapfrog.h:35).
__attribute__((visibility("hidden"))) int u1_initialize(clb_handle *h, int32_t correct_adot)
{
  kick_sweep(h, 0, true, true, U1Kick{});
  uint32_t fl = T_STORE_ALL;
  if (h->cfg.expansion && correct_adot == 1 && !h->fb) fl |= T_CORRECT_ADOT; // modelinitializer.h:74-80
  if (h->cfg.expansion && h->cfg.evolver == CLB_LF && correct_adot != CLB_INIT_RESTART) fl |= T_LF_CTOR;
  tail(h, fl, true);
  h->synced = !(correct_adot == CLB_INIT_RESTART && h->cfg.evolver == CLB_LF); // leapfrog.h:30-31
  h->u1->lf_fresh = correct_adot != CLB_INIT_RESTART;
  h->u1->init_corrected = (fl & T_CORRECT_ADOT) != 0;
  return check(h, "clb_initialize");
}

__attribute__((visibility("hidden"))) int u1_evolve(clb_handle *h, int64_t nsteps)
{
  const double dt = h->cfg.dt;
  const bool ex = h->cfg.expansion != 0;
  cudaEventRecord(h->ev_call[0], h->stream);
  h->u1->lf_fresh = false;
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
        kick_sweep(h, 1, false, false, lf_kick(dt, h->synced ? 0.5 : 1.0));
        const double tm = h->fb_t - t0;
        tail(h, T_FB_AIM | T_FB_AI | T_FB_ASI, false, 0, 0, -1, h->fb_a(tm + dt), h->fb_a(tm + dt / 2.0));
        drift(h, 1.0);
        if (h->gw) gw_drift(h);
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
          drift(h, w, dt / 2);
          tail(h, T_PV_MODE | T_FB_PV_HALF, false, 0, 0, -1, 0.0, h->fb_a(tc + w * dt / 2.0));
          kick_sweep(h, 1, false, false, lf_kick(dt, w));
          tail(h, T_PV_MODE | T_FB_AI, false, 0, 0, -1, h->fb_a(tc + w * dt));
          drift(h, w, dt / 2);
          tc += dt * w;
        }
        if (h->gw) gw_drift(h);
        h->fb_t += dt;
      }
    } else {
      auto vv_fb = [&](int64_t n) {
        const int64_t total = n * (int64_t)S;
        kick_sweep(h, 1, false, false, vv_kick(dt, wof(0), 0.0));
        double tc = h->fb_t - t0;
        for (int64_t k = 0; k < total; ++k) {
          const size_t i = (size_t)(k % (int64_t)S);
          const double w = wof(i);
          const bool more = k + 1 < total;
          const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
          tail(h, T_FB_AIM | T_FB_AI, false, 0, 0, -1, h->fb_a(tc + w * dt));
          drift(h, w);
          kick_sweep(h, more ? 2 : 1, false, false, vv_kick(dt, w, wn));
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
    // LeapFrog::evolve: kick (1/2 dt after a sync), <pi^2>, a kick and drift, field drifts, field averages
    // With GWs (evolver.h:102-124): a GW kick before each step's kick (the step's fields, the
    // momenta half a step back, a_I) and a GW drift after its drift (its a_SI)
    const double weight = h->synced ? 0.5 : 1.0;
    if (h->gw) gw_kick_step(h);
    kick_sweep(h, 1, false, ex, lf_kick(dt, weight));
    if (ex) tail(h, T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true);
    for (int64_t s = 0; s < nsteps; ++s) {
      drift(h, 1.0);
      if (h->gw) gw_drift(h);
      if (s + 1 < nsteps) {
        if (h->gw) gw_kick_step(h);
        kick_sweep(h, 1, ex, ex, lf_kick(dt, 1.0));
        if (ex) tail(h, T_STORE_FIELDS | T_HIST_EARLY | T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true, 0, 0, s);
      } else {
        if (ex) {
          kick_sweep(h, 0, true, false, U1Kick{});
          tail(h, T_STORE_FIELDS | T_HIST_EARLY, true, 0, 0, s);
        }
      }
    }
    h->synced = false;
  } else if (is_pv(h->cfg.evolver)) {
    // PositionVerlet::evolve (positionverlet.h:45-99): drift(dt/2 w), a first half-drift, kick(w dt)
    // at the half-step a (its sweep also reduces the half-step field sums), the momentum sums, the
    // a-kick and second half-drift, drift(dt/2 w); each step ends with a field-sum sweep.  The
    // first a half-drift of a stage is booked in the tail before its first field drift, whose
    // coefficient then comes from aIM.
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
        drift(h, w, dt / 2);
        kick_sweep(h, 1, ex, ex, lf_kick(dt, w));
        if (ex)
          tail(h, T_PV_MODE | T_PV_STORE_SI | T_PV_STORE_PI2 | T_PV_KICK | T_PV_DRIFT_A2 | (last ? 0u : T_PV_DRIFT_A1),
               true, w, last ? 0.0 : wof(i + 1));
        drift(h, w, dt / 2);
        if (last && h->gw) {
          gw_drift(h);
          if (s + 1 < nsteps) gw_kick_step(h);
        }
        if (last && ex) {
          kick_sweep(h, 0, true, false, U1Kick{});
          tail(h, T_PV_MODE | T_STORE_FIELDS | (s + 1 < nsteps ? T_PV_DRIFT_A1 : 0u), true, 0, w0, s);
        }
      }
  } else if (h->gw) {
    // the GW leapfrog around each matter step (evolver.h:102-124): its kick reads the gauge
    // momenta at integer time, which the merged sweep between two steps never stores, so the steps
    // run one by one (the schedule of one-step clb_evolve calls)
    for (int64_t s = 0; s < nsteps; ++s) {
      gw_kick_step(h);
      vv_run(h, 1, nullptr, true, s);
      gw_drift(h);
    }
  } else {
    vv_run(h, nsteps, nullptr);
  }
  cudaEventRecord(h->ev_call[1], h->stream);
  const int r = check(h, "clb_evolve");
  float ms = 0;
  if (cudaEventElapsedTime(&ms, h->ev_call[0], h->ev_call[1]) == cudaSuccess) h->last_evolve_ms = ms;
  return r;
}

// LeapFrog::sync (leapfrog.h:96-116); a no-op on the VV.
__attribute__((visibility("hidden"))) int u1_sync(clb_handle *h)
{
  if (h->gw) gw_sync(h); // evolver.h:134-137, before the matter sync
  if (h->cfg.evolver == CLB_LF && !h->synced) {
    h->u1->lf_fresh = false;
    kick_sweep(h, 1, false, h->cfg.expansion != 0 && !h->fb, lf_kick(h->cfg.dt, 0.5));
    if (h->cfg.expansion && !h->fb) tail(h, T_STORE_PI2_I | T_LF_SYNC, true);
  }
  if (h->fb) tail(h, T_FB_ADOT, false, 0, 0, -1, 0.0, h->fb_adot(h->fb_t - h->cfg.t0));
  h->synced = true;
  return check(h, "clb_sync");
}

// Frequent measurement of lphi4U1: energies (energiesmeasurer.h:45-122), complex scalar means
// (complexscalarmeasurer.h:61-72), U(1) |E|, |B| means and the Gauss check (u1measurer.h:78-87).
__attribute__((visibility("hidden"))) int u1_measure(clb_handle *h, double e0, clb_measurement *m)
{
  U1Sector *u = h->u1;
  U1State s;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&s, u->d_st, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  measure_sums(h);
  double v[kU1Meas];
  e = cudaMemcpyAsync(v, u->d_sums, sizeof(v), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  collect_profile(h);
  const double inv = 1.0 / (double)h->n3;
  for (double &x : v) x *= inv;
  std::memset(m, 0, sizeof(*m));
  const double al = h->md.alpha;
  auto ipow = [](double x, int n) {
    double r = x;
    for (int i = 1; i < n; ++i) r = r * x;
    return r;
  };
  const double am6 = 1.0 / ipow(s.aI, 6), am2 = 1.0 / ipow(s.aI, 2), e4 = u->prm.el0 / ipow(s.aI, 4);
  const double Ekcs = v[0] * am6, Egcs = v[1] * am2, Eel = e4 * v[2], Emag = e4 * v[3], V = v[4];
  const double Etot = ((Ekcs + Egcs) + (Eel + Emag)) + V;
  const double en[6] = {Ekcs, Egcs, Eel, Emag, V, Etot};
  for (int k = 0; k < 6; ++k) m->energies[k] = en[k];
  m->n_energies = 6;
  if (h->cfg.expansion) {
    // HubbleConstraint::get refreshes the cached averages (energies.h:219) before forming rho
    s.potI = s.potSI = v[4];
    s.u1Pi2I = s.u1Pi2SI = v[2];
    s.u1Mag2I = v[3];
    s.csPi2I = s.csPi2SI = v[0];
    s.csGrad2I = v[1];
    const double rho = (((s.csPi2I * am6 + s.csGrad2I * am2) + e4 * s.u1Pi2I) + e4 * s.u1Mag2I) + s.potI;
    const double LHS = s.aDotI * s.aDotI;
    const double RHS = std::pow(s.aI, 2 * al + 2) / 3. * u->prm.fm2 * rho;
    m->friedmann[0] = (LHS - RHS) / (LHS + RHS);
    m->friedmann[1] = LHS;
    m->friedmann[2] = RHS;
    set_coefs(s, al);
    e = cudaMemcpy(u->d_st, &s, sizeof(s), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_measure");
  } else {
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  }
  const double am = std::pow(s.aI, al - 3), ag = std::pow(s.aI, al - 1), r2 = std::sqrt(2.0);
  auto row = [&](int r, double a1, double b1, double a2, double b2) {
    const double r1 = a2 - a1 * a1, rr = b2 - b1 * b1;
    m->means[r][0] = a1;
    m->means[r][1] = b1;
    m->means[r][2] = a2;
    m->means[r][3] = b2;
    m->means[r][4] = r1 > 0 ? std::sqrt(r1) : 0;
    m->means[r][5] = rr > 0 ? std::sqrt(rr) : 0;
  };
  row(0, r2 * v[5], r2 * am * v[11], 2 * v[6], 2 * am * am * v[12]);
  row(1, r2 * v[7], r2 * am * v[13], 2 * v[8], 2 * am * am * v[14]);
  row(2, v[9], am * v[15], v[10], am * am * v[16]);
  row(3, ag * v[17], v[18], ag * ag * v[2], v[3]);
  m->n_means = 4;
  m->gauss_u1[0] = v[19] / v[20];
  m->gauss_u1[1] = v[22];
  m->gauss_u1[2] = v[21];
  m->aI = s.aI;
  m->aDotI = s.aDotI;
  m->hubble = s.aDotI / s.aI;
  return CLB_OK;
}

// ---- adjoint: forward with checkpoints, backward by segment recompute -------------------------
namespace {

constexpr int kAvgN = 5; // <|pi_phi|^2>, <|D phi|^2>, <pi_A^2>, <B^2>, <V>

// Scale-factor equation F(a, <.>) (scalefactorkernels.h:73-77) and its partial derivatives.
struct SFGrad {
  double dA[kAvgN];
  double da;
};
SFGrad sf_grad(const U1Params &p, double a, const double (&A)[kAvgN])
{
  const double al = p.alpha, e = p.el0;
  const double c = std::pow(a, 2 * al + 1) / 3.0 * p.fm2, dc = (2 * al + 1) * std::pow(a, 2 * al) / 3.0 * p.fm2;
  const double br = (al - 2) * A[0] * std::pow(a, -6) + al * A[1] * std::pow(a, -2) +
                    (al - 1) * e * std::pow(a, -4) * (A[2] + A[3]) + (al + 1) * A[4];
  const double dbr = (al - 2) * A[0] * -6 * std::pow(a, -7) + al * A[1] * -2 * std::pow(a, -3) +
                     (al - 1) * e * -4 * std::pow(a, -5) * (A[2] + A[3]);
  SFGrad g;
  g.dA[0] = c * (al - 2) * std::pow(a, -6);
  g.dA[1] = c * al * std::pow(a, -2);
  g.dA[2] = g.dA[3] = c * (al - 1) * e * std::pow(a, -4);
  g.dA[4] = c * (al + 1);
  g.da = dc * br + c * dbr;
  return g;
}

void averages_of(const U1State &s, double (&A)[kAvgN])
{
  A[0] = s.csPi2I;
  A[1] = s.csGrad2I;
  A[2] = s.u1Pi2I;
  A[3] = s.u1Mag2I;
  A[4] = s.potI;
}

// Energies (energiesmeasurer.h:45-122) from the five averages at scale factor a.
void energies_of(const U1Params &p, double a, const double (&A)[kAvgN], double (&E)[kAvgN])
{
  E[0] = A[0] * std::pow(a, -6);
  E[1] = A[1] * std::pow(a, -2);
  E[2] = p.el0 * std::pow(a, -4) * A[2];
  E[3] = p.el0 * std::pow(a, -4) * A[3];
  E[4] = A[4];
}

template <class T>
void adj_launch(clb_handle *h, const void *f, const void *p, const double *pin, double *pout, const U1AdjArgs &g)
{
  U1Sector *u = h->u1;
  if (u->tile_lx > 0) { // the sweep on staged planes (CLB_U1_TILE=0: site by site)
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_u1_adj_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, U1AdjRing<T>::BYTES);
      attr = true;
    }
    k_u1_adj_tile<T><<<kU1Blocks, U1AdjRing<T>::THREADS, U1AdjRing<T>::BYTES, h->stream>>>(
        static_cast<const T *>(f), static_cast<const T *>(p), pin, u->qbar, pout, u->prm, g, u->d_apart, u->adj_lx);
    return;
  }
  k_u1_adj<T><<<kU1Blocks, 256, 0, h->stream>>>(static_cast<const T *>(f), static_cast<const T *>(p), pin, u->qbar,
                                                 pout, u->prm, g, u->d_apart);
}

// One fused adjoint sweep at a boundary state and its dot products S.
int adj_sweep(clb_handle *h, const void *f, const void *p, const double *pin, double *pout, const U1AdjArgs &g,
              double (&S)[kAdjSlots])
{
  U1Sector *u = h->u1;
  if (u->fp32)
    CLB_LAUNCH(h, K_U1_ADJ, adj_launch<float>(h, f, p, pin, pout, g));
  else
    CLB_LAUNCH(h, K_U1_ADJ, adj_launch<double>(h, f, p, pin, pout, g));
  CLB_LAUNCH(h, K_TAIL, k_sum_partials<kAdjSlots><<<1, 256, 0, h->stream>>>(u->d_apart, kU1Blocks, u->d_asums));
  cudaError_t e = cudaMemcpyAsync(S, u->d_asums, sizeof(S), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? CLB_OK : h->cuda_fail(e, "clb_backward");
}

// Sweep arguments at scale factor a with both parts empty: kick coefficients and their a-derivatives.
U1AdjArgs adj_base(const U1Params &p, double a)
{
  const double al = p.alpha;
  U1AdjArgs g{};
  g.kA = std::pow(a, 1 + al);
  g.kB2 = std::pow(a, 3 + al) / 2;
  g.kG = std::pow(a, al - 1);
  g.dkA = (1 + al) * std::pow(a, al);
  g.dkB2 = (3 + al) * std::pow(a, 2 + al) / 2;
  g.dkG = (al - 1) * std::pow(a, al - 2);
  g.J0 = p.J0;
  g.r2 = p.J0 * p.dx; // 2 (fStar/omegaStar)^2
  g.inv_n3 = p.inv_n3;
  return g;
}

} // namespace

// Forward pass of the adjoint pair: nsteps VV steps from the current (initialized) state with a
// checkpoint every K steps, then the observable O = sum_k w_k E_k / E_tot over the energy
// components (E_kin, E_grad of the complex scalar, E_el, E_mag, V).
__attribute__((visibility("hidden"))) int u1_forward(clb_handle *h, int64_t nsteps, int32_t K, const double *w,
                                                     int32_t nw, double *obs)
{
  U1Sector *u = h->u1;
  const bool lf = h->cfg.evolver == CLB_LF;
  if (is_pv(h->cfg.evolver))
    return h->fail(CLB_EUNSUPPORTED, "clb_forward: the adjoint covers the VV evolvers and the leapfrog");
  if (h->fb) return h->fail(CLB_EUNSUPPORTED, "clb_forward: the adjoint covers the self-consistent expansion");
  if (h->gw) return h->fail(CLB_EUNSUPPORTED, "clb_forward: the adjoint runs without the GW sector");
  if (nsteps < 1 || K < 1) return h->fail(CLB_EINVAL, "clb_forward: nsteps and checkpoint_every must be >= 1");
  if (nw < 0 || nw > kAvgN || (nw > 0 && !w)) return h->fail(CLB_EINVAL, "clb_forward: up to 5 energy weights");
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_forward");
  const size_t bytes = 5 * h->n3 * u->esz, dbytes = 5 * h->n3 * sizeof(double);
  const int64_t nck = (nsteps + K - 1) / K;
  const int64_t S = lf ? 1 : 2 * (int64_t)h->ws.size() - 1; // boundaries per step
  const int64_t seg_states = std::min<int64_t>(K, nsteps) * S + 1;
  // the storage of the previous pair is kept when its layout fits (same checkpoint count and
  // segment length); the observable is reset either way
  u->fwd_steps = -1;
  u->seed_which = -1;
  if (!(u->ckpt.size() == (size_t)nck + 1 && u->seg_cap == seg_states && u->qbar)) {
    free_adjoint(u);
    bool ok = true;
    u->ckpt.resize((size_t)nck + 1); // + the end state, restored after the backward pass
    for (auto &c : u->ckpt) ok = ok && cudaMalloc(&c.f, bytes) == cudaSuccess && cudaMalloc(&c.p, bytes) == cudaSuccess;
    ok = ok && cudaMalloc(&u->seg, (size_t)seg_states * 2 * bytes) == cudaSuccess;
    ok = ok && cudaMalloc(&u->d_rec, (size_t)seg_states * sizeof(U1State)) == cudaSuccess;
    ok = ok && cudaMalloc(&u->qbar, dbytes) == cudaSuccess && cudaMalloc(&u->pbar[0], dbytes) == cudaSuccess &&
         cudaMalloc(&u->pbar[1], dbytes) == cudaSuccess;
    ok = ok && cudaMalloc(&u->d_apart, (size_t)kU1Blocks * kAdjSlots * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&u->d_asums, kAdjSlots * sizeof(double)) == cudaSuccess;
    if (!ok) {
      free_adjoint(u);
      return h->fail(CLB_ENOMEM, "clb_forward: checkpoint or segment storage does not fit; use a smaller checkpoint_every");
    }
    u->seg_cap = seg_states;
  }
  cudaEventRecord(h->ev_call[0], h->stream);
  u->fwd_w0 = h->synced ? 0.5 : 1.0;
  u->fwd_fresh = lf && u->lf_fresh;
  u->lf_fresh = false;
  for (int64_t c = 0; c < nck; ++c) {
    U1Sector::Ckpt &ck = u->ckpt[(size_t)c];
    if ((e = copy_state(h, ck.f, ck.p, false)) != cudaSuccess) return h->cuda_fail(e, "clb_forward");
    if ((e = cudaMemcpyAsync(&ck.st, u->d_st, sizeof(U1State), cudaMemcpyDeviceToHost, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_forward");
    if (lf)
      lf_run(h, std::min<int64_t>(K, nsteps - c * K), nullptr); // the launches of clb_evolve
    else
      vv_run(h, std::min<int64_t>(K, nsteps - c * K), nullptr, false); // the merged schedule of clb_evolve
  }
  if (lf) { // LeapFrog::sync: the observable is measured at integer-time momenta
    const bool ex = h->cfg.expansion != 0;
    kick_sweep(h, 1, false, ex, lf_kick(h->cfg.dt, 0.5));
    if (ex) tail(h, T_STORE_PI2_I | T_LF_SYNC, true);
  }
  cudaEventRecord(h->ev_call[1], h->stream);
  {
    U1Sector::Ckpt &c = u->ckpt.back();
    if ((e = copy_state(h, c.f, c.p, false)) != cudaSuccess) return h->cuda_fail(e, "clb_forward");
    if ((e = cudaMemcpyAsync(&c.st, u->d_st, sizeof(U1State), cudaMemcpyDeviceToHost, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_forward");
  }
  int r = check(h, "clb_forward");
  if (r != CLB_OK) return r;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, h->ev_call[0], h->ev_call[1]) == cudaSuccess) h->last_evolve_ms = ms;
  // final averages (one measurement sweep) and the observable
  measure_sums(h);
  double v[kU1Meas];
  U1State s;
  e = cudaMemcpyAsync(v, u->d_sums, sizeof(v), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&s, u->d_st, sizeof(s), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_forward");
  const double inv = u->prm.inv_n3;
  u->fwd_avg[0] = v[0] * inv;
  u->fwd_avg[1] = v[1] * inv;
  u->fwd_avg[2] = v[2] * inv;
  u->fwd_avg[3] = v[3] * inv;
  u->fwd_avg[4] = v[4] * inv;
  u->fwd_a = s.aI;
  for (int k = 0; k < kAvgN; ++k) u->fwd_w[k] = k < nw ? w[k] : 0.0;
  double E[kAvgN], Et = 0, Ew = 0;
  energies_of(u->prm, s.aI, u->fwd_avg, E);
  for (int k = 0; k < kAvgN; ++k) {
    Et += E[k];
    Ew += u->fwd_w[k] * E[k];
  }
  u->fwd_obs = Ew / Et;
  u->fwd_steps = nsteps;
  u->fwd_K = K;
  h->synced = true;
  if (obs) *obs = u->fwd_obs;
  return CLB_OK;
}

// Backward pass: cotangents of the forward start state and of the couplings for the observable
// of the last u1_forward.  Segments are recomputed from their (bitwise) checkpoints with the
// forward's merged schedule, keeping every stage-boundary state and scalar record; the FP64
// recompute evaluates the kernel in FD arithmetic (contracted, divisions as reciprocal multiplies),
// which moves the linearisation point by rounding only.  Then one fused adjoint sweep per
// boundary walks the segment backwards (part A: the
// first kick of the stage starting there, part B: the second kick of the stage ending there).
// With through_init the start state is taken as produced by clb_initialize(correct_adot = 1),
// whose aDot = sqrt(Friedmann RHS) (modelinitializer.h:77-78) is differentiated too.
namespace {
// pbar += (2 X_phi / N^3) p_phi, (2 X_A / N^3) p_A: the cotangents X of the two momentum averages
// of the momenta p (storage type of the state), or pbar = that (set).
void pbar_axpy(clb_handle *h, double *pbar, const void *p, double Xphi, double XA, bool set)
{
  U1Sector *u = h->u1;
  const double c = 2.0 * u->prm.inv_n3;
  if (u->fp32)
    k_u1_pbar_axpy<float><<<kU1Blocks, 256, 0, h->stream>>>(pbar, static_cast<const float *>(p), h->n3, c * Xphi,
                                                             c * XA, set ? 1 : 0);
  else
    k_u1_pbar_axpy<double><<<kU1Blocks, 256, 0, h->stream>>>(pbar, static_cast<const double *>(p), h->n3, c * Xphi,
                                                              c * XA, set ? 1 : 0);
}

// The backward pass of the leapfrog (LeapFrog::evolve, leapfrog.h:42-89, then sync, :96-116).
// Boundary n is the state before step n's kick: fields f_n, momenta p_{n-1/2}; boundary N the
// state before the sync.  One adjoint sweep per boundary: part A is the kick at f_n (w dt; dt/2
// for the sync, 1/2 of dt for a first step right after a sync), part B the drift of step n - 1
// (no kick: hB = 0).  The scale-factor chain of step n - 1 (a-drift, aDot kick with
// F(a_{n-1}; <.>)) is reversed on the host after boundary n's sweep; its <pi^2> inputs are the
// means of the averages of p_{n-3/2} and p_{n-1/2} (leapfrog.h:152-167), so the cotangent of
// boundary n's momentum average is complete only then, and is added to the sweep's output by
// pbar_axpy.  The sweep's dot products do not depend on it (hB = 0).
int u1_backward_lf(clb_handle *h, int32_t through_init, double *fields_bar, double *momenta_bar,
                   clb_adjoint_grad *out)
{
  U1Sector *u = h->u1;
  const U1Params &prm = u->prm;
  const bool ex = h->cfg.expansion != 0;
  const double dt = h->cfg.dt, al = prm.alpha, el = prm.el0, inv = prm.inv_n3;
  const size_t bytes = 5 * h->n3 * sizeof(double);
  cudaError_t e = cudaSuccess;
  double thg = 0, thc = 0, Sd[kAdjSlots];
  int cur = 0, r = CLB_OK;
  // seed at the synced end state: O = sum_k w_k E_k / E_tot, or a spectrum observable
  double E[kAvgN], Et = 0, Ew = 0, Aend[kAvgN] = {0, 0, 0, 0, 0}, abar = 0;
  {
    const double a = u->fwd_a;
    energies_of(prm, a, u->fwd_avg, E);
    for (int k = 0; k < kAvgN; ++k) {
      Et += E[k];
      Ew += u->fwd_w[k] * E[k];
    }
    double Ebar[kAvgN];
    for (int k = 0; k < kAvgN; ++k) Ebar[k] = u->seed_which >= 0 ? 0.0 : (u->fwd_w[k] - Ew / Et) / Et;
    Aend[0] = Ebar[0] * std::pow(a, -6);
    Aend[1] = Ebar[1] * std::pow(a, -2);
    Aend[2] = Ebar[2] * el * std::pow(a, -4);
    Aend[3] = Ebar[3] * el * std::pow(a, -4);
    Aend[4] = Ebar[4];
    abar = ex ? Ebar[0] * u->fwd_avg[0] * -6 * std::pow(a, -7) + Ebar[1] * u->fwd_avg[1] * -2 * std::pow(a, -3) +
                    (Ebar[2] * u->fwd_avg[2] + Ebar[3] * u->fwd_avg[3]) * el * -4 * std::pow(a, -5)
              : 0.0;
    if (u->seed_which >= 0) abar = ex ? u->seed_abar : 0.0;
  }
  // cotangents of the synced end state: fields (qbar), momenta p_N (the sync kick's lambda_A)
  const U1Sector::Ckpt &end = u->ckpt.back();
  if ((e = cudaMemsetAsync(u->qbar, 0, bytes, h->stream)) != cudaSuccess) return h->cuda_fail(e, "clb_backward");
  pbar_axpy(h, u->pbar[cur], end.p, Aend[0], Aend[2], true);
  if (u->seed_which >= 0) {
    double *dst = (u->seed_which == 0 ? u->qbar : u->pbar[cur]) + (size_t)u->seed_comp * h->n3;
    if ((e = cudaMemcpyAsync(dst, u->seed, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_backward");
  }
  double fieldA[3] = {Aend[1], Aend[3], Aend[4]}; // <|D phi|^2>, <B^2>, <V> cotangents at the next boundary's fields
  double adbar = 0;                               // cotangent of aDot_{n-1/2} (the sync's aDot enters no energy)
  double piHalf[2] = {0, 0};                      // part of the cotangent of <pi^2>(p_{n-1/2}) from step n's F
  const int64_t N = u->fwd_steps, K = u->fwd_K;
  const int64_t nck = (int64_t)u->ckpt.size() - 1;
  const size_t half = 5 * h->n3 * u->esz;
  SegSave sv{u->seg, half, u->d_rec};
  auto segf = [&](int64_t b) -> void * { return u->seg + (size_t)b * 2 * half; };
  auto segp = [&](int64_t b) -> void * { return u->seg + (size_t)b * 2 * half + half; };
  std::vector<U1State> rec((size_t)u->seg_cap);
  for (int64_t c = nck - 1; c >= 0; --c) {
    const int64_t s0 = c * K, s1 = std::min(N, s0 + K), nb = s1 - s0;
    U1Sector::Ckpt &ck = u->ckpt[(size_t)c];
    if ((e = copy_state(h, ck.f, ck.p, true)) != cudaSuccess ||
        (e = cudaMemcpyAsync(u->d_st, &ck.st, sizeof(U1State), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_backward");
    h->synced = c == 0 && u->fwd_w0 == 0.5;
    lf_run(h, nb, &sv);
    e = cudaMemcpyAsync(rec.data(), u->d_rec, (size_t)(nb + 1) * sizeof(U1State), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_backward");
    // a_n at boundary b: before step b's a-drift; the segment's end from its last step
    auto a_at = [&](int64_t b) { return ex ? (b < nb ? rec[(size_t)b].aIM : rec[(size_t)nb - 1].aI) : rec[0].aI; };
    for (int64_t b = nb; b >= (c == 0 ? 0 : 1); --b) {
      const int64_t n = s0 + b;
      const double an = a_at(b);
      U1AdjArgs g = adj_base(prm, an);
      const double wA = n == N ? 0.5 : (n == 0 ? u->fwd_w0 : 1.0);
      g.hA[0] = g.hA[1] = wA * dt;
      double aS = 0;
      if (b >= 1) {
        aS = rec[(size_t)b - 1].aSI;
        g.cdf = dt * std::pow(aS, al - 3);
        g.cda = dt * std::pow(aS, al - 1);
      }
      double piPrev[2] = {piHalf[0], piHalf[1]}; // cotangent of <pi^2>(p_{n-1/2}) so far
      if (n == 0 && ex && u->fwd_fresh) {
        // clb_initialize's aDot_{-1/2} = aDot_0 - dt/2 F(a_0, <.>_0) (leapfrog.h:35) and, through_init,
        // aDot_0 = sqrt(RHS(a_0, <.>_0)) (modelinitializer.h:77-80); <pi^2>_0 of the start momenta,
        // the field averages of f_0
        const U1State &R0 = ck.st;
        double A0[kAvgN], Ain[kAvgN] = {0, 0, 0, 0, 0};
        averages_of(R0, A0);
        const double a0 = an, ad0bar = adbar;
        const SFGrad gc = sf_grad(prm, a0, A0);
        const double Fc = -dt / 2.0 * ad0bar;
        abar += Fc * gc.da;
        for (int k = 0; k < kAvgN; ++k) Ain[k] += Fc * gc.dA[k];
        if (through_init && u->init_corrected) {
          const double C = std::pow(a0, 2 * al + 2) / 3.0 * prm.fm2, dC = (2 * al + 2) * std::pow(a0, 2 * al + 1) / 3.0 * prm.fm2;
          const double rho = A0[0] * std::pow(a0, -6) + A0[1] * std::pow(a0, -2) + el * std::pow(a0, -4) * (A0[2] + A0[3]) + A0[4];
          const double drho = A0[0] * -6 * std::pow(a0, -7) + A0[1] * -2 * std::pow(a0, -3) + el * -4 * std::pow(a0, -5) * (A0[2] + A0[3]);
          const double RHSbar = ad0bar / (2 * R0.aDotI);
          abar += RHSbar * (dC * rho + C * drho);
          Ain[0] += RHSbar * C * std::pow(a0, -6);
          Ain[1] += RHSbar * C * std::pow(a0, -2);
          Ain[2] += RHSbar * C * el * std::pow(a0, -4);
          Ain[3] += RHSbar * C * el * std::pow(a0, -4);
          Ain[4] += RHSbar * C;
        }
        fieldA[0] += Ain[1];
        fieldA[1] += Ain[3];
        fieldA[2] += Ain[4];
        piPrev[0] += Ain[0];
        piPrev[1] += Ain[2];
        adbar = through_init && u->init_corrected ? 0.0 : ad0bar; // then the cotangent of aDotI at the start
      }
      g.AD = fieldA[0];
      g.AB = fieldA[1];
      g.AV = fieldA[2];
      if ((r = adj_sweep(h, segf(b), segp(b), u->pbar[cur], u->pbar[cur ^ 1], g, Sd)) != CLB_OK) return r;
      cur ^= 1;
      thg += Sd[2] + g.AD * inv * Sd[4];
      thc += Sd[3] + g.AV * inv * Sd[5];
      if (ex) abar += Sd[0]; // a_n in the kick coefficients
      for (double &x : fieldA) x = 0;
      piHalf[0] = piHalf[1] = 0;
      if (b >= 1 && ex) {
        // step n - 1 backwards: f_n = f_{n-1} + dt D(aS) p (the sweep's dots 6, 7), a_n = a_{n-1} +
        // dt aDot_{n-1/2}, aS = (a_{n-1} + a_n)/2, aDot_{n-1/2} = aDot_{n-3/2} + dt F(a_{n-1}; <.>)
        const double aSbar = dt * ((al - 3) * std::pow(aS, al - 4) * Sd[6] + (al - 1) * std::pow(aS, al - 2) * Sd[7]);
        const double abar_n = abar + aSbar / 2;
        adbar += dt * abar_n;
        abar = abar_n + aSbar / 2;
        const U1State &R = rec[(size_t)b - 1];
        double A[kAvgN];
        averages_of(R, A); // <pi^2> the mean over p_{n-3/2}, p_{n-1/2}; the fields' of f_{n-1}
        const SFGrad g1 = sf_grad(prm, R.aIM, A);
        const double Fbar = dt * adbar;
        abar += Fbar * g1.da;
        piPrev[0] += 0.5 * Fbar * g1.dA[0];
        piPrev[1] += 0.5 * Fbar * g1.dA[2];
        piHalf[0] = 0.5 * Fbar * g1.dA[0];
        piHalf[1] = 0.5 * Fbar * g1.dA[2];
        fieldA[0] = Fbar * g1.dA[1];
        fieldA[1] = Fbar * g1.dA[3];
        fieldA[2] = Fbar * g1.dA[4];
      }
      // the momentum average of this boundary's momenta p_{n-1/2} (step n's <pi^2> of the previous
      // half step, and step n - 1's own; at n = 0 the start momenta's only right after
      // clb_initialize, where the stored average is theirs)
      if (ex && (b >= 1 || u->fwd_fresh)) pbar_axpy(h, u->pbar[cur], segp(b), piPrev[0], piPrev[1], false);
    }
  }
  {
    const U1Sector::Ckpt &fin = u->ckpt.back();
    if ((e = copy_state(h, fin.f, fin.p, true)) != cudaSuccess ||
        (e = cudaMemcpyAsync(u->d_st, &fin.st, sizeof(U1State), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_backward");
  }
  h->synced = true;
  if (fields_bar) e = cudaMemcpyAsync(fields_bar, u->qbar, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess && momenta_bar) e = cudaMemcpyAsync(momenta_bar, u->pbar[cur], bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_backward");
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->dO_dcouplings[0] = thc;
    out->dO_dcouplings[1] = thg;
    out->dO_dscalefactor[0] = ex ? abar : 0.0;
    // aDotI at the start (after clb_initialize; a later start: the half-step aDot before it)
    out->dO_dscalefactor[1] = ex ? adbar : 0.0;
    out->observable = u->fwd_obs;
  }
  return check(h, "clb_backward");
}
} // namespace

__attribute__((visibility("hidden"))) int u1_backward(clb_handle *h, int32_t through_init, double *fields_bar,
                                                      double *momenta_bar, clb_adjoint_grad *out)
{
  U1Sector *u = h->u1;
  if (u->fwd_steps < 0) return h->fail(CLB_ESTATE, "clb_backward: call clb_forward first");
  if (h->cfg.evolver == CLB_LF) return u1_backward_lf(h, through_init, fields_bar, momenta_bar, out);
  const U1Params &prm = u->prm;
  const bool ex = h->cfg.expansion != 0;
  const double dt = h->cfg.dt, al = prm.alpha, el = prm.el0;
  const size_t bytes = 5 * h->n3 * sizeof(double); // cotangents are FP64 in either form
  const std::vector<double> &ws = h->ws;
  const size_t P = ws.size();
  const int64_t S = 2 * (int64_t)P - 1;
  auto wof = [&](int64_t i) { return ws[(size_t)i < P ? (size_t)i : (size_t)(S - i - 1)]; };
  cudaError_t e = cudaSuccess;
  double thg = 0, thc = 0; // explicit d/dgQ, d/dc4
  double Sd[kAdjSlots];
  int cur = 0;
  int r = CLB_OK;
  // seed: O = sum_k w_k E_k / E_tot at the final state
  double E[kAvgN], Et = 0, Ew = 0;
  energies_of(prm, u->fwd_a, u->fwd_avg, E);
  for (int k = 0; k < kAvgN; ++k) {
    Et += E[k];
    Ew += u->fwd_w[k] * E[k];
  }
  double Ebar[kAvgN];
  for (int k = 0; k < kAvgN; ++k) Ebar[k] = u->seed_which >= 0 ? 0.0 : (u->fwd_w[k] - Ew / Et) / Et;
  // part A pending at the next boundary to process: the transposed first kick of the stage that
  // starts there (or the observable's seed, with no kick), its average cotangents, and the
  // cotangents of a and aDot there before its a-dot products are added
  struct PendA {
    bool on;
    double h[2];
    double Abar[kAvgN];
    double abar, adbar;
  } pend{};
  {
    const double a = u->fwd_a;
    pend.on = true;
    pend.Abar[0] = Ebar[0] * std::pow(a, -6);
    pend.Abar[1] = Ebar[1] * std::pow(a, -2);
    pend.Abar[2] = Ebar[2] * el * std::pow(a, -4);
    pend.Abar[3] = Ebar[3] * el * std::pow(a, -4);
    pend.Abar[4] = Ebar[4];
    pend.abar = ex ? Ebar[0] * u->fwd_avg[0] * -6 * std::pow(a, -7) + Ebar[1] * u->fwd_avg[1] * -2 * std::pow(a, -3) +
                         (Ebar[2] * u->fwd_avg[2] + Ebar[3] * u->fwd_avg[3]) * el * -4 * std::pow(a, -5)
                   : 0.0;
    if (u->seed_which >= 0) pend.abar = ex ? u->seed_abar : 0.0;
    pend.adbar = 0;
  }
  double abar = 0, adbar = 0; // cotangents of a, aDot at the boundary just processed
  if ((e = cudaMemsetAsync(u->qbar, 0, bytes, h->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(u->pbar[cur], 0, bytes, h->stream)) != cudaSuccess)
    return h->cuda_fail(e, "clb_backward");
  if (u->seed_which >= 0) {
    // a spectrum observable: its gradient with respect to one component at the end state
    double *dst = (u->seed_which == 0 ? u->qbar : u->pbar[cur]) + (size_t)u->seed_comp * h->n3;
    if ((e = cudaMemcpyAsync(dst, u->seed, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_backward");
  }
  std::vector<U1State> rec((size_t)u->seg_cap);
  const int64_t nck = (int64_t)u->ckpt.size() - 1; // the last entry holds the forward's end state
  const size_t half = 5 * h->n3 * u->esz;
  SegSave sv{u->seg, half, u->d_rec};
  auto segf = [&](int64_t b) -> void * { return u->seg + (size_t)b * 2 * half; };
  auto segp = [&](int64_t b) -> void * { return u->seg + (size_t)b * 2 * half + half; };
  for (int64_t c = nck - 1; c >= 0; --c) {
    const int64_t s0 = c * u->fwd_K, s1 = std::min(u->fwd_steps, s0 + u->fwd_K);
    const int64_t nb = (s1 - s0) * S; // stages in this segment
    // recompute the segment from its checkpoint, keeping every boundary state and record
    U1Sector::Ckpt &ck = u->ckpt[(size_t)c];
    if ((e = copy_state(h, ck.f, ck.p, true)) != cudaSuccess ||
        (e = cudaMemcpyAsync(u->d_st, &ck.st, sizeof(U1State), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_backward");
    vv_run(h, s1 - s0, &sv);
    e = cudaMemcpyAsync(rec.data(), u->d_rec, (size_t)(nb + 1) * sizeof(U1State), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "clb_backward");
    for (int64_t b = nb; b >= 0; --b) {
      const U1State &Rb = rec[(size_t)b];
      double Ab[kAvgN];
      averages_of(Rb, Ab);
      const double ab = Rb.aI; // without expansion a stays at its set value
      U1AdjArgs g = adj_base(prm, ab);
      double AD = 0, AB = 0, AV = 0;
      const bool partA = pend.on, partB = b >= 1;
      const bool init = partA && c == 0 && b == 0 && through_init && ex;
      double Ib[kAvgN] = {0, 0, 0, 0, 0}, RHSbar = 0;
      if (init) {
        // aDot0 = sqrt(RHS), RHS = a^{2 alpha + 2}/3 fm2 rho(<.>)  (hubbleconstraint.h:27-36): its
        // average cotangents join part A's at the start state
        const double C = std::pow(ab, 2 * al + 2) / 3.0 * prm.fm2;
        RHSbar = pend.adbar / (2 * Rb.aDotI);
        Ib[0] = RHSbar * C * std::pow(ab, -6);
        Ib[1] = RHSbar * C * std::pow(ab, -2);
        Ib[2] = Ib[3] = RHSbar * C * el * std::pow(ab, -4);
        Ib[4] = RHSbar * C;
      }
      if (partA) {
        g.hA[0] = pend.h[0];
        g.hA[1] = pend.h[1];
        g.ApiA = pend.Abar[0] + Ib[0];
        g.AEA = pend.Abar[2] + Ib[2];
        AD += pend.Abar[1] + Ib[1];
        AB += pend.Abar[3] + Ib[3];
        AV += pend.Abar[4] + Ib[4];
      }
      // part B: the stage b - 1 ending here, maps 6 (aDot1 = aDotS + dt/2 w F(a1, <.>1)), 5 and 4
      const int64_t sb = b - 1;
      const double wB = partB ? wof(sb % S) : 0.0, dtwB = dt * wB;
      const double adbar_b = partA ? pend.adbar : adbar; // aDot cotangent at this boundary
      double F6 = 0, A1bar[kAvgN] = {0, 0, 0, 0, 0};
      SFGrad g1{};
      const double aS = Rb.aSI; // the stage ending here set aSI
      if (partB) {
        g.hB[0] = dt / 2 * wB;
        g.hB[1] = dt * wB / 2;
        if (ex) {
          g1 = sf_grad(prm, ab, Ab);
          F6 = dt / 2 * wB * adbar_b;
          for (int k = 0; k < kAvgN; ++k) A1bar[k] = F6 * g1.dA[k];
        }
        g.ApiB = A1bar[0];
        g.AEB = A1bar[2];
        AD += A1bar[1];
        AB += A1bar[3];
        AV += A1bar[4];
        g.cdf = dtwB * std::pow(aS, al - 3);
        g.cda = dtwB * std::pow(aS, al - 1);
      }
      g.AD = AD;
      g.AB = AB;
      g.AV = AV;
      if ((r = adj_sweep(h, segf(b), segp(b), u->pbar[cur], u->pbar[cur ^ 1], g, Sd)) != CLB_OK) return r;
      cur ^= 1;
      thg += Sd[2] + AD * prm.inv_n3 * Sd[4];
      thc += Sd[3] + AV * prm.inv_n3 * Sd[5];
      if (partA) {
        abar = ex ? pend.abar + Sd[0] : 0.0;
        adbar = pend.adbar;
        pend.on = false;
      }
      if (init) {
        const double C = std::pow(ab, 2 * al + 2) / 3.0 * prm.fm2, dC = (2 * al + 2) * std::pow(ab, 2 * al + 1) / 3.0 * prm.fm2;
        const double rho = Ab[0] * std::pow(ab, -6) + Ab[1] * std::pow(ab, -2) + el * std::pow(ab, -4) * (Ab[2] + Ab[3]) + Ab[4];
        const double drho = Ab[0] * -6 * std::pow(ab, -7) + Ab[1] * -2 * std::pow(ab, -3) + el * -4 * std::pow(ab, -5) * (Ab[2] + Ab[3]);
        abar += RHSbar * (dC * rho + C * drho);
        adbar = 0;
      }
      if (partB) {
        // the rest of stage b - 1: maps 6, 4, 3 and 1; its part A is pending at boundary b - 1
        pend.on = true;
        pend.h[0] = dt / 2 * wB;
        pend.h[1] = dt * wB / 2;
        for (int k = 0; k < kAvgN; ++k) pend.Abar[k] = 0;
        pend.abar = pend.adbar = 0;
        if (ex) {
          double abar1 = abar + F6 * g1.da + Sd[1];
          double adS = adbar_b;
          const double aSbar = dtwB * ((al - 3) * std::pow(aS, al - 4) * Sd[6] + (al - 1) * std::pow(aS, al - 2) * Sd[7]);
          // map 3: a1 = a0 + dt w aDotS, aS = (a0 + a1)/2
          abar1 += aSbar / 2;
          double abar0 = aSbar / 2 + abar1;
          adS += dtwB * abar1;
          // map 1: aDotS = aDot0 + dt/2 w F(a0, <.>0)
          const U1State &R0 = rec[(size_t)sb];
          double A0[kAvgN];
          averages_of(R0, A0);
          const SFGrad g0 = sf_grad(prm, R0.aI, A0);
          const double F1 = dt / 2 * wB * adS;
          abar0 += F1 * g0.da;
          for (int k = 0; k < kAvgN; ++k) pend.Abar[k] = F1 * g0.dA[k];
          pend.abar = abar0;
          pend.adbar = adS;
        }
      }
    }
  }
  // leave the live state at the forward's end again
  {
    const U1Sector::Ckpt &end = u->ckpt.back();
    if ((e = copy_state(h, end.f, end.p, true)) != cudaSuccess ||
        (e = cudaMemcpyAsync(u->d_st, &end.st, sizeof(U1State), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
      return h->cuda_fail(e, "clb_backward");
  }
  if (fields_bar) e = cudaMemcpyAsync(fields_bar, u->qbar, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess && momenta_bar) e = cudaMemcpyAsync(momenta_bar, u->pbar[cur], bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_backward");
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->dO_dcouplings[0] = thc;
    out->dO_dcouplings[1] = thg;
    out->dO_dscalefactor[0] = ex ? abar : 0.0;
    out->dO_dscalefactor[1] = ex ? adbar : 0.0;
    out->observable = u->fwd_obs;
  }
  return check(h, "clb_backward");
}

// The observable of the last u1_forward becomes a spectrum observable O with the given cotangent
// of component comp of the fields (which 0) or momenta (which 1) at the end state (N^3, device)
// and of a there (clb_forward_spectrum).
__attribute__((visibility("hidden"))) int u1_set_spectrum_seed(clb_handle *h, int which, int comp, const double *d_grad,
                                                               double O, double abar)
{
  U1Sector *u = h->u1;
  if (u->fwd_steps < 0) return h->fail(CLB_ESTATE, "clb_forward_spectrum: no forward pass");
  cudaError_t e = cudaSuccess;
  if (!u->seed) e = cudaMalloc(&u->seed, h->n3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(u->seed, d_grad, h->n3 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "clb_forward_spectrum");
  u->seed_which = which;
  u->seed_comp = comp;
  u->seed_abar = abar;
  u->fwd_obs = O;
  return CLB_OK;
}

// Device array of one state component (clb_spectrum): which 0 fields, 1 momenta; gauge tells
// whether the component belongs to the U(1) field.
__attribute__((visibility("hidden"))) const double *u1_component(clb_handle *h, int which, int comp, bool *gauge)
{
  U1Sector *u = h->u1;
  if (comp < 0 || comp >= 5) return nullptr;
  *gauge = comp >= 2;
  if (!u->fp32) return static_cast<const double *>(which == 0 ? u->f : u->p) + (size_t)comp * h->n3;
  // FP32 form: the component in FP64 in the staging buffer (ordered on the handle's stream)
  const float *src = static_cast<const float *>(which == 0 ? u->f : u->p) + (size_t)comp * h->n3;
  k_convert<float, double><<<kU1Blocks, 256, 0, h->stream>>>(src, u->d_stage, h->n3);
  return u->d_stage;
}

} // namespace clb
