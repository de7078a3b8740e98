// clb_u1.cu - complex scalar + U(1) gauge sector (lphi4U1) behind the libclb200 C ABI.
//
// Schedules restate VelocityVerlet::evolve (evolvers/velocityverlet.h:51-114, 140-210) and
// LeapFrog::evolve / sync (evolvers/leapfrog.h:42-116, 141-217) for a model with one complex
// scalar and one U(1) field.  The second kick of a VV stage and the first kick of the next use the
// same kernel (no field or scale-factor change in between), so they run as one sweep that applies
// both kicks in sequence and reduces the momenta after each; on the leapfrog the field averages of
// a step are reduced by the next step's kick sweep, which reads the same fields.

#include "clb_handle.cuh"
#include "clb_u1.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace clb {

namespace {
constexpr int kU1Blocks = 148 * 8; // grid-stride sweeps: 8 resident 256-thread blocks per SM
}

struct U1Sector {
  double *f = nullptr, *p = nullptr; // 5 x N^3 each
  U1State *d_st = nullptr;
  double *d_part = nullptr; // kU1Blocks x kU1Meas
  double *d_sums = nullptr; // kU1Meas
  U1Params prm{};
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

template <int NK, bool RF, bool RP> void kick(clb_handle *h, int kind, const U1Kick &kc)
{
  U1Sector *u = h->u1;
  CLB_LAUNCH(h, kind,
             k_u1_kick<NK, RF, RP><<<kU1Blocks, 256, 0, h->stream>>>(u->f, u->p, u->prm, kc, u->d_st, u->d_part));
}

void drift(clb_handle *h, double w)
{
  U1Sector *u = h->u1;
  CLB_LAUNCH(h, K_U1_DRIFT,
             k_u1_drift<<<kU1Blocks, 256, 0, h->stream>>>(u->f, u->p, h->n3, w, h->cfg.dt, u->d_st));
}

void tail(clb_handle *h, uint32_t flags, bool reduced, double w = 0, double w2 = 0, int64_t hist_row = -1)
{
  U1Sector *u = h->u1;
  TailOp op{flags, reduced ? kU1Blocks : 0, w, w2, hist_row >= 0 ? h->d_hist : nullptr, hist_row};
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

__attribute__((visibility("hidden"))) int u1_create(clb_handle *h)
{
  U1Sector *u = new U1Sector();
  h->u1 = u;
  h->NS = 5;
  u->prm = make_params(h);
  const size_t bytes = 5 * h->n3 * sizeof(double);
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc(&u->f, bytes) == cudaSuccess && cudaMalloc(&u->p, bytes) == cudaSuccess;
  ok = ok && cudaMemset(u->f, 0, bytes) == cudaSuccess && cudaMemset(u->p, 0, bytes) == cudaSuccess;
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

__attribute__((visibility("hidden"))) void u1_destroy(clb_handle *h)
{
  U1Sector *u = h->u1;
  if (!u) return;
  if (u->f) cudaFree(u->f);
  if (u->p) cudaFree(u->p);
  if (u->d_st) cudaFree(u->d_st);
  if (u->d_part) cudaFree(u->d_part);
  if (u->d_sums) cudaFree(u->d_sums);
  delete u;
  h->u1 = nullptr;
}

__attribute__((visibility("hidden"))) int u1_set_state(clb_handle *h, const double *fields, const double *momenta,
                                                       const clb_scalefactor *sf)
{
  U1Sector *u = h->u1;
  const size_t bytes = 5 * h->n3 * sizeof(double);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(u->f, fields, bytes, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(u->p, momenta, bytes, cudaMemcpyHostToDevice, h->stream);
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
  if (e == cudaSuccess && fields) e = cudaMemcpyAsync(fields, u->f, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess && momenta) e = cudaMemcpyAsync(momenta, u->p, bytes, cudaMemcpyDeviceToHost, h->stream);
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
  if (h->cfg.expansion && correct_adot) fl |= T_CORRECT_ADOT;
  if (h->cfg.expansion && h->cfg.evolver == CLB_LF) fl |= T_LF_CTOR;
  tail(h, fl, true);
  h->synced = true;
  return check(h, "clb_initialize");
}

__attribute__((visibility("hidden"))) int u1_evolve(clb_handle *h, int64_t nsteps)
{
  const double dt = h->cfg.dt;
  const bool ex = h->cfg.expansion != 0;
  cudaEventRecord(h->ev_call[0], h->stream);
  if (h->cfg.evolver == CLB_LF) {
    // LeapFrog::evolve: kick (1/2 dt after a sync), <pi^2>, a kick and drift, field drifts, field averages
    const double weight = h->synced ? 0.5 : 1.0;
    kick_sweep(h, 1, false, ex, lf_kick(dt, weight));
    if (ex) tail(h, T_STORE_PI2_LF | T_LF_KICK | T_LF_DRIFT, true);
    for (int64_t s = 0; s < nsteps; ++s) {
      drift(h, 1.0);
      if (s + 1 < nsteps) {
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
  } else {
    const std::vector<double> &ws = h->ws;
    const size_t P = ws.size(), S = 2 * P - 1;
    auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
    const int64_t total = nsteps * (int64_t)S;
    const double w0 = wof(0);
    if (ex) tail(h, T_VV_KICK_HALF, false, 0, w0); // kickScaleFactorHalf
    kick_sweep(h, 1, false, ex, vv_kick(dt, w0, 0.0));
    if (ex) tail(h, T_STORE_PI2_I | T_VV_DRIFT, true, 0, w0); // <pi^2>, driftScaleFactor
    for (int64_t k = 0; k < total; ++k) {
      const size_t i = (size_t)(k % (int64_t)S);
      const double w = wof(i);
      const bool more = k + 1 < total;
      const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
      drift(h, w);
      kick_sweep(h, more ? 2 : 1, ex, ex, vv_kick(dt, w, wn));
      if (ex) {
        uint32_t fl = T_STORE_FIELDS | T_STORE_PI2_I | T_VV_KICK_ONE;
        if (more) fl |= T_VV_KICK_HALF | T_STORE_PI2_B | T_VV_DRIFT;
        tail(h, fl, true, w, wn, i + 1 == S ? k / (int64_t)S : -1);
      }
    }
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
  if (h->cfg.evolver == CLB_LF && !h->synced) {
    kick_sweep(h, 1, false, h->cfg.expansion != 0, lf_kick(h->cfg.dt, 0.5));
    if (h->cfg.expansion) tail(h, T_STORE_PI2_I | T_LF_SYNC, true);
  }
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
  CLB_LAUNCH(h, K_MEASURE, k_u1_measure<<<kU1Blocks, 256, 0, h->stream>>>(u->f, u->p, u->prm, u->d_part));
  CLB_LAUNCH(h, K_MEASURE, k_sum_partials<kU1Meas><<<1, 256, 0, h->stream>>>(u->d_part, kU1Blocks, u->d_sums));
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

} // namespace clb
