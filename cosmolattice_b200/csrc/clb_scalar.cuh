// clb_scalar.cuh - sm_100a kernels of the scalar-singlet sector (lphi4 family).
//
// Layout: each real component is one N^3 array, row-major with x slowest and z fastest; the
// Ns fields of a state are contiguous components.  Periodic boundaries by index wrap (the
// reference's one-site ghost layer, source/cosmolattice.cpp:73-82, is not materialised).
//
// The stencil sweep marches along x.  A block owns a BY x BZ tile of (y, z) columns; the
// centre column's x-1, x, x+1 values sit in registers, the in-plane neighbours of plane x come
// from a triple-buffered shared-memory tile (with a one-site halo ring) that is filled while
// plane x-1 is still being read.  Each site's phi and pi are read from HBM once per sweep
// (halo re-reads are served by L2), and phi', pi' are written once.
#pragma once

#include "clb_internal.cuh"

#ifndef CLB_SCALAR_MODEL
#define CLB_SCALAR_MODEL_HEADER "models/lphi4.h"
#define CLB_SCALAR_MODEL lphi4
#endif
#include CLB_SCALAR_MODEL_HEADER

namespace clb {

using ScalarModel = clb_models::CLB_SCALAR_MODEL;
using ModelCouplings = ScalarModel::Couplings;
// The handle and the kernel arguments hold a model's couplings in a fixed 8-double slot, so the
// handle has one layout whichever header a build uses (the units that do not read the potential
// are shared between the builds).
static_assert(sizeof(ModelCouplings) <= 8 * sizeof(double), "a model header's Couplings holds at most 8 doubles");
union CouplingSlot {
  ModelCouplings mc;
  double pad[8];
};

struct ScalarArgs {
  int N;
  int LX;           // x planes per block
  double inv_dx2;   // 1 / (dx dx)                      (gaugederivatives.h:38)
  CouplingSlot cs;   // the model header's couplings (models/lphi4.h: c0, q, c0/4, q/2) in cs.mc
  double dtw;       // dt * w of the drift              (velocityverlet.h:183)
  double h1;        // first kick weight  (w dt / 2)    (velocityverlet.h:131)
  double h2;        // second kick weight (w' dt / 2), 0 when the sweep ends on a half kick
};

// ---- the scalar-singlet model's potential ----------------------------------------------------
// The potential, its derivatives and its terms come from a model header shaped like the
// reference's (potentialTerms / potDeriv / potDeriv2 per Tag: models/model_api.h), chosen when the
// library is built, as the reference chooses its model when it compiles (CMakeLists.txt:133-146).
// SPot evaluates the header's terms at one site in the arithmetic of Ar<R>: FP64 pins every
// rounding (the order the header writes, which the oracle shares).
template <class R, int NS> struct SPot {
  using M = ScalarModel;
  static __device__ __forceinline__ R dV(int f, const R (&v)[NS], const ModelCouplings &c)
  {
    return clb_models::pot_deriv<M, Ar<R>>(f, v, c);
  }
  static __device__ __forceinline__ R V(const R (&v)[NS], const ModelCouplings &c)
  {
    return clb_models::potential<M, Ar<R>>(v, c);
  }
  static __device__ __forceinline__ R Vterm(int k, const R (&v)[NS], const ModelCouplings &c)
  {
    return clb_models::potential_term<M, Ar<R>>(k, v, c);
  }
};

// phi + p (dtw pi) with the reference's rounding order (velocityverlet.h:183).  FP32: one FMA.
template <class R> __device__ __forceinline__ R drift_val(R f, R p, R pd, R dtw);
template <> __device__ __forceinline__ double drift_val<double>(double f, double p, double pd, double dtw)
{
  return __dadd_rn(f, __dmul_rn(pd, __dmul_rn(dtw, p)));
}
template <> __device__ __forceinline__ float drift_val<float>(float f, float p, float pd, float dtw)
{
  return fmaf(pd * dtw, p, f);
}

// pi + h1 K then + h2 K.  FP64: two rounded steps like the reference's two kicks.
// FP32 (compensated): both increments are added in FP64 and the result rounded once.
template <class R> struct KickOut {
  R next;
  double mid;
};
template <class R> __device__ __forceinline__ KickOut<R> kick_val(R p, R K, double h1, double h2);
template <> __device__ __forceinline__ KickOut<double> kick_val<double>(double p, double K, double h1, double h2)
{
  const double mid = __dadd_rn(p, __dmul_rn(h1, K));
  const double nxt = h2 == 0.0 ? mid : __dadd_rn(mid, __dmul_rn(h2, K));
  return {nxt, mid};
}
template <> __device__ __forceinline__ KickOut<float> kick_val<float>(float p, float K, double h1, double h2)
{
  const double Kd = (double)K;
  const double mid = (double)p + h1 * Kd;
  const double nxt = mid + h2 * Kd;
  return {(float)nxt, mid};
}

// ---- the stencil sweep ---------------------------------------------------------------------
// DRIFT: phi' = phi + p (dtw pi) on the fly at every stencil point, written to fout.
// KICK : pi' = pi + h1 K(phi') [+ h2 K(phi')], written to pout.
// RED  : bit 0 -> sum of pi_mid^2; bit 1 -> sum of grad^2(phi') and V(phi').
// fin/pin are never written (fout/pout alias them only when !DRIFT, where each site's pi is
// read and written by its own thread alone).
template <class R, int NS, int BZ, int BY, bool DRIFT, bool KICK, int RED>
__global__ void __launch_bounds__(BZ *BY)
    k_scalar_sweep(const R *fin, const R *pin, R *fout, R *pout, ScalarArgs a, const DevState *__restrict__ st,
                   double *__restrict__ partials)
{
  using A = Ar<R>;
  using Pot = SPot<R, NS>;
  __shared__ R tile[3][NS][BY + 2][BZ + 2];
  __shared__ double red_smem[(BZ * BY / 32) * kRedSlots];

  const int N = a.N;
  const size_t n3 = (size_t)N * N * N;
  const int tz = threadIdx.x, ty = threadIdx.y;
  const int z0 = blockIdx.x * BZ, y0 = blockIdx.y * BY;
  const int hz = min(BZ, N - z0), hy = min(BY, N - y0);
  const int x0 = blockIdx.z * a.LX;
  const int x1 = min(N, x0 + a.LX);
  const bool valid = tz < hz && ty < hy;
  const int y = y0 + ty, z = z0 + tz;
  const int ym = y0 == 0 ? N - 1 : y0 - 1;
  const int yp = y0 + hy == N ? 0 : y0 + hy;
  const int zm = z0 == 0 ? N - 1 : z0 - 1;
  const int zp = z0 + hz == N ? 0 : z0 + hz;

  R pd = R(0), dtw = R(0), KA = R(0), KB = R(0);
  if (DRIFT) {
    pd = (R)st->drift_p;
    dtw = (R)a.dtw;
  }
  if (KICK) {
    KA = (R)st->kick_A;
    KB = (R)st->kick_B;
  }
  const R inv_dx2 = (R)a.inv_dx2;
  const R two = R(2);

  auto sidx = [&](int x, int yy, int zz) -> size_t { return ((size_t)x * N + yy) * N + zz; };
  auto ld = [&](int f, size_t s) -> R {
    R v = fin[f * n3 + s];
    if (DRIFT) v = drift_val<R>(v, pin[f * n3 + s], pd, dtw);
    return v;
  };

  double acc_pi2 = 0, acc_g2 = 0, acc_v = 0;
  R prev[NS], cur[NS], nxt[NS], piC[NS], piN[NS];

  if (x0 < x1) {
    const int xm = x0 == 0 ? N - 1 : x0 - 1;
    if (valid) {
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        prev[f] = ld(f, sidx(xm, y, z));
        cur[f] = ld(f, sidx(x0, y, z));
        tile[0][f][ty + 1][tz + 1] = cur[f];
        if (ty == 0) tile[0][f][0][tz + 1] = ld(f, sidx(x0, ym, z));
        if (ty == hy - 1) tile[0][f][hy + 1][tz + 1] = ld(f, sidx(x0, yp, z));
        if (tz == 0) tile[0][f][ty + 1][0] = ld(f, sidx(x0, y, zm));
        if (tz == hz - 1) tile[0][f][ty + 1][hz + 1] = ld(f, sidx(x0, y, zp));
        if (KICK || (RED & 1)) piC[f] = pin[f * n3 + sidx(x0, y, z)];
      }
    }
    int b = 0;
    for (int x = x0; x < x1; ++x) {
      const int bn = b == 2 ? 0 : b + 1;
      const int xn = x + 1 == N ? 0 : x + 1;
      const bool last = x + 1 == x1;
      if (valid) {
#pragma unroll
        for (int f = 0; f < NS; ++f) {
          nxt[f] = ld(f, sidx(xn, y, z));
          if (!last) {
            tile[bn][f][ty + 1][tz + 1] = nxt[f];
            if (ty == 0) tile[bn][f][0][tz + 1] = ld(f, sidx(xn, ym, z));
            if (ty == hy - 1) tile[bn][f][hy + 1][tz + 1] = ld(f, sidx(xn, yp, z));
            if (tz == 0) tile[bn][f][ty + 1][0] = ld(f, sidx(xn, y, zm));
            if (tz == hz - 1) tile[bn][f][ty + 1][hz + 1] = ld(f, sidx(xn, y, zp));
            if (KICK || (RED & 1)) piN[f] = pin[f * n3 + sidx(xn, y, z)];
          }
        }
      }
      __syncthreads();
      if (valid) {
        const size_t s = sidx(x, y, z);
        double site_pi2 = 0;
#pragma unroll
        for (int f = 0; f < NS; ++f) {
          if (DRIFT) fout[f * n3 + s] = cur[f];
          if (KICK) {
            const R c = cur[f];
            const R tx = A::sub(A::add(nxt[f], prev[f]), A::mul(two, c));
            const R tyv = A::sub(A::add(tile[b][f][ty + 2][tz + 1], tile[b][f][ty][tz + 1]), A::mul(two, c));
            const R tzv = A::sub(A::add(tile[b][f][ty + 1][tz + 2], tile[b][f][ty + 1][tz]), A::mul(two, c));
            const R lap = A::mul(inv_dx2, A::add(A::add(tx, tyv), tzv));
            const R K = A::sub(A::mul(KA, lap), A::mul(KB, Pot::dV(f, cur, a.cs.mc)));
            const KickOut<R> ko = kick_val<R>(piC[f], K, a.h1, a.h2);
            pout[f * n3 + s] = ko.next;
            if (RED & 1) site_pi2 = f == 0 ? ko.mid * ko.mid : site_pi2 + ko.mid * ko.mid;
          } else if (RED & 1) {
            const double pc = (double)piC[f];
            site_pi2 = f == 0 ? pc * pc : site_pi2 + pc * pc;
          }
          if (RED & 2) {
            const R c = cur[f];
            const R gx = A::sub(nxt[f], c);
            const R gy = A::sub(tile[b][f][ty + 2][tz + 1], c);
            const R gz = A::sub(tile[b][f][ty + 1][tz + 2], c);
            const R g2 = A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
            acc_g2 += (double)g2;
          }
        }
        if (RED & 1) acc_pi2 += site_pi2;
        if (RED & 2) acc_v += (double)Pot::V(cur, a.cs.mc);
      }
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        prev[f] = cur[f];
        cur[f] = nxt[f];
        if (KICK || (RED & 1)) piC[f] = piN[f];
      }
      b = bn;
    }
  }

  if (RED) {
    double v[kRedSlots] = {acc_pi2, acc_g2, acc_v};
    block_reduce<kRedSlots, BZ * BY>(v, red_smem);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) {
      const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
      for (int k = 0; k < kRedSlots; ++k) partials[bid * kRedSlots + k] = v[k];
    }
  }
}

// ---- elementwise kernels --------------------------------------------------------------------
// Drift of every component in place: phi += p (dtw pi)  (velocityverlet.h:181-184).
// With FP32 split storage (padded layout) the first thread also advances the FP64 references
// from slot rs into slot rs ^ 1 (ns fields).
template <class R>
__global__ void __launch_bounds__(256)
    k_drift(R *fld, const R *pi, size_t n, double dtw, const DevState *__restrict__ st, int rs = 0, int ns = 0)
{
  const R pd = (R)st->drift_p, w = (R)dtw;
  if (sizeof(R) == 4 && ns > 0 && blockIdx.x == 0 && threadIdx.x == 0) {
    DevState *sw = const_cast<DevState *>(st); // slot rs ^ 1 is read by nobody during this launch
    for (int f = 0; f < ns; ++f) {
      sw->ref_phi[rs ^ 1][f] = __dadd_rn(st->ref_phi[rs][f], __dmul_rn(st->drift_p, __dmul_rn(dtw, st->ref_pi[rs][f])));
      sw->ref_pi[rs ^ 1][f] = st->ref_pi[rs][f];
    }
  }
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    fld[i] = drift_val<R>(fld[i], pi[i], pd, w);
}

// Sum over sites of sum_f pi_f^2 into slot 0 of each block's partial row.
template <class R, int NS>
__global__ void __launch_bounds__(256) k_reduce_pi2(const R *pi, size_t n3, double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * kRedSlots];
  double acc = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    double v = 0;
#pragma unroll
    for (int f = 0; f < NS; ++f) {
      const double p = (double)pi[f * n3 + i];
      v = f == 0 ? p * p : v + p * p;
    }
    acc += v;
  }
  double v[kRedSlots] = {acc, 0.0, 0.0};
  block_reduce<kRedSlots, 256>(v, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kRedSlots; ++k) partials[(size_t)blockIdx.x * kRedSlots + k] = v[k];
}

// Measurement sums per field f (slot 6f + {pi^2, grad^2, phi, phi^2, mom, mom^2}) and potential
// terms (slot 6 NS + k), for EnergiesMeasurer / MeansMeasurer.  Plain stencil reads (rare).
template <class R, int NS>
__global__ void __launch_bounds__(256)
    k_measure(const R *fld, const R *pi, ScalarArgs a, double am, double *__restrict__ partials)
{
  using A = Ar<R>;
  using Pot = SPot<R, NS>;
  __shared__ double smem[(256 / 32) * kMeasSlots];
  const int N = a.N;
  const size_t n3 = (size_t)N * N * N;
  const R inv_dx2 = (R)a.inv_dx2;
  double acc[kMeasSlots];
#pragma unroll
  for (int k = 0; k < kMeasSlots; ++k) acc[k] = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i / ((size_t)N * N));
    const int y = (int)((i / N) % N);
    const int z = (int)(i % N);
    const size_t ix = ((size_t)(x + 1 == N ? 0 : x + 1) * N + y) * N + z;
    const size_t iy = ((size_t)x * N + (y + 1 == N ? 0 : y + 1)) * N + z;
    const size_t iz = ((size_t)x * N + y) * N + (z + 1 == N ? 0 : z + 1);
    R v[NS];
#pragma unroll
    for (int f = 0; f < NS; ++f) {
      const R c = fld[f * n3 + i];
      v[f] = c;
      const R gx = A::sub(fld[f * n3 + ix], c), gy = A::sub(fld[f * n3 + iy], c), gz = A::sub(fld[f * n3 + iz], c);
      const R g2 = A::mul(A::add(A::add(A::mul(gx, gx), A::mul(gy, gy)), A::mul(gz, gz)), inv_dx2);
      const double p = (double)pi[f * n3 + i];
      const double m = p * am;
      acc[6 * f + 0] += p * p;
      acc[6 * f + 1] += (double)g2;
      acc[6 * f + 2] += (double)c;
      acc[6 * f + 3] += (double)c * (double)c;
      acc[6 * f + 4] += m;
      acc[6 * f + 5] += m * m;
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) acc[6 * NS + k] += (double)Pot::Vterm(k, v, a.cs.mc);
  }
  block_reduce<kMeasSlots, 256>(acc, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kMeasSlots; ++k) partials[(size_t)blockIdx.x * kMeasSlots + k] = acc[k];
}

// ---- tail: fixed-order reduction of the block partials and the scale-factor update --------------
// x^e of the scale-factor bookkeeping.  The exponents are alpha + k; alpha is an integer in every
// model here (lphi4.h:125), and an integer power is a short multiply chain where pow() is a long
// serial one on the single tail thread (both within an ulp of x^e).
#ifndef CLB_TAIL_IPOW
#define CLB_TAIL_IPOW 1
#endif
__device__ __forceinline__ double apow(double x, double e)
{
  if (CLB_TAIL_IPOW && e == rint(e) && fabs(e) <= 8.0) return ipow_d(x, (int)e);
  return pow(x, e);
}

__device__ __forceinline__ double sf_kernel(const DevState &s, const SFParams &p)
{
  // ScaleFactorKernels::get (scalefactorkernels.h:73-77), scalar singlets:
  // kineticS = 0.5 <pi^2> a^-6, gradientS = 0.5 <grad^2> a^-2 (energies.h:37-45)
  const double al = p.alpha;
  const double Eks = __dmul_rn(0.5 * s.pi2AvI, ipow_d(s.aI, -6));
  const double Egs = __dmul_rn(0.5 * s.grad2AvI, ipow_d(s.aI, -2));
  const double br = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(al - 2, Eks), __dmul_rn(al, Egs)), __dmul_rn(al - 1, 0.0)),
                              __dmul_rn(al + 1, s.potAvI));
  return __dmul_rn(__dmul_rn(apow(s.aI, 2 * al + 1) / 3.0, p.fm2), br);
}

// ScaleFactorKernels::getSI (scalefactorkernels.h:83-119), scalar singlets: the half-step averages
// pi2AvSI, grad2AvSI, potAvSI at aI.
__device__ __forceinline__ double sf_kernel_si(const DevState &s, const SFParams &p)
{
  const double al = p.alpha;
  const double Eks = __dmul_rn(0.5 * s.pi2AvSI, ipow_d(s.aI, -6));
  const double Egs = __dmul_rn(0.5 * s.grad2AvSI, ipow_d(s.aI, -2));
  const double br = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(al - 2, Eks), __dmul_rn(al, Egs)), __dmul_rn(al - 1, 0.0)),
                              __dmul_rn(al + 1, s.potAvSI));
  return __dmul_rn(__dmul_rn(apow(s.aI, 2 * al + 1) / 3.0, p.fm2), br);
}

// Scale-factor bookkeeping of one tail (the flags of TailOp, in schedule order) given the volume
// sums of <pi^2>, <grad^2> and <V>; shared by the single-lattice and the batched tails.
__device__ __forceinline__ void tail_apply(DevState &s, const TailOp &op, const SFParams &p, double pi2s, double g2s,
                                           double pots)
{
  const double pi2 = pi2s * p.inv_n3, g2 = g2s * p.inv_n3, pot = pots * p.inv_n3;
  const double dt = p.dt;
  const uint32_t fl = op.flags;
  if (fl & T_STORE_ALL) {
    s.potAvI = pot;
    s.potAvSI = pot;
    s.pi2AvI = pi2;
    s.pi2AvSI = pi2;
    s.grad2AvI = g2;
  }
  auto write_hist = [&]() {
    double *r = op.hist + op.hist_row * kHistCols;
    r[0] = s.aI;
    r[1] = s.aDotI;
    r[2] = s.pi2AvI;
    r[3] = s.grad2AvI;
    r[4] = s.potAvI;
  };
  const bool hist = op.hist != nullptr && op.hist_row >= 0;
  if (fl & T_STORE_FIELDS) {
    s.grad2AvI = g2;
    s.potAvI = pot;
  }
  if (hist && (fl & T_HIST_EARLY)) write_hist();
  if (fl & T_STORE_PI2_I) s.pi2AvI = pi2;
  if (fl & T_STORE_PI2_LF) {
    s.pi2AvSIM = s.pi2AvSI;
    s.pi2AvSI = pi2;
    s.pi2AvI = 0.5 * (s.pi2AvSIM + s.pi2AvSI);
  }
  if (fl & T_CORRECT_ADOT) {
    // HubbleConstraint::get RHS (hubbleconstraint.h:27-36) with rho from energies.h:217-239
    const double rho = __dadd_rn(__dadd_rn(__dmul_rn(0.5 * s.pi2AvI, ipow_d(s.aI, -6)),
                                           __dmul_rn(0.5 * s.grad2AvI, ipow_d(s.aI, -2))),
                                 s.potAvI);
    const double RHS = __dmul_rn(__dmul_rn(apow(s.aI, 2 * p.alpha + 2) / 3., p.fm2), rho);
    s.aDotI = sqrt(RHS);
  }
  if (fl & T_VV_KICK_ONE) s.aDotI = __dadd_rn(s.aDotSI, __dmul_rn(__dmul_rn(dt / 2, sf_kernel(s, p)), op.w));
  if (hist && !(fl & T_HIST_EARLY)) write_hist();
  if (fl & T_LF_SYNC) s.aDotI = __dadd_rn(s.aDotSI, __dmul_rn(dt / 2.0, sf_kernel(s, p)));
  if (fl & T_LF_CTOR) s.aDotSI = __dsub_rn(s.aDotI, __dmul_rn(dt / 2.0, sf_kernel(s, p)));
  if (fl & T_LF_KICK) {
    s.aDotSIM = s.aDotSI;
    s.aDotSI = __dadd_rn(s.aDotSI, __dmul_rn(dt, sf_kernel(s, p)));
    s.aDotI = (s.aDotSIM + s.aDotSI) / 2.0;
  }
  if (fl & T_LF_DRIFT) {
    s.aIM = s.aI;
    s.aI = __dadd_rn(s.aI, __dmul_rn(dt, s.aDotSI));
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  if (fl & T_VV_KICK_HALF) s.aDotSI = __dadd_rn(s.aDotI, __dmul_rn(__dmul_rn(dt / 2, sf_kernel(s, p)), op.w2));
  if (fl & T_VV_DRIFT) {
    s.aIM = s.aI;
    s.aI = __dadd_rn(s.aI, __dmul_rn(__dmul_rn(dt, s.aDotSI), op.w2));
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  // PositionVerlet: the field averages at the half step, the momenta's, the a-kick, the second
  // a half-drift of a stage and the first of the next one
  if (fl & T_PV_STORE_SI) {
    s.grad2AvSI = g2;
    s.potAvSI = pot;
  }
  if (fl & T_PV_STORE_PI2) {
    s.pi2AvSIM = s.pi2AvI; // pi2AvIM
    s.pi2AvI = pi2;
    s.pi2AvSI = 0.5 * (s.pi2AvI + s.pi2AvSIM);
  }
  if (fl & T_PV_KICK) s.aDotI = __dadd_rn(s.aDotI, __dmul_rn(__dmul_rn(dt, sf_kernel_si(s, p)), op.w));
  if (fl & T_PV_DRIFT_A2) {
    s.aI = __dadd_rn(s.aI, __dmul_rn(__dmul_rn(dt / 2.0, s.aDotI), op.w));
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  if (fl & T_PV_DRIFT_A1) {
    s.aIM = s.aI;
    s.aI = __dadd_rn(s.aI, __dmul_rn(__dmul_rn(dt / 2.0, s.aDotI), op.w2));
    s.aSI = s.aI;
  }
  if (fl & T_FB_AIM) s.aIM = s.aI;
  if (fl & T_FB_AI) s.aI = op.fa;
  if (fl & T_FB_ASI) s.aSI = op.fb;
  if (fl & T_FB_PV_HALF) {
    s.aIM = s.aI;
    s.aI = op.fb;
    s.aSI = s.aI;
  }
  if (fl & T_FB_ADOT) s.aDotI = op.fb;
  if (fl & T_PV_MODE) // the next field drift happens before the first a half-drift of its stage
    s.drift_p = apow((fl & (T_PV_DRIFT_A1 | T_FB_PV_HALF)) ? s.aIM : s.aI, p.alpha - 3);
  else
    s.drift_p = apow(s.aSI, p.alpha - 3);
  s.kick_A = apow(s.aI, 1 + p.alpha);
  s.kick_B = apow(s.aI, 3 + p.alpha);
  if (!isfinite(s.aI) || !isfinite(s.aDotI) || !isfinite(s.aDotSI) || !isfinite(s.pi2AvI) ||
      !isfinite(s.grad2AvI) || !isfinite(s.potAvI))
    s.status = 1;
}

// The tail reduces one partial row per sweep block (8192 rows at 512^3): 1024 threads, each with
// four independent accumulators, so the loads overlap instead of waiting out the latency one by one.
constexpr int kTailThreads = 1024;

static __global__ void __launch_bounds__(kTailThreads)
    k_tail(const double *__restrict__ partials, TailOp op, DevState *__restrict__ st, SFParams p)
{
  __shared__ double smem[(kTailThreads / 32) * kRedSlots];
  griddep_wait();   // the sweep's partials and state are complete
  griddep_launch(); // the next sweep may set up its barriers meanwhile

  double v[kRedSlots] = {0, 0, 0};
  if (op.nblocks > 0) {
    double w[4][kRedSlots] = {};
    const int T = blockDim.x;
    int b = threadIdx.x;
    for (; b + 3 * T < op.nblocks; b += 4 * T) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) w[u][k] += partials[(size_t)(b + u * T) * kRedSlots + k];
    }
    for (; b < op.nblocks; b += T) {
#pragma unroll
      for (int k = 0; k < kRedSlots; ++k) w[0][k] += partials[(size_t)b * kRedSlots + k];
    }
#pragma unroll
    for (int k = 0; k < kRedSlots; ++k) v[k] = (w[0][k] + w[1][k]) + (w[2][k] + w[3][k]);
    block_reduce<kRedSlots, kTailThreads>(v, smem);
  }
  if (threadIdx.x != 0) return;
  DevState s = *st;
  tail_apply(s, op, p, v[0], v[1], v[2]);
  *st = s;
}

// Element type conversion for staged host transfers (FP32 storage from FP64 host arrays).
template <class S, class D>
__global__ void __launch_bounds__(256) k_convert(const S *__restrict__ src, D *__restrict__ dst, size_t n)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}

// Fixed-order sum of NV-slot block partials into out[NV] (measurement path).
template <int NV>
__global__ void __launch_bounds__(256) k_sum_partials(const double *__restrict__ partials, int nblocks, double *out)
{
  __shared__ double smem[(256 / 32) * NV];
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0;
#pragma unroll 5
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += partials[(size_t)b * NV + k];
  block_reduce<NV, 256>(v, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < NV; ++k) out[k] = v[k];
}

} // namespace clb
